// fi_grid.cuh -- grid-wide pieces shared by the persistent executors (fi_persist.cu,
// fi_ensemble.cu): the bounded grid barrier, the phase timeline marks and the step
// controller run by one warp.
//
// The grid barrier is an arrival counter plus a generation word.  Each wait is
// bounded: after PERSIST_SPIN_LIMIT polls the block raises the abort word and leaves,
// every other block sees the abort word at its next poll and leaves too, and the
// host reports FI_ERR_TIMEOUT.  A cooperative launch guarantees that all blocks are
// resident, so the bound is only reached if the launch is broken.
#pragma once
#include "fi_phases.cuh"

namespace fi {


// Returns false (in every thread of the block) when the barrier was abandoned.
// polls: the wait bound (PERSIST_SPIN_LIMIT unless a test lowers it).
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int nblocks, int* s_ok,
                                             long long polls = PERSIST_SPIN_LIMIT) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = bar + 1;
        volatile unsigned int* vabort = bar + 2;
        const unsigned int gen = *vgen;
        int ok = 1;
        __threadfence();
        const unsigned int prev = atomicAdd(bar, 1u);
        if (prev == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long npoll = 0;
            while (*vgen == gen) {
                if (*vabort) { ok = 0; break; }
                if (++npoll > polls) {
                    atomicExch(bar + 2, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// phase timeline (block 0, thread 0): time since the previous mark goes to phase ph
__device__ __forceinline__ void trace_mark(unsigned long long* trace, unsigned long long* last, int ph) {
    if (trace && blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned long long now = globaltimer_ns();
        trace[2 * ph] += now - *last;
        trace[2 * ph + 1] += 1;
        *last = now;
    }
}

// loop footer + header of the next attempt (finish_attempt of the per-phase kernels),
// run by the first warp: lanes 0 and 1 evaluate the controller's two powers side by side
__device__ inline void finish_attempt_warp(const Member& m, Ctl* c, double EEst) {
    const int lane = threadIdx.x & 31;
    const double base = lane == 0 ? EEst : c->qold;
    const double ex = lane == 0 ? PI_BETA1 : PI_BETA2;
    const bool pw = (EEst == EEst) && EEst != 0.0;
    const double pv = (pw && lane < 2) ? pow(base, ex) : 1.0;
    const double qold_b2 = __shfl_sync(0xffffffffu, pv, 1);
    if (lane != 0) return;
    controller_update_pw(c, EEst, pw ? pv : 0.0, pw ? qold_b2 : 1.0, m.tout);
    int active = (c->status == FI_OK);
    c->nsteps_seg += 1;
    if (c->accept_step && (c->pending_output || !(c->t < c->t_stop))) active = 0;
    if (active) {
        loopheader_prep(c);
        if (c->status != FI_OK) active = 0;
    }
    c->active = active;
    c->gate = 0;
    if (active) gate_eval(m, c, c->t + C2 * c->dt);
}

}  // namespace fi
