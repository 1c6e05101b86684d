// fi_grid.cuh -- grid-wide pieces shared by the persistent executors (fi_persist.cu,
// fi_ensemble.cu): the bounded grid barrier, the phase timeline marks and the step
// controller run by one warp.
//
// The grid barrier is one 64-bit arrival counter that only grows (zeroed by the host
// before each launch): a block adds 1 with acq_rel semantics and waits, polling with
// acquire loads, until the counter reaches the next multiple of the block count, so
// one atomic round trip and one load round trip are the whole critical path.  Each
// wait is bounded: after PERSIST_SPIN_LIMIT polls the block raises the abort word
// (bar[2]) and leaves, every other block sees the abort word at one of its next polls
// and leaves too, and the host reports FI_ERR_TIMEOUT.  A cooperative launch
// guarantees that all blocks are resident, so the bound is only reached if the launch
// is broken (or a test asks for more arrivals than blocks).
#pragma once
#include "fi_phases.cuh"

namespace fi {


// Returns false (in every thread of the block) when the barrier was abandoned.
// polls: the wait bound (PERSIST_SPIN_LIMIT unless a test lowers it).  bar: 16 bytes,
// 8-byte aligned: [0..1] the arrival counter, [2] the abort word.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned int nblocks, int* s_ok,
                                             long long polls = PERSIST_SPIN_LIMIT) {
    __syncthreads();  // the block's writes happen before thread 0's release
    if (threadIdx.x == 0) {
        unsigned long long* cnt = reinterpret_cast<unsigned long long*>(bar);
        const volatile unsigned int* vabort = bar + 2;
        unsigned long long old, cur;
        asm volatile("atom.add.acq_rel.gpu.u64 %0, [%1], 1;" : "=l"(old) : "l"(cnt) : "memory");
        const unsigned long long target = (old / nblocks + 1) * nblocks;
        int ok = 1;
        if (old + 1 != target) {
            long long npoll = 0;
            for (;;) {
                asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(cur) : "l"(cnt) : "memory");
                if (cur >= target) break;
                if (++npoll > polls) {
                    atomicExch(bar + 2, 1u);
                    ok = 0;
                    break;
                }
                if ((npoll & 63) == 0 && *vabort) {
                    ok = 0;
                    break;
                }
                if (npoll > 4096) __nanosleep(100);
            }
        }  // else: the last arrival, whose acq_rel atomic read every other block's release
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
