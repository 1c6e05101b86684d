// fi_persist.cu -- persistent BS3 step executor of the fused FP32 form.
//
// One cooperative launch runs one output segment: every BS3 step attempt
// (perform_step! of BS3, src/integrators.jl:154-173, with OrdinaryDiffEq's PI
// controller) until t reaches the next tstop, an output time is passed, or an error
// stops the integration.  The phases of fi_phases.cuh run back to back, separated by
// a grid barrier:
//
//   [sparse update: conv rows | conv cols | conv rows-inverse]   when the gate opens
//   rows_fwd(2) | cols(2) | rows_inv(k2)+rows_fwd(3) | cols(3) |
//   rows_inv(k3)+rows_fwd(4) | cols(4) | rows_inv(k4)+error norm | controller
//
// Every block keeps its own copy of the control block in shared memory and runs the
// step controller, the sparse-update gate and the corner bookkeeping itself, on the
// same inputs in the same order, so all copies stay identical without any exchange;
// block 0 writes its copy back when the segment ends.  Values produced by one block
// and needed by all (the error-norm partials per row tile, the convolution corner
// values) travel through global memory across a barrier.  The member descriptor,
// the four transform plans with their twiddles and the ice-time table are staged in
// shared memory once per launch.
//
// The grid barrier, the phase timeline marks and the warp-level controller are in
// fi_grid.cuh.
#include "fi_grid.cuh"

namespace fi {

// The executor body, inlined into two kernels whose register budgets differ: k_persist
// for two blocks per SM (64 registers a thread) where shared memory fits two blocks,
// k_persist1 for one (no spills) where it fits only one.
// SX / SY: the compiled radix sequences of the row and column transforms (0: the
// plans' runtime passes).
template <int SX, int SY, int WIDE>
__device__ __forceinline__ void persist_body(const PersistArgs& a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Member sm;
    __shared__ Ctl sc;
    __shared__ FftPlan pl[4];
    __shared__ FwdScalars fs;
    __shared__ FwdViews fv;
    __shared__ ErrTerms es;
    __shared__ double s_red[32 * 4];
    __shared__ double s_uc[4];
    __shared__ double s_c4[4];
    __shared__ int s_ok;
    const int tid = threadIdx.x, bid = blockIdx.x;
    const unsigned int G = gridDim.x;
    const unsigned int GB = G + a.bar_extra;  // arrivals a grid barrier waits for

    // ---- stage the member, the control block, the plans and the ice times ----
    copy_words(&sm, a.mem, sizeof(Member));
    __syncthreads();
    copy_words(&sc, sm.ctl, sizeof(Ctl));
    float2* tw = (float2*)(smem + a.ws_bytes);
    for (int q = 0; q < 4; q++) {
        const FftPlan& p = q == 0 ? sm.px : q == 1 ? sm.py : q == 2 ? sm.pMx : sm.pMy;
        float2* dst = a.tw_off[q] >= 0 ? tw + a.tw_off[q] : nullptr;  // padded lengths: global twiddles
        if (dst)
            for (int i = tid; i < p.L; i += RT) dst[i] = p.tw32[i];
        if (tid == 0) {
            pl[q] = p;
            if (dst) pl[q].tw32 = dst;
        }
    }
    const double* tice = sm.t_ice;
    if (a.tice_off >= 0 && !sm.ice_external) {
        double* st = (double*)(tw + a.tice_off);
        for (int i = tid; i < sm.K; i += RT) st[i] = sm.t_ice[i];
        tice = st;
    }
    // ---- segment start: loop header of the first attempt ----
    if (tid == 0) {
        Ctl* c = &sc;
        int active = (c->status == FI_OK) && (c->t < c->t_stop);
        c->pending_output = 0;
        c->nsteps_seg = 0;
        if (active) {
            loopheader_prep(c);
            if (c->status != FI_OK) active = 0;
        }
        c->active = active;
        c->gate = 0;
        if (active) gate_eval(sm, c, c->t + C2 * c->dt);
    }
    __syncthreads();
    const Member& m = sm;
    const int nx = m.nx, ny = m.ny;
    bool ok = true;
    unsigned long long* trace = a.trace;
    unsigned long long tlast = (trace && bid == 0 && tid == 0) ? globaltimer_ns() : 0ull;
    if (tid < 4) s_uc[tid] = __ldcg(&m.u[sc.ibuf][corner_index(tid, nx, ny)]);
    __syncthreads();

    while (sc.active && ok) {
        for (int stage = 2; stage <= 4 && ok; stage++) {
            if (sc.gate) {
                // sparse update: the convolutions read the column anomalies of the last call
                for (int t = bid; t < a.n_crow; t += G) ph_conv_rows(m, pl[2], smem, t, a.h_conv);
                if (!(ok = grid_barrier(a.bar, GB, &s_ok, a.polls))) break;
                trace_mark(trace, &tlast, PH_CONV_ROWS);
                for (int t = bid; t < a.n_ccol; t += G) ph_conv_cols(m, pl[3], smem, t, a.B_conv);
                if (!(ok = grid_barrier(a.bar, GB, &s_ok, a.polls))) break;
                trace_mark(trace, &tlast, PH_CONV_COLS);
                const int iue = sc.iue;
                for (int t = bid; t < a.n_crowi; t += G)
                    ph_conv_rows_inv(m, pl[2], smem, t, a.h_conv, iue, m.ctl->ue_corner[iue], m.ctl->dz_corner);
                if (!(ok = grid_barrier(a.bar, GB, &s_ok, a.polls))) break;
                trace_mark(trace, &tlast, PH_CONV_ROWS_INV);
                if (tid < 4) {
                    const volatile double* ue_c = m.ctl->ue_corner[iue];
                    const volatile double* dz_c = m.ctl->dz_corner;
                    sc.ue_corner[iue][tid] = ue_c[tid];
                    sc.dz_corner[tid] = dz_c[tid];
                }
                __syncthreads();
            }
            // ---- forward rows (stages 3, 4: with the inverse rows of the previous stage) ----
            const int inv = stage > 2;
            const float2* Sprev = m.S[stage == 4 ? 1 : 0];
            float2* Sout = m.S[stage == 3 ? 1 : 0];
            float* kdst = stage == 3 ? m.k2 : m.k3;
            int t = bid;
            // warps 0-3 sum the previous stage's corner partials while a thread of warp 4
            // sets up the stage's scalars; then the views and the corner offsets
            if (inv) corners_from_partials_g(m.cpart, m.ncols, s_c4);
            if (tid == 128) {
                fwd_static(m, sc, stage, nullptr, tice, fs);
                if (fs.status != FI_OK) sc.status = fs.status;
            }
            __syncthreads();
            if (t < a.n_rows) fwd_prefetch(m, fs, smem, row_ranges(t, a.h_rows, ny), inv, Sprev, &fv);
            if (tid == 0) {
                if (inv)
                    for (int q = 0; q < 4; q++) sc.kcorner[stage == 3 ? 2 : 3][q] = s_c4[q];
                fwd_offsets(m, sc, s_uc, fs);
            }
            cpa_wait();
            __syncthreads();
            while (t < a.n_rows) {
                ph_rows_fwd<SX, WIDE>(m, fs, fv, pl[0], smem, row_ranges(t, a.h_rows, ny), a.h_rows, Sout, inv, Sprev, kdst);
                t += G;
                if (t < a.n_rows) {
                    fwd_prefetch(m, fs, smem, row_ranges(t, a.h_rows, ny), inv, Sprev, &fv);
                    cpa_wait();
                    __syncthreads();
                }
            }
            if (!(ok = grid_barrier(a.bar, GB, &s_ok, a.polls))) break;
            trace_mark(trace, &tlast, PH_ROWS_FWD2 + 2 * (stage - 2));
            // ---- columns; count the call and evaluate the gate of the next one ----
            for (int tc = bid; tc < a.n_cols; tc += G)
                ph_cols<SY>(m, pl[1], pl[0].tw32, smem, tc, a.B_cols, Sout, m.cpart + 4 * tc);
            if (tid == 0) {
                sc.nf += 1;
                if (stage < 4) gate_eval(m, &sc, sc.t + (stage == 2 ? C3 : 1.0) * sc.dt);
            }
            if (!(ok = grid_barrier(a.bar, GB, &s_ok, a.polls))) break;
            trace_mark(trace, &tlast, PH_COLS2 + 2 * (stage - 2));
        }
        if (!ok) break;
        // ---- inverse rows of the last stage -> k4 and the embedded error norm ----
        {
            const int ik = sc.ik;
            if (tid == 0) {
                ErrTerms& e = es;
                e.dt = sc.dt; e.abstol = sc.abstol; e.reltol = sc.reltol;
                e.cc1 = cmean(sc.kcorner[ik], m.border_v);
                e.cc2 = cmean(sc.kcorner[2], m.border_v);
                e.cc3 = cmean(sc.kcorner[3], m.border_v);
                e.up = m.u[sc.ibuf];
                e.un = m.u[sc.ibuf ^ 1];
                e.k1 = m.k14[ik];
            }
            __syncthreads();
            InvLayout L;
            inv_layout(nx, a.h_rows, m.ncols, &L);
            int t = bid;
            if (t < a.n_rows) inv_prefetch(m, m.S[0], smem, t, a.h_rows, &es);
            corners_from_partials_g(m.cpart, m.ncols, s_c4);
            cpa_wait();
            __syncthreads();
            while (t < a.n_rows) {
                const double sum = ph_rows_inv<SX>(m, pl[0], smem, s_red, t, a.h_rows, m.k14[ik ^ 1], &es, s_c4);
                if (tid == 0) m.partial[t] = sum;
                t += G;
                if (t < a.n_rows) {
                    inv_prefetch(m, m.S[0], smem, t, a.h_rows, &es);
                    cpa_wait();
                    __syncthreads();
                }
            }
            if (tid == 0)
                for (int q = 0; q < 4; q++) sc.kcorner[ik ^ 1][q] = s_c4[q];
        }
        if (!(ok = grid_barrier(a.bar, GB, &s_ok, a.polls))) break;
        trace_mark(trace, &tlast, PH_ROWS_INV4);
        // ---- step controller, replicated: the partials in a fixed order per lane ----
        if (tid < 32) {
            const double acc = partials_sum(m.partial, a.n_rows);
            finish_attempt_warp(m, &sc, sqrt(acc / ((double)nx * ny)));
        }
        __syncthreads();
        if (tid < 4 && sc.active) s_uc[tid] = __ldcg(&m.u[sc.ibuf][corner_index(tid, nx, ny)]);
        __syncthreads();
        trace_mark(trace, &tlast, PH_CONTROLLER);
    }
    if (!ok && tid == 0) sc.status = FI_ERR_TIMEOUT;
    __syncthreads();
    if (bid == 0) copy_words(m.ctl, &sc, sizeof(Ctl));
}

// Shared-memory layout of the persistent kernel: [phase workspace][x twiddles]
// [y twiddles][ice times]; the padded-length plans of the sparse update read their
// twiddles from global memory.
size_t persist_layout(int nx, int ny, int Mx, int My, int K, int fwd_bytes, int h_rows, int ncols, int B_cols,
                      int h_conv, int B_conv, PersistArgs* a) {
    size_t ws = (size_t)fwd_bytes;
    const size_t others[] = {ws_cols(ny, B_cols), ws_rows_inv(nx, h_rows, ncols), ws_conv_rows(Mx, h_conv),
                             ws_conv_cols(My, B_conv)};
    for (size_t q : others) ws = q > ws ? q : ws;
    a->ws_bytes = (int)ws;
    a->tw_off[0] = 0;
    a->tw_off[1] = nx;
    a->tw_off[2] = -1;
    a->tw_off[3] = -1;
    const int ntw = nx + ny;
    a->tice_off = (K <= TICE_MAX) ? ntw : -1;
    return ws + (size_t)ntw * sizeof(float2) + (K <= TICE_MAX ? (size_t)K * sizeof(double) : 0);
}

template <int SX, int SY>
__global__ void __launch_bounds__(RT, 2) k_persist(PersistArgs a) { persist_body<SX, SY, 0>(a); }
template <int SX, int SY>
__global__ void __launch_bounds__(RT, 1) k_persist1(PersistArgs a) { persist_body<SX, SY, 1>(a); }

// The compiled (row, column) sequence pairs: the tuned schedules of the square grids of
// the benchmark configurations (350 = 5*5*2*7, 1024 = 8*4*8*4) and the runtime passes.
const void* persist_kernel(int seqx, int seqy, int minb) {
#define FI_PERSIST_PAIR(X, Y)                                                              \
    if (seqx == X && seqy == Y)                                                            \
        return minb == 1 ? (const void*)k_persist1<X, Y> : (const void*)k_persist<X, Y>;
    FI_PERSIST_PAIR(5527, 5527)
    FI_PERSIST_PAIR(8484, 8484)
#undef FI_PERSIST_PAIR
    return minb == 1 ? (const void*)k_persist1<0, 0> : (const void*)k_persist<0, 0>;
}

}  // namespace fi
