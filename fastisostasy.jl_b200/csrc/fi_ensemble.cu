// fi_ensemble.cu -- persistent step executor of a batched ensemble (mixed grids).
//
// One cooperative launch advances every member of an ensemble by one output segment
// each.  All members take their BS3 step attempts in lock step: an attempt is the
// sequence of phases of fi_phases.cuh over the union of the active members' tiles,
//
//   [sparse update of the gated members: conv rows | conv cols | conv rows-inverse]
//   rows_fwd(2) | cols(2) | ... | rows_inv(k4)+error norm | controller
//
// separated by grid barriers (fi_grid.cuh).  Within a phase the tiles are handed out
// in chunks of consecutive tasks by a monotonic task counter, so blocks stay busy
// whatever the mix of grid sizes and a block's tiles mostly belong to one member.
// Each block caches the descriptor, control block, twiddles and ice times of the
// member it is working on in shared memory and reloads them only when its next tile
// belongs to another member.  Per-member control (the step controller, the sparse
// gate, the call counter, the corner values) is written to the member's control block
// in global memory by exactly one block per member and phase; the next phase reads it
// after the barrier.  A member leaves the active set when its segment ends (tstop,
// output time or error); the launch ends when no member is active.
//
// Every member computes exactly what it computes alone: the phase bodies, their
// reductions and the controller are the same code on the same inputs.
#include "fi_grid.cuh"

namespace fi {

enum { K_ROWS = 0, K_COLS, K_CROW, K_CCOL, K_CROWI, K_NKIND };

// per-block plan of the current attempt
struct EnsPlan {
    int nact, ngate;
    short act[ENS_MAX_MEMBERS];    // active members, ascending
    short gated[ENS_MAX_MEMBERS];  // active members whose sparse gate is open, ascending
    int off[ENS_MAX_MEMBERS + 1];  // task-count prefix of the current phase
    short cnt[K_NKIND][ENS_MAX_MEMBERS];
};

struct EnsCache {
    Member m;
    Ctl c;
    FftPlan pl;
    FwdScalars fs;
    FwdViews fv;
    ErrTerms es;
    double c4[4];
    double uc[4];
    int cm;  // cached member (-1: none)
    int task;
    int ok;
};

// Block-wide (warp 0) exclusive prefix of cnt[kind][list[i]] into plan.off; returns the total.
__device__ int plan_prefix(EnsPlan& P, const short* list, int n, int kind) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const int per = (n + 31) / 32;
        const int i0 = lane * per, i1 = min(i0 + per, n);
        int s = 0;
        for (int i = i0; i < i1; i++) s += P.cnt[kind][list[i]];
        int incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        int run = incl - s;
        for (int i = i0; i < i1; i++) {
            P.off[i] = run;
            run += P.cnt[kind][list[i]];
        }
        if (lane == 31) P.off[n] = incl;
    }
    __syncthreads();
    return P.off[n];
}

// Active set and gated set from the members' control blocks (global memory).
__device__ void plan_members(const EnsArgs& a, EnsPlan& P, int only_gate) {
    __shared__ int s_flag[ENS_MAX_MEMBERS];
    __shared__ int s_gate[ENS_MAX_MEMBERS];
    const int tid = threadIdx.x;
    if (!only_gate) {
        for (int i = tid; i < a.nmem; i += RT) {
            const volatile Ctl* c = a.ctls[i];
            const int act = c->active;
            s_flag[i] = act;
            s_gate[i] = act ? c->gate : 0;
        }
    } else {
        for (int i = tid; i < P.nact; i += RT) {
            const volatile Ctl* c = a.ctls[P.act[i]];
            s_gate[P.act[i]] = c->gate;
        }
    }
    __syncthreads();
    if (tid == 0) {
        if (!only_gate) {
            int n = 0;
            for (int i = 0; i < a.nmem; i++)
                if (s_flag[i]) P.act[n++] = (short)i;
            P.nact = n;
        }
        int g = 0;
        for (int i = 0; i < P.nact; i++)
            if (s_gate[P.act[i]]) P.gated[g++] = P.act[i];
        P.ngate = g;
    }
    __syncthreads();
}

// Loads member m's descriptor, control block, one plan's twiddles (which: 0 x, 1 y,
// 2 padded x, 3 padded y) and, with tice_smem, the ice times.
__device__ void cache_member(const EnsArgs& a, EnsCache& C, int m, int which, unsigned char* tw_smem,
                             double* tice_smem) {
    copy_words(&C.m, &a.mems[m], sizeof(Member));
    __syncthreads();
    copy_words(&C.c, C.m.ctl, sizeof(Ctl));
    const FftPlan& p = which == 0 ? C.m.px : which == 1 ? C.m.py : which == 2 ? C.m.pMx : C.m.pMy;
    float2* tw = (float2*)tw_smem;
    const bool stage_tw = p.L <= a.tw_cap;
    if (stage_tw)
        for (int i = threadIdx.x; i < p.L; i += RT) tw[i] = p.tw32[i];
    if (tice_smem && !C.m.ice_external && C.m.K <= a.tice_cap)
        for (int i = threadIdx.x; i < C.m.K; i += RT) tice_smem[i] = C.m.t_ice[i];
    if (threadIdx.x == 0) {
        C.pl = p;
        if (stage_tw) C.pl.tw32 = tw;
        C.cm = m;
    }
    __syncthreads();
}

// Grabs the next chunk of K consecutive tasks of the current phase; returns its first
// task in every thread (>= total: done).
__device__ __forceinline__ int next_chunk(const EnsArgs& a, EnsCache& C, unsigned long long base, int K) {
    if (threadIdx.x == 0) C.task = (int)(atomicAdd(a.counter, (unsigned long long)K) - base);
    __syncthreads();
    const int t = C.task;
    __syncthreads();
    return t;
}

// tasks per grab: about two grabs per block and phase
__device__ __forceinline__ int chunk_of(int total, unsigned int G) {
    const int k = (total + 2 * (int)G - 1) / (2 * (int)G);
    return k > 0 ? k : 1;
}

// counter advance of a phase: ceil(total / K) successful grabs plus one failed grab per block
__device__ __forceinline__ unsigned long long phase_span(int total, int K, unsigned int G) {
    return ((unsigned long long)((total + K - 1) / K) + G) * (unsigned long long)K;
}

__device__ __forceinline__ int find_member(const EnsPlan& P, int n, int t) {
    int lo = 0, hi = n - 1;  // last i with off[i] <= t
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.off[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int ENS_SEQ>
__global__ void __launch_bounds__(RT, 2) k_ens(EnsArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ EnsPlan P;
    __shared__ EnsCache C;
    __shared__ double s_red[32 * 4];
    const int tid = threadIdx.x, bid = blockIdx.x;
    const unsigned int G = gridDim.x;
    unsigned char* ws = smem;
    unsigned char* tw_smem = smem + a.ws_bytes;
    double* tice_smem = (double*)(tw_smem + (size_t)a.tw_cap * sizeof(float2));
    unsigned long long base = 0;  // task-counter base of the current phase (same in every block)
    bool ok = true;
    unsigned long long* trace = a.trace;
    unsigned long long tlast = (trace && bid == 0 && tid == 0) ? globaltimer_ns() : 0ull;

    for (int i = tid; i < a.nmem; i += RT) {
        const Member& mm = a.mems[i];
        P.cnt[K_ROWS][i] = (short)mm.n_rows;
        P.cnt[K_COLS][i] = (short)mm.ncols;
        P.cnt[K_CROW][i] = (short)mm.n_crow;
        P.cnt[K_CCOL][i] = (short)mm.n_ccol;
        P.cnt[K_CROWI][i] = (short)mm.n_crowi;
    }
    // ---- segment start of every member (loop header of its first attempt) ----
    for (int i = bid; i < a.nmem; i += G) {
        cache_member(a, C, i, 0, tw_smem, nullptr);
        if (tid == 0) {
            Ctl* c = &C.c;
            int active = (c->status == FI_OK) && (c->t < c->t_stop);
            c->pending_output = 0;
            c->nsteps_seg = 0;
            if (active) {
                loopheader_prep(c);
                if (c->status != FI_OK) active = 0;
            }
            c->active = active;
            c->gate = 0;
            if (active) gate_eval(C.m, c, c->t + C2 * c->dt);
        }
        __syncthreads();
        copy_words(C.m.ctl, &C.c, sizeof(Ctl));
        __syncthreads();
    }
    ok = grid_barrier(a.bar, G, &C.ok);
    if (ok) plan_members(a, P, 0);

    while (ok && P.nact > 0) {
        for (int stage = 2; stage <= 4 && ok; stage++) {
            if (stage > 2) plan_members(a, P, 1);  // the gate of this stage was set by the columns
            if (P.ngate > 0) {
                // ---- sparse update of the gated members ----
                const int kinds[3] = {K_CROW, K_CCOL, K_CROWI};
                for (int q = 0; q < 3 && ok; q++) {
                    const int total = plan_prefix(P, P.gated, P.ngate, kinds[q]);
                    const int K = chunk_of(total, G);
                    if (tid == 0) C.cm = -1;
                    __syncthreads();
                    for (int t0 = next_chunk(a, C, base, K); t0 < total; t0 = next_chunk(a, C, base, K))
                        for (int t = t0; t < min(t0 + K, total); t++) {
                            const int gi = find_member(P, P.ngate, t);
                            const int m = P.gated[gi], tile = t - P.off[gi];
                            if (C.cm != m) cache_member(a, C, m, q == 1 ? 3 : 2, tw_smem, nullptr);
                            if (q == 0) {
                                ph_conv_rows(C.m, C.pl, ws, tile, C.m.h_conv);
                            } else if (q == 1) {
                                ph_conv_cols(C.m, C.pl, ws, tile, C.m.B_conv);
                            } else {
                                const int iue = C.c.iue;
                                ph_conv_rows_inv(C.m, C.pl, ws, tile, C.m.h_conv, iue, C.m.ctl->ue_corner[iue],
                                                 C.m.ctl->dz_corner);
                            }
                        }
                    base += phase_span(total, K, G);
                    ok = grid_barrier(a.bar, G, &C.ok);
                    trace_mark(trace, &tlast, PH_CONV_ROWS + q);
                }
                if (!ok) break;
            }
            // ---- forward rows (stages 3, 4: with the inverse rows of the previous stage) ----
            const int inv = stage > 2;
            {
                const int total = plan_prefix(P, P.act, P.nact, K_ROWS);
                const int K = chunk_of(total, G);
                if (tid == 0) C.cm = -1;
                __syncthreads();
                for (int t0 = next_chunk(a, C, base, K); t0 < total; t0 = next_chunk(a, C, base, K))
                    for (int t = t0; t < min(t0 + K, total); t++) {
                        const int ai = find_member(P, P.nact, t);
                        const int m = P.act[ai], tile = t - P.off[ai];
                        if (C.cm != m) {
                            cache_member(a, C, m, 0, tw_smem, tice_smem);
                            const double* tice =
                                (!C.m.ice_external && C.m.K <= a.tice_cap) ? tice_smem : C.m.t_ice;
                            if (tid == 0) {
                                fwd_static(C.m, C.c, stage, nullptr, tice, C.fs);
                                if (C.fs.status != FI_OK) C.m.ctl->status = C.fs.status;
                            }
                            if (tid < 4) C.uc[tid] = __ldcg(&C.m.u[C.c.ibuf][corner_index(tid, C.m.nx, C.m.ny)]);
                            if (inv) {
                                cpa_bytes(ws + C.m.fl.cpart, C.m.cpart, C.m.ncols * 32);
                                cpa_wait();
                                __syncthreads();
                                corners_from_partials((const double*)(ws + C.m.fl.cpart), C.m.ncols, C.c4);
                                __syncthreads();
                                if (tid == 0)
                                    for (int q = 0; q < 4; q++) C.c.kcorner[stage == 3 ? 2 : 3][q] = C.c4[q];
                            }
                            __syncthreads();
                            if (tid == 0) fwd_offsets(C.m, C.c, C.uc, C.fs);
                            __syncthreads();
                        }
                        const RowRanges rr = row_ranges(tile, C.m.h_rows, C.m.ny);
                        const float2* Sprev = C.m.S[stage == 4 ? 1 : 0];
                        fwd_prefetch(C.m, C.fs, ws, rr, inv, Sprev, &C.fv);
                        cpa_wait();
                        __syncthreads();
                        if (inv && tile == 0 && tid == 0)
                            for (int q = 0; q < 4; q++) C.m.ctl->kcorner[stage == 3 ? 2 : 3][q] = C.c4[q];
                        ph_rows_fwd<ENS_SEQ>(C.m, C.fs, C.fv, C.pl, ws, rr, C.m.h_rows, C.m.S[stage == 3 ? 1 : 0], inv,
                                    Sprev, stage == 3 ? C.m.k2 : C.m.k3);
                    }
                base += phase_span(total, K, G);
                if (!(ok = grid_barrier(a.bar, G, &C.ok))) break;
                trace_mark(trace, &tlast, PH_ROWS_FWD2 + 2 * (stage - 2));
            }
            // ---- columns; count the call and evaluate the gate of the next one ----
            {
                const int total = plan_prefix(P, P.act, P.nact, K_COLS);
                const int K = chunk_of(total, G);
                if (tid == 0) C.cm = -1;
                __syncthreads();
                for (int t0 = next_chunk(a, C, base, K); t0 < total; t0 = next_chunk(a, C, base, K))
                    for (int t = t0; t < min(t0 + K, total); t++) {
                        const int ai = find_member(P, P.nact, t);
                        const int m = P.act[ai], tile = t - P.off[ai];
                        if (C.cm != m) cache_member(a, C, m, 1, tw_smem, nullptr);
                        ph_cols<ENS_SEQ>(C.m, C.pl, C.m.px.tw32, ws, tile, C.m.B_cols, C.m.S[stage == 3 ? 1 : 0],
                                C.m.cpart + 4 * tile);
                        if (tile == 0 && tid == 0) {
                            Ctl* gc = C.m.ctl;
                            gc->nf += 1;
                            if (stage < 4) gate_eval(C.m, gc, C.c.t + (stage == 2 ? C3 : 1.0) * C.c.dt);
                        }
                    }
                base += phase_span(total, K, G);
                if (!(ok = grid_barrier(a.bar, G, &C.ok))) break;
                trace_mark(trace, &tlast, PH_COLS2 + 2 * (stage - 2));
            }
        }
        if (!ok) break;
        // ---- inverse rows of the last stage -> k4 and the error-norm partials ----
        {
            const int total = plan_prefix(P, P.act, P.nact, K_ROWS);
            const int K = chunk_of(total, G);
            if (tid == 0) C.cm = -1;
            __syncthreads();
            for (int t0 = next_chunk(a, C, base, K); t0 < total; t0 = next_chunk(a, C, base, K))
                for (int t = t0; t < min(t0 + K, total); t++) {
                    const int ai = find_member(P, P.nact, t);
                    const int m = P.act[ai], tile = t - P.off[ai];
                    InvLayout L;
                    if (C.cm != m) {
                        cache_member(a, C, m, 0, tw_smem, nullptr);
                        inv_layout(C.m.nx, C.m.h_rows, C.m.ncols, &L);
                        if (tid == 0) {
                            const Ctl& c = C.c;
                            const int ik = c.ik;
                            C.es.dt = c.dt; C.es.abstol = c.abstol; C.es.reltol = c.reltol;
                            C.es.cc1 = cmean(c.kcorner[ik], C.m.border_v);
                            C.es.cc2 = cmean(c.kcorner[2], C.m.border_v);
                            C.es.cc3 = cmean(c.kcorner[3], C.m.border_v);
                            C.es.up = C.m.u[c.ibuf];
                            C.es.un = C.m.u[c.ibuf ^ 1];
                            C.es.k1 = C.m.k14[ik];
                        }
                        cpa_bytes(ws + L.cpart, C.m.cpart, C.m.ncols * 32);
                        cpa_wait();
                        __syncthreads();
                        corners_from_partials((const double*)(ws + L.cpart), C.m.ncols, C.c4);
                        __syncthreads();
                    } else {
                        inv_layout(C.m.nx, C.m.h_rows, C.m.ncols, &L);
                    }
                    inv_prefetch(C.m, C.m.S[0], ws, tile, C.m.h_rows, &C.es);
                    cpa_wait();
                    __syncthreads();
                    const int ik = C.c.ik;
                    const double sum =
                        ph_rows_inv<ENS_SEQ>(C.m, C.pl, ws, s_red, tile, C.m.h_rows, C.m.k14[ik ^ 1], &C.es, C.c4);
                    if (tid == 0) {
                        C.m.partial[tile] = sum;
                        if (tile == 0)
                            for (int q = 0; q < 4; q++) C.m.ctl->kcorner[ik ^ 1][q] = C.c4[q];
                    }
                }
            base += phase_span(total, K, G);
            if (!(ok = grid_barrier(a.bar, G, &C.ok))) break;
            trace_mark(trace, &tlast, PH_ROWS_INV4);
        }
        // ---- step controllers: member act[i] on block i mod G ----
        for (int i = bid; i < P.nact; i += G) {
            cache_member(a, C, P.act[i], 0, tw_smem, nullptr);
            if (tid < 32) {
                const double acc = partials_sum(C.m.partial, C.m.n_rows);
                finish_attempt_warp(C.m, &C.c, sqrt(acc / ((double)C.m.nx * C.m.ny)));
            }
            __syncthreads();
            copy_words(C.m.ctl, &C.c, sizeof(Ctl));
            __syncthreads();
        }
        if (!(ok = grid_barrier(a.bar, G, &C.ok))) break;
        trace_mark(trace, &tlast, PH_CONTROLLER);
        plan_members(a, P, 0);
    }
    if (!ok && tid == 0) atomicExch(a.bar + 2, 1u);
}

// Shared-memory layout: [phase workspace][one twiddle table][ice times]
size_t ens_layout(const Member* host_mems, int n, EnsArgs* a) {
    size_t ws = 0;
    int twc = 0, tic = 0;
    for (int i = 0; i < n; i++) {
        const Member& m = host_mems[i];
        const size_t q[] = {(size_t)m.fl.bytes, ws_cols(m.ny, m.B_cols), ws_rows_inv(m.nx, m.h_rows, m.ncols),
                            ws_conv_rows(m.Mx, m.h_conv), ws_conv_cols(m.My, m.B_conv)};
        for (size_t v : q) ws = v > ws ? v : ws;
        const int L[] = {m.nx, m.ny, m.Mx, m.My};
        for (int v : L) twc = v > twc ? v : twc;
        if (!m.ice_external && m.K <= TICE_MAX) tic = m.K > tic ? m.K : tic;
    }
    a->ws_bytes = (int)al16(ws);
    a->tw_cap = twc;
    a->tice_cap = tic;
    return (size_t)a->ws_bytes + (size_t)twc * sizeof(float2) + (size_t)tic * sizeof(double);
}

// The ensemble kernel whose row and column transforms dispatch per task on the
// member's schedule (compiled sequences of the grids 64 .. 256), or with dispatch = 0
// the one that runs every plan's runtime passes.
const void* ens_kernel(int dispatch) {
    return dispatch ? (const void*)k_ens<SEQ_DISPATCH> : (const void*)k_ens<0>;
}

}  // namespace fi
