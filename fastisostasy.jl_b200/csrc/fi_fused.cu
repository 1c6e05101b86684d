// fi_fused.cu -- FP32 fused kernels of the LV-ELVA right-hand side and BS3 step, one
// kernel per phase (fi_phases.cuh).  They serve the host-driven right-hand sides
// (fi_rhs, init_problem!, the FSAL evaluations and the initial-dt probe), the
// CUDA-graph step executor and per-phase timing; fi_persist.cu runs the same phases
// in one persistent launch per output segment.
//
// One right-hand side (update_diagnostics!, src/simulation.jl:335-393) is:
//   k_rows_fwd  [stages 3/4: inverse row FFT of the previous stage's spectrum for the
//               tile rows plus a 2-row halo -> k_{s-1}] -> stage state -> column
//               anomalies -> flexure operator -> times K/(2 eta) -> real row FFT.
//   k_cols      column FFT, multiply by spy/(nx ny R|k|) with DC zeroed, inverse
//               column FFT; counts the call and evaluates the sparse-update gate of
//               the next one.
//   k_rows_inv  (last stage of a step / host-driven calls) inverse real row FFT ->
//               dudt in physical space; for stage 4 the embedded BS3 error norm and
//               the step controller (last block of the grid).
// The dudt corner BC (deformation.jl:101) is evaluated directly from the spectrum
// (corner values of an inverse real DFT) and applied by every consumer.
// The sparse elastic / sea-surface update (deformation.jl:175-184,
// sealevel.jl:173-201, convolutions.jl:134-143) is k_conv_rows, k_conv_cols,
// k_conv_rows_inv, gated per call on the device.
//
// Every kernel starts by staging its member descriptor, control block, transform
// plan with twiddles (and the ice-time table) in shared memory with all threads, so
// the dependent global round trips per launch stay at three.
#include "fi_phases.cuh"

namespace fi {

// ---------------------------------------------------------------------------
// kernel head: member + control block + plan (+ twiddles, ice times, state corners)
// ---------------------------------------------------------------------------
struct KHead {
    Member m;
    Ctl c;
    FftPlan plan;
    double ucorn[2][4];
};

// which: 0 = rows (nx), 1 = columns (ny), 2 = padded rows (Mx), 3 = padded columns (My).
// stw: shared twiddle table (plan.L entries) or null; stice: shared ice times or null;
// ucorn: 1 = the corners of both state buffers, 2 = of uin.  Returns ctl->active.
__device__ bool head_load(KHead& hd, const Member* __restrict__ mems, const Task& tk, int which, float2* stw,
                          double* stice, int ucorn, const double* uin) {
    const int tid = threadIdx.x, nth = blockDim.x;
    copy_words(&hd.m, &mems[tk.member], sizeof(Member));
    __syncthreads();
    const Member& m = hd.m;
    const FftPlan& p = which == 0 ? m.px : which == 1 ? m.py : which == 2 ? m.pMx : m.pMy;
    copy_words(&hd.c, m.ctl, sizeof(Ctl));
    if (stw)
        for (int i = tid; i < p.L; i += nth) stw[i] = p.tw32[i];
    if (stice && !m.ice_external)
        for (int i = tid; i < m.K; i += nth) stice[i] = m.t_ice[i];
    if (ucorn && tid < 8) {
        const int b = tid >> 2, q = tid & 3;
        const double* u = (ucorn == 2) ? uin : m.u[b];
        hd.ucorn[b][q] = (ucorn == 2 && b == 1) ? 0.0 : u[corner_index(q, m.nx, m.ny)];
    }
    if (tid == 0) {
        hd.plan = p;
        if (stw) hd.plan.tw32 = stw;
    }
    __syncthreads();
    return hd.c.active != 0;
}

// ---------------------------------------------------------------------------
// gate for a host-driven right-hand side at time t (stage 0/1 calls)
// ---------------------------------------------------------------------------
__global__ void k_gate(const Member* __restrict__ mems, int nmem, double t, int use_ctl_t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmem) return;
    const Member& m = mems[i];
    Ctl* c = m.ctl;
    c->active = (c->status == FI_OK);
    if (!c->active) return;
    c->t_call = use_ctl_t ? c->t : t;
    gate_eval(m, c, c->t_call);
}

// ---------------------------------------------------------------------------
// shared-memory sizes: [phase workspace][twiddles][ice times]
// ---------------------------------------------------------------------------
size_t rows_fwd_smem(int ws_bytes, int nx, int K) {
    return (size_t)ws_bytes + (size_t)nx * sizeof(float2) + (K <= TICE_MAX ? (size_t)K * sizeof(double) : 0);
}
size_t cols_smem(int ny, int B) { return ws_cols(ny, B) + (size_t)ny * sizeof(float2); }
size_t rows_inv_smem(int nx, int h, int ncols) { return ws_rows_inv(nx, h, ncols) + (size_t)nx * sizeof(float2); }
size_t conv_rows_smem(int Mx, int h) { return ws_conv_rows(Mx, h) + (size_t)Mx * sizeof(float2); }
size_t conv_cols_smem(int My, int B) { return ws_conv_cols(My, B) + (size_t)My * sizeof(float2); }

// ---------------------------------------------------------------------------
// forward rows.  stage 0: uin at t_call; stage 1: the state at t_call; stages 2-4:
// BS3 stage vectors; inv_prev (stages 3, 4) fuses the previous stage's inverse rows.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(RT, 2)
k_rows_fwd(const Member* __restrict__ mems, const Task* __restrict__ tasks, int stage, int h, const double* uin,
           int inv_prev) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    __shared__ FwdScalars fs;
    __shared__ FwdViews fv;
    __shared__ double s_c4[4];
    const Task tk = tasks[blockIdx.x];
    {
        // the shared layout needs nx, K and the workspace size before the head is staged
        const Member* mp = &mems[tk.member];
        const int nx0 = mp->nx, K0 = mp->K;
        float2* stw = (float2*)(smem + mp->fl.bytes);
        double* stice = (K0 <= TICE_MAX) ? (double*)(stw + nx0) : nullptr;
        if (!head_load(hd, mems, tk, 0, stw, stice, stage == 0 ? 2 : 1, uin)) return;
    }
    const Member& m = hd.m;
    Ctl* ctl = m.ctl;
    const int tid = threadIdx.x;
    const float2* Sprev = m.S[stage == 4 ? 1 : 0];
    float2* Sout = m.S[stage == 3 ? 1 : 0];
    const RowRanges rr = row_ranges(tk.tile, h, m.ny);
    const double* tice = m.K <= TICE_MAX ? (const double*)((float2*)(smem + m.fl.bytes) + m.nx) : m.t_ice;
    if (tid == 0) {
        fwd_static(m, hd.c, stage, uin, tice, fs);
        if (fs.status != FI_OK && tk.tile == 0) ctl->status = fs.status;
    }
    __syncthreads();
    fwd_prefetch(m, fs, smem, rr, inv_prev, Sprev, &fv);
    if (inv_prev) cpa_bytes(smem + m.fl.cpart, m.cpart, m.ncols * 32);
    cpa_wait();
    __syncthreads();
    if (inv_prev) {
        corners_from_partials((const double*)(smem + m.fl.cpart), m.ncols, s_c4);
        __syncthreads();
        if (tid == 0) {
            const int slot = stage == 3 ? 2 : 3;
            for (int q = 0; q < 4; q++) hd.c.kcorner[slot][q] = s_c4[q];
            if (tk.tile == 0)
                for (int q = 0; q < 4; q++) ctl->kcorner[slot][q] = s_c4[q];
        }
    }
    if (tid == 0) fwd_offsets(m, hd.c, hd.ucorn[stage == 0 ? 0 : hd.c.ibuf], fs);
    __syncthreads();
    ph_rows_fwd(m, fs, fv, hd.plan, smem, rr, h, Sout, inv_prev, Sprev, stage == 3 ? m.k2 : m.k3);
}

// ---------------------------------------------------------------------------
// columns.  next_stage (3 or 4): evaluates the sparse gate of the next right-hand
// side.  Every right-hand side passes here once: it is counted here.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(RT, 2)
k_cols(const Member* __restrict__ mems, const Task* __restrict__ tasks, int B, int next_stage,
       cudaGraphConditionalHandle h_gate) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    const Task tk = tasks[blockIdx.x];
    {
        const int ny0 = mems[tk.member].ny;
        float2* stw = (float2*)(smem + ws_cols(ny0, B));
        if (!head_load(hd, mems, tk, 1, stw, nullptr, 0, nullptr)) return;
    }
    const Member& m = hd.m;
    Ctl* ctl = m.ctl;
    if (threadIdx.x == 0 && tk.tile == 0) {
        ctl->nf += 1;
        if (next_stage >= 3) {
            const int g = gate_eval(m, ctl, hd.c.t + (next_stage == 3 ? C3 : 1.0) * hd.c.dt);
            if (h_gate) cudaGraphSetConditional(h_gate, g);
        }
    }
    ph_cols(m, hd.plan, m.px.tw32, smem, tk.tile, B, m.S[next_stage == 4 ? 1 : 0], m.cpart + 4 * tk.tile);
}

// ---------------------------------------------------------------------------
// inverse rows of the last stage; stage 4: embedded BS3 error norm and the step
// controller (last block); stages 0/1: output to vout / k1.
// ---------------------------------------------------------------------------
__device__ void finish_attempt(const Member& m, Ctl* c, double EEst, cudaGraphConditionalHandle h_gate,
                               cudaGraphConditionalHandle h_loop) {
    controller_update(c, EEst, m.tout);
    int active = (c->status == FI_OK);
    c->nsteps_seg += 1;
    if (c->accept_step && (c->pending_output || !(c->t < c->t_stop))) active = 0;
    if (active) {
        loopheader_prep(c);
        if (c->status != FI_OK) active = 0;
    }
    c->active = active;
    int g = 0;
    if (active) g = gate_eval(m, c, c->t + C2 * c->dt);
    if (h_gate) cudaGraphSetConditional(h_gate, g);
    if (h_loop) cudaGraphSetConditional(h_loop, active);
}

__global__ void __launch_bounds__(RT, 2)
k_rows_inv(const Member* __restrict__ mems, const Task* __restrict__ tasks, int stage, int h, float* vout,
           double* cout, cudaGraphConditionalHandle h_gate, cudaGraphConditionalHandle h_loop) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    __shared__ double s_red[32 * 4];
    __shared__ double s_c4[4];
    __shared__ int s_last;
    const Task tk = tasks[blockIdx.x];
    {
        const Member* mp = &mems[tk.member];
        float2* stw = (float2*)(smem + ws_rows_inv(mp->nx, h, mp->ncols));
        if (!head_load(hd, mems, tk, 0, stw, nullptr, 0, nullptr)) return;
    }
    const Member& m = hd.m;
    const Ctl& c = hd.c;
    Ctl* ctl = m.ctl;
    const int tid = threadIdx.x;
    const int ik = c.ik;
    int slot;
    float* dst;
    if (stage == 0) { slot = -1; dst = vout; }
    else if (stage == 1) { slot = ik; dst = m.k14[ik]; }
    else { slot = ik ^ 1; dst = m.k14[ik ^ 1]; }
    __shared__ ErrTerms e;
    if (stage == 4 && tid == 0) {
        e.dt = c.dt; e.abstol = c.abstol; e.reltol = c.reltol;
        e.cc1 = cmean(c.kcorner[ik], m.border_v);
        e.cc2 = cmean(c.kcorner[2], m.border_v);
        e.cc3 = cmean(c.kcorner[3], m.border_v);
        e.up = m.u[c.ibuf];
        e.un = m.u[c.ibuf ^ 1];
        e.k1 = m.k14[ik];
    }
    __syncthreads();
    InvLayout L;
    inv_layout(m.nx, h, m.ncols, &L);
    inv_prefetch(m, m.S[0], smem, tk.tile, h, stage == 4 ? &e : nullptr);
    cpa_bytes(smem + L.cpart, m.cpart, m.ncols * 32);
    cpa_wait();
    __syncthreads();
    corners_from_partials((const double*)(smem + L.cpart), m.ncols, s_c4);
    __syncthreads();
    const double sum = ph_rows_inv(m, hd.plan, smem, s_red, tk.tile, h, dst, stage == 4 ? &e : nullptr, s_c4);
    if (stage != 4) {
        if (tk.tile == 0 && tid == 0) {
            double* cdst = (stage == 0) ? cout : ctl->kcorner[slot];
            for (int q = 0; q < 4; q++) cdst[q] = s_c4[q];
        }
        return;
    }
    // stage 4: error-norm reduction over the member's row tiles, last block decides
    if (tid == 0) {
        m.partial[tk.tile] = sum;
        __threadfence();
        const unsigned int ntiles = (unsigned int)((m.ny + h - 1) / h);
        const unsigned int prev = atomicAdd(&ctl->arrive, 1u);
        s_last = (prev == ntiles - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        const int ntiles = (m.ny + h - 1) / h;
        if (tid < 32) {
            const double acc = partials_sum(m.partial, ntiles);
            if (tid == 0) {
                ctl->arrive = 0;
                for (int q = 0; q < 4; q++) ctl->kcorner[slot][q] = s_c4[q];
                const double EEst = sqrt(acc / ((double)m.nx * m.ny));
                finish_attempt(m, ctl, EEst, h_gate, h_loop);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// sparse update: padded linear convolutions of the elastic (channel A) and
// sea-surface (channel B) loads, crop + raw corner values
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(RT, 2)
k_conv_rows(const Member* __restrict__ mems, const Task* __restrict__ tasks, int h) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    const Task tk = tasks[blockIdx.x];
    {
        const int Mx0 = mems[tk.member].Mx;
        float2* stw = (float2*)(smem + ws_conv_rows(Mx0, h));
        if (!head_load(hd, mems, tk, 2, stw, nullptr, 0, nullptr)) return;
    }
    if (!hd.c.gate) return;
    ph_conv_rows(hd.m, hd.plan, smem, tk.tile, h);
}

__global__ void __launch_bounds__(RT, 2)
k_conv_cols(const Member* __restrict__ mems, const Task* __restrict__ tasks, int B) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    const Task tk = tasks[blockIdx.x];
    {
        const int My0 = mems[tk.member].My;
        float2* stw = (float2*)(smem + ws_conv_cols(My0, B));
        if (!head_load(hd, mems, tk, 3, stw, nullptr, 0, nullptr)) return;
    }
    if (!hd.c.gate) return;
    ph_conv_cols(hd.m, hd.plan, smem, tk.tile, B);
}

__global__ void __launch_bounds__(RT, 2)
k_conv_rows_inv(const Member* __restrict__ mems, const Task* __restrict__ tasks, int h) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    const Task tk = tasks[blockIdx.x];
    {
        const int Mx0 = mems[tk.member].Mx;
        float2* stw = (float2*)(smem + ws_conv_rows(Mx0, h));
        if (!head_load(hd, mems, tk, 2, stw, nullptr, 0, nullptr)) return;
    }
    if (!hd.c.gate) return;
    Ctl* ctl = hd.m.ctl;
    const int iue = hd.c.iue;
    ph_conv_rows_inv(hd.m, hd.plan, smem, tk.tile, h, iue, ctl->ue_corner[iue], ctl->dz_corner);
}

// segment start: loop header of the first attempt after the host set t_stop
__global__ void k_segment_start(const Member* __restrict__ mems, int nmem, cudaGraphConditionalHandle h_gate,
                                cudaGraphConditionalHandle h_loop) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmem) return;
    const Member& m = mems[i];
    Ctl* c = m.ctl;
    int active = (c->status == FI_OK) && (c->t < c->t_stop);
    c->pending_output = 0;
    c->nsteps_seg = 0;
    if (active) {
        loopheader_prep(c);
        if (c->status != FI_OK) active = 0;
    }
    c->active = active;
    int g = 0;
    if (active) g = gate_eval(m, c, c->t + C2 * c->dt);
    if (nmem == 1) {
        if (h_gate) cudaGraphSetConditional(h_gate, g);
        if (h_loop) cudaGraphSetConditional(h_loop, active);
    }
}

// ---------------------------------------------------------------------------
// initial-dt heuristic helpers (ode_determine_initdt) for FP64 state and raw FP32
// derivatives with a corner offset c = mean(corners) - border
// ---------------------------------------------------------------------------
__global__ void kf_initdt_norms(const double* u, const float* v, const double* vc, double border, double abstol,
                                double reltol, double* partial, size_t n) {
    __shared__ double red[64];
    const double c = cmean(vc, border);
    double s0 = 0.0, s1 = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double sk = abstol + fabs(u[i]) * reltol;
        const double a = u[i] / sk, b = ((double)v[i] - c) / sk;
        s0 += a * a;
        s1 += b * b;
    }
    double w[2] = {s0, s1};
    block_sum<2>(w, red);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = w[0]; partial[2 * blockIdx.x + 1] = w[1]; }
}

__global__ void kf_initdt_u1(double* u1, const double* u, const float* v, const double* vc, double border,
                             double dt0, size_t n) {
    const double c = cmean(vc, border);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        u1[i] = u[i] + dt0 * ((double)v[i] - c);
}

__global__ void kf_initdt_d2(const double* u, const float* v0, const double* c0p, const float* v1,
                             const double* c1p, double border, double abstol, double reltol, double* partial,
                             size_t n) {
    __shared__ double red[64];
    const double c0 = cmean(c0p, border), c1 = cmean(c1p, border);
    double s = 0.0, eq = 1.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double sk = abstol + fabs(u[i]) * reltol;
        const double f0 = (double)v0[i] - c0, f1 = (double)v1[i] - c1;
        const double a = (f1 - f0) / sk;
        s += a * a;
        if (f0 != f1) eq = 0.0;
    }
    double w[2] = {s, eq};
    block_sum<2>(w, red);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = w[0]; partial[2 * blockIdx.x + 1] = w[1]; }
}

}  // namespace fi
