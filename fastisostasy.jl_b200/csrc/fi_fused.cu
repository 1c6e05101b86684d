// fi_fused.cu -- FP32 fused kernels of the LV-ELVA right-hand side and BS3 step.
//
// One right-hand side (update_diagnostics!, src/simulation.jl:335-393) is:
//   k_rows_fwd  [stages 3/4: inverse row FFT of the previous stage's spectrum for the
//               tile rows plus a 2-row halo -> k_{s-1}] -> stage state
//               u = uprev + dt*sum(a_sj k_j) in FP64 -> corner BC
//               (boundary_conditions.jl:144-148) -> column anomalies
//               (loads.jl:31-106, topography.jl:30-39) -> flexure operator
//               rhs = -g sigma_full + dxx Mxx + 2 dxy Mxy + dyy Myy with the CPU edge
//               rules (deformation.jl:110-131, derivatives.jl:48-191; u-derivatives in
//               FP64, moment derivatives in FP32) -> times K/(2 eta) -> real row FFT
//               (two rows per complex FFT).
//   k_cols      column FFT, multiply by spy/(nx ny R|k|) with DC zeroed, inverse
//               column FFT (deformation.jl:95-98, solidearth.jl:222); counts the call
//               and evaluates the sparse-update gate of the next one.
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
#include "fi_device.cuh"
#include "fi_kernels.h"

namespace fi {

constexpr int RT = ROW_THREADS, TX = 128, TY = RT / TX;

// ---------------------------------------------------------------------------
// kernel head: member + control block + plan (+ twiddles, ice times, state corners)
// ---------------------------------------------------------------------------
struct KHead {
    Member m;
    Ctl c;
    FftPlan plan;
    double ucorn[2][4];
};

__device__ __forceinline__ void copy_words(void* dst, const void* src, int bytes) {
    const unsigned long long* s = (const unsigned long long*)src;
    unsigned long long* d = (unsigned long long*)dst;
    for (int i = threadIdx.x; i < bytes / 8; i += blockDim.x) d[i] = s[i];
}

__device__ __forceinline__ int corner_index(int q, int nx, int ny) {
    return q == 0 ? 0 : q == 1 ? nx - 1 : q == 2 ? (ny - 1) * nx : (ny - 1) * nx + nx - 1;
}

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
// row kernels
// ---------------------------------------------------------------------------
struct RowRanges {
    int y0, y1, loM, hiM, loU, hiU;
};

__device__ __forceinline__ RowRanges row_ranges(int tile, int h, int ny) {
    RowRanges r;
    r.y0 = tile * h;
    r.y1 = min(r.y0 + h, ny);
    r.loM = (r.y0 == 0) ? 0 : r.y0 - 1;
    r.hiM = (r.y1 == ny) ? ny : r.y1 + 1;
    if (r.y0 == 0) r.hiM = max(r.hiM, min(3, ny));
    if (r.y1 == ny) r.loM = min(r.loM, ny - 3);
    r.loU = (r.loM == 0) ? 0 : r.loM - 1;
    r.hiU = (r.hiM == ny) ? ny : r.hiM + 1;
    if (r.loM == 0) r.hiU = max(r.hiU, min(3, ny));
    if (r.hiM == ny) r.loU = min(r.loU, ny - 3);
    return r;
}

__host__ __device__ inline int capU_of(int h) { return h + 4 > 5 ? h + 4 : 5; }
__host__ __device__ inline int capM_of(int h) { return h + 2 > 3 ? h + 2 : 3; }

// layout: [sU f64 capU*nx][sM 3*capM*nx][sR h*nx][sK capU*nx (inv)][tw nx float2][tice K]
// the inverse prologue's transforms (2*ceil(capU/2)*nx float2) alias the front.
__host__ __device__ inline size_t rows_fwd_lead_bytes(int nx, int h, int inv) {
    const size_t capU = capU_of(h), capM = capM_of(h);
    size_t lead = capU * nx * sizeof(double) + 3 * capM * nx * sizeof(float);
    const size_t inv_fft = (size_t)2 * ((capU + 1) / 2) * nx * sizeof(float2);
    if (inv && inv_fft > lead) lead = inv_fft;
    return lead;
}

__host__ __device__ inline size_t rows_fwd_body_bytes(int nx, int h, int inv) {
    size_t s = rows_fwd_lead_bytes(nx, h, inv) + (size_t)h * nx * sizeof(float);
    if (inv) s += (size_t)capU_of(h) * nx * sizeof(float);
    return (s + 15) / 16 * 16;
}

size_t rows_fwd_smem(int nx, int h, int inv, int K) {
    return rows_fwd_body_bytes(nx, h, inv) + (size_t)nx * sizeof(float2) +
           (K <= TICE_MAX ? (size_t)K * sizeof(double) : 0);
}

// Inverse real row transform of spectrum rows [lo, hi) into dst[(r - lo) * nx + x]
// (two rows per complex FFT); zb: 2 * ceil((hi-lo)/2) * nx complex scratch.
__device__ void rows_inverse_to(const Member& m, const FftPlan& plan, int lo, int hi, float2* zb, float* dst) {
    const int nx = m.nx, NH = m.NH, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int np = (hi - lo + 1) / 2;
    for (int p = ty; p < np; p += TY) {
        const int ra = lo + 2 * p;
        const bool hasb = ra + 1 < hi;
        const float2* Sa = m.S + (size_t)ra * m.sp;
        const float2* Sb = m.S + (size_t)(ra + 1) * m.sp;
        for (int k = tx; k < nx; k += TX) {
            const int kk = (k < NH) ? k : nx - k;
            const float2 A = Sa[kk];
            const float2 Bv = hasb ? Sb[kk] : make_float2(0.0f, 0.0f);
            zb[(size_t)p * nx + k] = (k < NH) ? make_float2(A.x - Bv.y, A.y + Bv.x) : make_float2(A.x + Bv.y, -A.y + Bv.x);
        }
    }
    __syncthreads();
    float2* res = fft_batch<true, float>(zb, zb + (size_t)np * nx, plan, np, nx);
    for (int rl = ty; rl < hi - lo; rl += TY) {
        const int p = rl >> 1, q = rl & 1;
        for (int x = tx; x < nx; x += TX) {
            const float2 z = res[(size_t)p * nx + x];
            dst[(size_t)rl * nx + x] = q ? z.y : z.x;
        }
    }
}

// corner values (0,0),(nx-1,0),(0,ny-1),(nx-1,ny-1) of the field whose half spectrum is
// S, evaluated directly (every thread gets them)
__device__ void spectrum_corners(const Member& m, const FftPlan& plan, double* red, double* out4) {
    double v[4] = {0, 0, 0, 0};
    const float* twr = (const float*)plan.tw32;
    row_corner_partial(m.S, m.nx, twr, &v[0], &v[1]);
    row_corner_partial(m.S + (size_t)(m.ny - 1) * m.sp, m.nx, twr, &v[2], &v[3]);
    block_sum<4>(v, red);
    for (int q = 0; q < 4; q++) out4[q] = v[q];
}

__device__ __forceinline__ double cmean(const double* c, double border) {
    return 0.25 * (c[0] + c[1] + c[2] + c[3]) - border;
}

// Forward row kernel of one right-hand side.  stage 0: uin at t_call; stage 1: the
// state at t_call; stages 2-4: BS3 stage vectors.  inv_prev (stages 3, 4): S holds
// the previous stage's spectrum after the column pass; its rows [loU, hiU) are
// inverted here (halo recomputed) and its own rows stored as k_{stage-1}.
__global__ void __launch_bounds__(RT, 2)
k_rows_fwd(const Member* __restrict__ mems, const Task* __restrict__ tasks, int stage, int h, const double* uin,
           int inv_prev) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    __shared__ double s_d[16];
    __shared__ double s_red[32 * 4];
    __shared__ int s_i[4];
    const Task tk = tasks[blockIdx.x];
    {
        // the shared layout needs nx and K before the head is staged
        const Member* mp = &mems[tk.member];
        const int nx0 = mp->nx, K0 = mp->K;
        float2* stw = (float2*)(smem + rows_fwd_body_bytes(nx0, h, inv_prev));
        double* stice = (K0 <= TICE_MAX) ? (double*)(stw + nx0) : nullptr;
        if (!head_load(hd, mems, tk, 0, stw, stice, stage == 0 ? 2 : 1, uin)) return;
    }
    const Member& m = hd.m;
    const Ctl& c = hd.c;
    Ctl* ctl = m.ctl;
    const int nx = m.nx, ny = m.ny, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const RowRanges rr = row_ranges(tk.tile, h, ny);
    const int capU = capU_of(h), capM = capM_of(h);
    double* sU = (double*)smem;
    float* sMxx = (float*)(sU + (size_t)capU * nx);
    float* sMyy = sMxx + (size_t)capM * nx;
    float* sMxy = sMyy + (size_t)capM * nx;
    float* sR = (float*)(smem + rows_fwd_lead_bytes(nx, h, inv_prev));
    float* sK = sR + (size_t)h * nx;
    const double* stice = (const double*)((float2*)(smem + rows_fwd_body_bytes(nx, h, inv_prev)) + nx);
    const double* __restrict__ uprev = (stage == 0) ? uin : m.u[c.ibuf];
    const int ik = c.ik;
    const float* __restrict__ k1 = m.k14[ik];
    const float* __restrict__ k2 = m.k2;
    const float* __restrict__ k3 = m.k3;
    double cprev[4] = {0, 0, 0, 0};
    if (inv_prev) {
        spectrum_corners(m, hd.plan, s_red, cprev);
        rows_inverse_to(m, hd.plan, rr.loU, rr.hiU, (float2*)smem, sK);
        __syncthreads();
        float* kdst = (stage == 3) ? m.k2 : m.k3;
        for (int r = rr.y0 + ty; r < rr.y1; r += TY)
            for (int x = tx; x < nx; x += TX) kdst[(size_t)r * nx + x] = sK[(size_t)(r - rr.loU) * nx + x];
        if (tk.tile == 0 && tid == 0) {
            double* cd = ctl->kcorner[stage == 3 ? 2 : 3];
            for (int q = 0; q < 4; q++) cd[q] = cprev[q];
        }
    }
    if (tid == 0) {
        const double t = c.t, dt = c.dt;
        double a1 = 0, a2 = 0, a3 = 0, tr = 0;
        if (stage <= 1) tr = c.t_call;
        else if (stage == 2) { tr = t + C2 * dt; a1 = dt * A21; }
        else if (stage == 3) { tr = t + C3 * dt; a2 = dt * A32; }
        else { tr = t + dt; a1 = dt * A41; a2 = dt * A42; a3 = dt * A43; }
        const double* kc1 = c.kcorner[ik];
        const double* kc2 = (stage == 3) ? cprev : c.kcorner[2];
        const double* kc3 = (stage == 4) ? cprev : c.kcorner[3];
        const double c1 = cmean(kc1, m.border_v), c2 = cmean(kc2, m.border_v), c3 = cmean(kc3, m.border_v);
        const double* uc = hd.ucorn[stage == 0 ? 0 : c.ibuf];
        double us = 0.0;
        for (int q = 0; q < 4; q++) {
            double v = uc[q];
            if (a1 != 0.0) v += a1 * (kc1[q] - c1);
            if (a2 != 0.0) v += a2 * (kc2[q] - c2);
            if (a3 != 0.0) v += a3 * (kc3[q] - c3);
            us += 0.25 * v;
        }
        s_d[0] = a1; s_d[1] = a2; s_d[2] = a3;
        s_d[3] = c1; s_d[4] = c2; s_d[5] = c3;
        s_d[6] = us - m.border_v;
        s_d[7] = cmean(c.ue_corner[c.iue], m.border_e);
        s_d[8] = cmean(c.ue_corner[c.iue_zb], m.border_e);
        s_d[9] = cmean(c.dz_corner, m.border_g);
        int ii = 0;
        double w = 0.0;
        if (!m.ice_external) {
            const int st = ice_lookup(m.K <= TICE_MAX ? stice : m.t_ice, m.K, m.ice_flat, tr, &ii, &w);
            if (st != FI_OK && tk.tile == 0) ctl->status = st;
        }
        s_d[10] = w;
        s_i[0] = ii;
    }
    __syncthreads();
    const double a1 = s_d[0], a2 = s_d[1], a3 = s_d[2], c1 = s_d[3], c2 = s_d[4], c3 = s_d[5], off = s_d[6];

    // phase 1: stage vector rows [loU, hiU) in FP64, corner BC applied
    for (int r = rr.loU + ty; r < rr.hiU; r += TY) {
        const size_t rb = (size_t)r * nx;
        const float* kr = sK + (size_t)(r - rr.loU) * nx;
        double* dstU = sU + (size_t)(r - rr.loU) * nx;
        for (int x = tx; x < nx; x += TX) {
            const size_t g = rb + x;
            double v = uprev[g];
            if (a1 != 0.0) v += a1 * ((double)k1[g] - c1);
            if (a2 != 0.0) v += a2 * ((double)(stage == 3 && inv_prev ? kr[x] : k2[g]) - c2);
            if (a3 != 0.0) v += a3 * ((double)(inv_prev ? kr[x] : k3[g]) - c3);
            dstU[x] = v - off;
        }
    }
    __syncthreads();

    // phase 2a: bending moments on rows [loM, hiM) (u-derivatives in FP64)
    {
        const double dx = m.dx, dy = m.dy, nu = m.nu;
        const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy), i2dx = 1.0 / (2 * dx), idx = 1.0 / dx;
        const double i2dy = 1.0 / (2 * dy), idy = 1.0 / dy;
        for (int r = rr.loM + ty; r < rr.hiM; r += TY) {
            const double* Ur = sU + (size_t)(r - rr.loU) * nx;
            const int rc = min(max(r, 1), ny - 2);
            const double* U0 = sU + (size_t)(rc - rr.loU) * nx;
            const double* Ua;
            const double* Ub;
            double sy;
            if (r == 0) { Ua = sU + (size_t)(1 - rr.loU) * nx; Ub = sU + (size_t)(0 - rr.loU) * nx; sy = idy; }
            else if (r == ny - 1) { Ua = sU + (size_t)(ny - 1 - rr.loU) * nx; Ub = sU + (size_t)(ny - 2 - rr.loU) * nx; sy = idy; }
            else { Ua = Ur + nx; Ub = Ur - nx; sy = i2dy; }
            const size_t mo = (size_t)(r - rr.loM) * nx;
            const float* Dr = m.D + (size_t)r * nx;
            for (int x = tx; x < nx; x += TX) {
                const int xc = min(max(x, 1), nx - 2);
                const double uxx = (Ur[xc + 1] - 2.0 * Ur[xc] + Ur[xc - 1]) * idx2;
                const double uyy = (U0[nx + x] - 2.0 * U0[x] + U0[x - nx]) * idy2;
                double da, db;
                if (x == 0) { da = (Ua[1] - Ua[0]) * idx; db = (Ub[1] - Ub[0]) * idx; }
                else if (x == nx - 1) { da = (Ua[nx - 1] - Ua[nx - 2]) * idx; db = (Ub[nx - 1] - Ub[nx - 2]) * idx; }
                else { da = (Ua[x + 1] - Ua[x - 1]) * i2dx; db = (Ub[x + 1] - Ub[x - 1]) * i2dx; }
                const double uxy = (da - db) * sy;
                const double D = (double)Dr[x];
                sMxx[mo + x] = (float)(-D * (nu * uyy + uxx));
                sMyy[mo + x] = (float)(-D * (nu * uxx + uyy));
                sMxy[mo + x] = (float)(-D * (1.0 - nu) * uxy);
            }
        }
    }
    // phase 2b: column anomalies on the own rows; -g sigma_full to sR
    {
        const double cue = s_d[7], cuz = s_d[8], cdz = s_d[9], w = s_d[10];
        const float* Ha = m.ice_external ? m.H_ext : m.H_tab + (size_t)s_i[0] * nx * ny;
        const float* Hb = (w != 0.0) ? Ha + (size_t)nx * ny : Ha;
        const float* ue = m.ue[c.iue];
        const float* uz = m.ue[c.iue_zb];
        const float fw = (float)w;
        double* unew = (stage == 4 || stage <= 1) ? m.u[c.ibuf ^ 1] : nullptr;
        const int flags = m.flags;
        for (int r = rr.y0 + ty; r < rr.y1; r += TY) {
            const double* Urow = sU + (size_t)(r - rr.loU) * nx;
            for (int x = tx; x < nx; x += TX) {
                const size_t g = (size_t)r * nx + x;
                const double u = Urow[x];
                const float ha = Ha[g];
                const double H = (double)(fw != 0.0f ? ha + (Hb[g] - ha) * fw : ha);
                const double uev = (double)ue[g] - cue;
                const double zdiff = (double)((flags & FLAG_ZBSS) ? m.zbss_ref[g] : m.zbss_scalar) +
                                     ((double)uz[g] - cuz) + u - ((double)m.dz[g] - cdz);
                double haf = H + (zdiff < 0.0 ? zdiff : 0.0) * m.rho_sw_ice;
                haf = haf > 0.0 ? haf : 0.0;
                const double mk = (flags & FLAG_MASK) ? (double)m.mask[g] : 1.0;
                const double hafref = (flags & FLAG_HAFREF) ? (double)m.H_af_ref[g] : 0.0;
                const double sload = mk * (m.rho_ice * (haf - hafref));
                double sfull = mk * (m.rho_ice * haf + m.rho_litho * uev + m.rho_um * u);
                if (flags & FLAG_SIGREF) sfull -= (double)m.sigma_ref[g];
                m.sig_load[g] = (float)sload;
                double geo = sfull;
                if (m.column_compressible) {
                    const double uer = (flags & FLAG_UEREF) ? (double)m.ue_ref[g] : 0.0;
                    geo = sfull - mk * m.rho_litho * (uev - uer);
                }
                m.sig_geo[g] = (float)(m.A * geo);
                sR[(size_t)(r - rr.y0) * nx + x] = (float)(-m.g * sfull);
                if (unew) unew[g] = u;
            }
        }
    }
    __syncthreads();

    // phase 3: moment divergence in FP32 -> f = rhs * K/(2 eta), rows packed in pairs
    float2* zb = (float2*)smem;  // aliases sU (dead now)
    const int np = (rr.y1 - rr.y0 + 1) / 2;
    {
        const float idx2 = (float)(1.0 / (m.dx * m.dx)), idy2 = (float)(1.0 / (m.dy * m.dy));
        const float i2dx = (float)(1.0 / (2 * m.dx)), idx = (float)(1.0 / m.dx);
        const float i2dy = (float)(1.0 / (2 * m.dy)), idy = (float)(1.0 / m.dy);
        for (int rl = ty; rl < 2 * np; rl += TY) {
            const int r = rr.y0 + rl;
            const int p = rl >> 1, q = rl & 1;
            const bool valid = r < rr.y1;
            const int rv = valid ? r : rr.y1 - 1;
            const float* Mx = sMxx + (size_t)(rv - rr.loM) * nx;
            const int rc = min(max(rv, 1), ny - 2);
            const float* My0 = sMyy + (size_t)(rc - rr.loM) * nx;
            const float* Ma;
            const float* Mb;
            float sy;
            if (rv == 0) { Ma = sMxy + (size_t)(1 - rr.loM) * nx; Mb = sMxy + (size_t)(0 - rr.loM) * nx; sy = idy; }
            else if (rv == ny - 1) { Ma = sMxy + (size_t)(ny - 1 - rr.loM) * nx; Mb = sMxy + (size_t)(ny - 2 - rr.loM) * nx; sy = idy; }
            else { Ma = sMxy + (size_t)(rv + 1 - rr.loM) * nx; Mb = sMxy + (size_t)(rv - 1 - rr.loM) * nx; sy = i2dy; }
            float* zrow = (float*)(zb + (size_t)p * nx) + q;
            const float* vf = m.visc_fac + (size_t)rv * nx;
            const float* sr = sR + (size_t)(rv - rr.y0) * nx;
            for (int x = tx; x < nx; x += TX) {
                float f = 0.0f;
                if (valid) {
                    const int xc = min(max(x, 1), nx - 2);
                    const float mxx = (Mx[xc + 1] - 2.0f * Mx[xc] + Mx[xc - 1]) * idx2;
                    const float myy = (My0[nx + x] - 2.0f * My0[x] + My0[x - nx]) * idy2;
                    float da, db;
                    if (x == 0) { da = (Ma[1] - Ma[0]) * idx; db = (Mb[1] - Mb[0]) * idx; }
                    else if (x == nx - 1) { da = (Ma[nx - 1] - Ma[nx - 2]) * idx; db = (Mb[nx - 1] - Mb[nx - 2]) * idx; }
                    else { da = (Ma[x + 1] - Ma[x - 1]) * i2dx; db = (Mb[x + 1] - Mb[x - 1]) * i2dx; }
                    const float mxy = (da - db) * sy;
                    const float rhs = sr[x] + (mxx + (2.0f * mxy + myy));
                    f = rhs * vf[x];
                }
                zrow[2 * x] = f;
            }
        }
    }
    __syncthreads();
    float2* res = fft_batch<false, float>(zb, zb + (size_t)np * nx, hd.plan, np, nx);
    // split the pair spectra, store the half-spectrum rows
    {
        const int NH = m.NH;
        for (int p = ty; p < np; p += TY) {
            const int ra = rr.y0 + 2 * p;
            const bool hb = ra + 1 < rr.y1;
            float2* Sa = m.S + (size_t)ra * m.sp;
            float2* Sb = m.S + (size_t)(ra + 1) * m.sp;
            for (int kx = tx; kx < NH; kx += TX) {
                const float2 Z = res[(size_t)p * nx + kx];
                const float2 Zc = res[(size_t)p * nx + (kx == 0 ? 0 : nx - kx)];
                Sa[kx] = make_float2(0.5f * (Z.x + Zc.x), 0.5f * (Z.y - Zc.y));
                if (hb) Sb[kx] = make_float2(0.5f * (Z.y + Zc.y), -0.5f * (Z.x - Zc.x));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// k_cols: column FFT, spectral multiply, inverse column FFT (in place on S).
// next_stage (3 or 4): evaluates the sparse gate of the next right-hand side.
// Every right-hand side passes here once: it is counted here.
// ---------------------------------------------------------------------------
size_t cols_smem(int ny, int B) { return (size_t)2 * B * ny * sizeof(float2) + (size_t)ny * sizeof(float2); }

__global__ void __launch_bounds__(RT, 2)
k_cols(const Member* __restrict__ mems, const Task* __restrict__ tasks, int B, int next_stage,
       cudaGraphConditionalHandle h_gate) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    const Task tk = tasks[blockIdx.x];
    {
        const int ny0 = mems[tk.member].ny;
        float2* stw = (float2*)smem + (size_t)2 * B * ny0;
        if (!head_load(hd, mems, tk, 1, stw, nullptr, 0, nullptr)) return;
    }
    const Member& m = hd.m;
    Ctl* ctl = m.ctl;
    const int ny = m.ny, tid = threadIdx.x;
    const int kx0 = tk.tile * B;
    const int nb = min(B, m.NH - kx0);
    if (tid == 0 && tk.tile == 0) {
        ctl->nf += 1;
        if (next_stage >= 3) {
            const int g = gate_eval(m, ctl, hd.c.t + (next_stage == 3 ? C3 : 1.0) * hd.c.dt);
            if (h_gate) cudaGraphSetConditional(h_gate, g);
        }
    }
    float2* b0 = (float2*)smem;
    float2* b1 = b0 + (size_t)B * ny;
    const int lanes = nb, rows_per = RT / lanes;
    const int b = tid % lanes, r0 = tid / lanes;
    if (r0 < rows_per)
        for (int y = r0; y < ny; y += rows_per) b0[(size_t)b * ny + y] = m.S[(size_t)y * m.sp + kx0 + b];
    __syncthreads();
    float2* r = fft_batch<false, float>(b0, b1, hd.plan, nb, ny);
    float2* o = (r == b0) ? b1 : b0;
    for (int bb = 0; bb < nb; bb++) {
        const float* mu = m.mult + (size_t)(kx0 + bb) * ny;
        float2* rr_ = r + (size_t)bb * ny;
        for (int ky = tid; ky < ny; ky += RT) {
            const float s = __ldg(&mu[ky]);
            const float2 v = rr_[ky];
            rr_[ky] = make_float2(v.x * s, v.y * s);
        }
    }
    __syncthreads();
    float2* q = fft_batch<true, float>(r, o, hd.plan, nb, ny);
    if (r0 < rows_per)
        for (int y = r0; y < ny; y += rows_per) m.S[(size_t)y * m.sp + kx0 + b] = q[(size_t)b * ny + y];
}

// ---------------------------------------------------------------------------
// k_rows_inv: inverse real row FFT of the last stage; stage 4: embedded BS3 error
// norm and the step controller (last block); stages 0/1: output to vout / k1.
// ---------------------------------------------------------------------------
size_t rows_inv_smem(int nx, int h) {
    return (size_t)2 * ((h + 1) / 2) * nx * sizeof(float2) + (size_t)h * nx * sizeof(float) +
           (size_t)nx * sizeof(float2);
}

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
    __shared__ int s_last;
    const Task tk = tasks[blockIdx.x];
    {
        const int nx0 = mems[tk.member].nx;
        float2* stw = (float2*)(smem + (size_t)2 * ((h + 1) / 2) * nx0 * sizeof(float2) + (size_t)h * nx0 * sizeof(float));
        if (!head_load(hd, mems, tk, 0, stw, nullptr, 0, nullptr)) return;
    }
    const Member& m = hd.m;
    const Ctl& c = hd.c;
    Ctl* ctl = m.ctl;
    const int nx = m.nx, ny = m.ny, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int y0 = tk.tile * h, y1 = min(y0 + h, ny);
    const int np = (y1 - y0 + 1) / 2;
    const int ik = c.ik;
    int slot;
    float* dst;
    if (stage == 0) { slot = -1; dst = vout; }
    else if (stage == 1) { slot = ik; dst = m.k14[ik]; }
    else { slot = ik ^ 1; dst = m.k14[ik ^ 1]; }
    double cs4[4];
    spectrum_corners(m, hd.plan, s_red, cs4);
    float* sv = (float*)(smem + (size_t)2 * np * nx * sizeof(float2));
    rows_inverse_to(m, hd.plan, y0, y1, (float2*)smem, sv);
    __syncthreads();
    const double cs = cmean(cs4, m.border_v);
    double acc = 0.0;
    {
        const double dt = c.dt, abstol = c.abstol, reltol = c.reltol;
        const double* up = m.u[c.ibuf];
        const double* un = m.u[c.ibuf ^ 1];
        const float* k1 = m.k14[ik];
        double cc1 = 0, cc2 = 0, cc3 = 0;
        if (stage == 4) {
            cc1 = cmean(c.kcorner[ik], m.border_v);
            cc2 = cmean(c.kcorner[2], m.border_v);
            cc3 = cmean(c.kcorner[3], m.border_v);
        }
        for (int r = y0 + ty; r < y1; r += TY) {
            const float* vr = sv + (size_t)(r - y0) * nx;
            for (int x = tx; x < nx; x += TX) {
                const size_t g = (size_t)r * nx + x;
                const float v = vr[x];
                dst[g] = v;
                if (stage == 4) {
                    const double ut = dt * (BT1 * ((double)k1[g] - cc1) + BT2 * ((double)m.k2[g] - cc2) +
                                            BT3 * ((double)m.k3[g] - cc3) + BT4 * ((double)v - cs));
                    const double a = fabs(up[g]), b = fabs(un[g]);
                    const double sc = ut / (abstol + (a > b ? a : b) * reltol);
                    acc += sc * sc;
                }
            }
        }
    }
    if (stage != 4) {
        if (tk.tile == 0 && tid == 0) {
            double* cdst = (stage == 0) ? cout : ctl->kcorner[slot];
            for (int q = 0; q < 4; q++) cdst[q] = cs4[q];
        }
        return;
    }
    // stage 4: error-norm reduction over the member's row tiles, last block decides
    {
        double v[1] = {acc};
        block_sum<1>(v, s_red);
        if (tid == 0) {
            m.partial[tk.tile] = v[0];
            __threadfence();
            const unsigned int ntiles = (unsigned int)((ny + h - 1) / h);
            const unsigned int prev = atomicAdd(&ctl->arrive, 1u);
            s_last = (prev == ntiles - 1);
        }
        __syncthreads();
        if (s_last) {
            // the last block sums the partials (fixed order per lane) with one warp
            __threadfence();
            const int ntiles = (ny + h - 1) / h;
            if (tid < 32) {
                double sum = 0.0;
                for (int i = tid; i < ntiles; i += 32) sum += ((volatile double*)m.partial)[i];
                sum = warp_sum(sum);
                if (tid == 0) {
                    ctl->arrive = 0;
                    for (int q = 0; q < 4; q++) ctl->kcorner[slot][q] = cs4[q];
                    const double EEst = sqrt(sum / ((double)nx * ny));
                    finish_attempt(m, ctl, EEst, h_gate, h_loop);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Sparse update: padded linear convolutions of the elastic (channel A) and
// sea-surface (channel B) loads, crop + extended-space corner BC.  Row pairs of the
// same channel share one complex FFT: packing the two channels together would mix
// their FP32 rounding (their inputs differ by the cell area, ~1e9).
// ---------------------------------------------------------------------------
size_t conv_rows_smem(int Mx, int h) {
    return (size_t)2 * 2 * ((h + 1) / 2) * Mx * sizeof(float2) + (size_t)Mx * sizeof(float2);
}

__global__ void __launch_bounds__(RT, 2)
k_conv_rows(const Member* __restrict__ mems, const Task* __restrict__ tasks, int h) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    const Task tk = tasks[blockIdx.x];
    {
        const int Mx0 = mems[tk.member].Mx;
        float2* stw = (float2*)smem + (size_t)2 * 2 * ((h + 1) / 2) * Mx0;
        if (!head_load(hd, mems, tk, 2, stw, nullptr, 0, nullptr)) return;
    }
    if (!hd.c.gate) return;
    const Member& m = hd.m;
    const int nx = m.nx, ny = m.ny, Mx = m.Mx, MH = m.MH, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int y0 = tk.tile * h, y1 = min(y0 + h, ny);
    const int np = (y1 - y0 + 1) / 2;
    const int nch = m.elastic_on + m.geoid_on;
    if (nch == 0) return;
    const float* in[2];
    float2* out[2];
    int cc = 0;
    if (m.elastic_on) { in[cc] = m.sig_load; out[cc] = m.SA; cc++; }  // * K^2, K == 1
    if (m.geoid_on) { in[cc] = m.sig_geo; out[cc] = m.SB; cc++; }
    const int nt = nch * np;
    float2* zb = (float2*)smem;
    for (int tr = ty; tr < nt; tr += TY) {
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        const bool hb = ra + 1 < y1;
        const float* ia = in[ch] + (size_t)ra * nx;
        const float* ib = in[ch] + (size_t)(ra + 1) * nx;
        for (int x = tx; x < Mx; x += TX)
            zb[(size_t)tr * Mx + x] = (x < nx) ? make_float2(ia[x], hb ? ib[x] : 0.0f) : make_float2(0.0f, 0.0f);
    }
    __syncthreads();
    float2* res = fft_batch<false, float>(zb, zb + (size_t)nt * Mx, hd.plan, nt, Mx);
    for (int tr = ty; tr < nt; tr += TY) {
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        const bool hb = ra + 1 < y1;
        float2* oa = out[ch] + (size_t)ra * m.msp;
        float2* ob = out[ch] + (size_t)(ra + 1) * m.msp;
        for (int kx = tx; kx < MH; kx += TX) {
            const float2 Z = res[(size_t)tr * Mx + kx];
            const float2 Zc = res[(size_t)tr * Mx + (kx == 0 ? 0 : Mx - kx)];
            oa[kx] = make_float2(0.5f * (Z.x + Zc.x), 0.5f * (Z.y - Zc.y));
            if (hb) ob[kx] = make_float2(0.5f * (Z.y + Zc.y), -0.5f * (Z.x - Zc.x));
        }
    }
}

size_t conv_cols_smem(int My, int B) { return (size_t)2 * 2 * B * My * sizeof(float2) + (size_t)My * sizeof(float2); }

__global__ void __launch_bounds__(RT, 2)
k_conv_cols(const Member* __restrict__ mems, const Task* __restrict__ tasks, int B) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    const Task tk = tasks[blockIdx.x];
    {
        const int My0 = mems[tk.member].My;
        float2* stw = (float2*)smem + (size_t)2 * 2 * B * My0;
        if (!head_load(hd, mems, tk, 3, stw, nullptr, 0, nullptr)) return;
    }
    if (!hd.c.gate) return;
    const Member& m = hd.m;
    const int ny = m.ny, My = m.My, tid = threadIdx.x;
    const int kx0 = tk.tile * B;
    const int nb = min(B, m.MH - kx0);
    // transform list: [channel][b][y]; channel 0 = A (elastic), 1 = B (sea surface)
    float2* b0 = (float2*)smem;
    float2* b1 = b0 + (size_t)2 * B * My;
    const int nt = 2 * nb;
    const int lanes = nb, rows_per = RT / lanes;
    const int bl = tid % lanes, r0 = tid / lanes;
    if (r0 < rows_per)
        for (int y = r0; y < My; y += rows_per) {
            const float2 za = (y < ny) ? m.SA[(size_t)y * m.msp + kx0 + bl] : make_float2(0.0f, 0.0f);
            const float2 zc = (y < ny) ? m.SB[(size_t)y * m.msp + kx0 + bl] : make_float2(0.0f, 0.0f);
            b0[(size_t)bl * My + y] = za;
            b0[(size_t)(nb + bl) * My + y] = zc;
        }
    __syncthreads();
    float2* r = fft_batch<false, float>(b0, b1, hd.plan, nt, My);
    float2* o = (r == b0) ? b1 : b0;
    for (int tr = 0; tr < nt; tr++) {
        const int ch = tr / nb, b = tr - ch * nb;
        const float2* G = (ch == 0 ? m.GA : m.GB) + (size_t)(kx0 + b) * My;
        float2* rt = r + (size_t)tr * My;
        for (int ky = tid; ky < My; ky += RT) rt[ky] = cmul(rt[ky], __ldg(&G[ky]));
    }
    __syncthreads();
    float2* q = fft_batch<true, float>(r, o, hd.plan, nt, My);
    // keep the crop window rows j1..j1+ny-1 and the two corner rows 0, 2ny-2
    const int nrow = ny + 2;
    if (r0 < rows_per)
        for (int ry = r0; ry < nrow; ry += rows_per) {
            const int y = ry < ny ? m.j1 + ry : (ry == ny ? 0 : 2 * ny - 2);
            m.TA[(size_t)ry * m.msp + kx0 + bl] = q[(size_t)bl * My + y];
            m.TB[(size_t)ry * m.msp + kx0 + bl] = q[(size_t)(nb + bl) * My + y];
        }
}

__global__ void __launch_bounds__(RT, 2)
k_conv_rows_inv(const Member* __restrict__ mems, const Task* __restrict__ tasks, int h) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KHead hd;
    const Task tk = tasks[blockIdx.x];
    {
        const int Mx0 = mems[tk.member].Mx;
        float2* stw = (float2*)smem + (size_t)2 * 2 * ((h + 1) / 2) * Mx0;
        if (!head_load(hd, mems, tk, 2, stw, nullptr, 0, nullptr)) return;
    }
    if (!hd.c.gate) return;
    const Member& m = hd.m;
    Ctl* ctl = m.ctl;
    const int nx = m.nx, ny = m.ny, Mx = m.Mx, MH = m.MH, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int nrow = ny + 2;  // crop rows j1..j1+ny-1, then corner rows 0 and 2ny-2
    const int y0 = tk.tile * h, y1 = min(y0 + h, nrow);
    const int np = (y1 - y0 + 1) / 2;
    const int iue = hd.c.iue;
    if (!m.elastic_on) {
        // RigidLithosphere: ue = 0 (src/deformation.jl:186-189)
        for (int ry = y0 + ty; ry < min(y1, ny); ry += TY)
            for (int x = tx; x < nx; x += TX) m.ue[iue][(size_t)ry * nx + x] = 0.0f;
        if (tid == 0 && y1 > ny)
            for (int q = 0; q < 4; q++) ctl->ue_corner[iue][q] = 0.0;
    }
    const int nch = m.elastic_on + m.geoid_on;
    if (nch == 0) return;
    const float2* src[2];
    float* dst[2];
    double* corner[2];
    int cc = 0;
    if (m.elastic_on) { src[cc] = m.TA; dst[cc] = m.ue[iue]; corner[cc] = ctl->ue_corner[iue]; cc++; }
    if (m.geoid_on) { src[cc] = m.TB; dst[cc] = m.dz; corner[cc] = ctl->dz_corner; cc++; }
    const int nt = nch * np;
    float2* zb = (float2*)smem;
    for (int tr = ty; tr < nt; tr += TY) {
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        const bool hb = ra + 1 < y1;
        const float2* Sa = src[ch] + (size_t)ra * m.msp;
        const float2* Sb = src[ch] + (size_t)(ra + 1) * m.msp;
        for (int k = tx; k < Mx; k += TX) {
            const int kk = (k < MH) ? k : Mx - k;
            const float2 A = Sa[kk];
            const float2 Bv = hb ? Sb[kk] : make_float2(0.0f, 0.0f);
            zb[(size_t)tr * Mx + k] = (k < MH) ? make_float2(A.x - Bv.y, A.y + Bv.x) : make_float2(A.x + Bv.y, -A.y + Bv.x);
        }
    }
    __syncthreads();
    float2* res = fft_batch<true, float>(zb, zb + (size_t)nt * Mx, hd.plan, nt, Mx);
    for (int tr = ty; tr < nt; tr += TY) {
        const int ch = tr / np, p = tr - ch * np;
        for (int q = 0; q < 2; q++) {
            const int ry = y0 + 2 * p + q;
            if (ry >= ny || ry >= y1) continue;
            float* d = dst[ch] + (size_t)ry * nx;
            const float2* z = res + (size_t)tr * Mx + m.i1;
            for (int x = tx; x < nx; x += TX) d[x] = q == 0 ? z[x].x : z[x].y;
        }
    }
    if (tid == 0) {
        // corners of the (2nx-1) x (2ny-1) linear convolution, order (0,0), (2nx-2,0),
        // (0,2ny-2), (2nx-2,2ny-2)
        for (int tr = 0; tr < nt; tr++) {
            const int ch = tr / np, p = tr - ch * np;
            for (int q = 0; q < 2; q++) {
                const int ry = y0 + 2 * p + q;
                if (ry < ny || ry >= y1) continue;
                const int q0 = (ry == ny) ? 0 : 2;
                const float2 za = res[(size_t)tr * Mx + 0];
                const float2 zc = res[(size_t)tr * Mx + 2 * nx - 2];
                corner[ch][q0] = (double)(q == 0 ? za.x : za.y);
                corner[ch][q0 + 1] = (double)(q == 0 ? zc.x : zc.y);
            }
        }
    }
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
