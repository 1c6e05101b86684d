// fi_fused.cu -- FP32 fused kernels of the LV-ELVA right-hand side and BS3 step.
//
// One right-hand side (update_diagnostics!, src/simulation.jl:335-393) is three
// launches:
//   k_rows_fwd  stage state u = uprev + dt*sum(a_sj k_j) (FP64) -> corner BC
//               (boundary_conditions.jl:144-148) -> column anomalies
//               (loads.jl:31-106, topography.jl:30-39) -> flexure operator
//               rhs = -g sigma_full + dxx Mxx + 2 dxy Mxy + dyy Myy with the CPU
//               edge rules (deformation.jl:110-131, derivatives.jl:48-191; the
//               u-derivatives in FP64, the moment derivatives in FP32)
//               -> times K/(2 eta) -> real row FFT (two rows per complex FFT).
//   k_cols      column FFT, multiply by spy/(nx ny R|k|) (DC zeroed), inverse
//               column FFT (deformation.jl:95-98, solidearth.jl:222).
//   k_rows_inv  inverse real row FFT -> k_s in physical space; its corner offset
//               (the dudt corner BC, deformation.jl:101) is evaluated directly
//               from the spectrum and applied by every consumer; for stage 4 the
//               embedded BS3 error norm and the step controller (last block).
// The sparse elastic / sea-surface update (deformation.jl:175-184,
// sealevel.jl:173-201, convolutions.jl:134-143) is k_conv_rows, k_conv_cols,
// k_conv_rows_inv, gated per call on the device.
#include "fi_device.cuh"
#include "fi_kernels.h"

namespace fi {

// ---------------------------------------------------------------------------
// gate for a host-driven right-hand side at time t (stage 0 calls)
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
// k_rows_fwd
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

size_t rows_fwd_smem(int nx, int h) {
    const size_t capU = (size_t)(h + 4 > 5 ? h + 4 : 5);
    const size_t capM = (size_t)(h + 2 > 3 ? h + 2 : 3);
    return capU * nx * sizeof(double) + 3 * capM * nx * sizeof(float) + (size_t)h * nx * sizeof(float);
}

__global__ void __launch_bounds__(256)
k_rows_fwd(const Member* __restrict__ mems, const Task* __restrict__ tasks, const FftPlan* __restrict__ plans,
           int stage, int h, const double* uin) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ FftPlan s_plan;
    __shared__ double s_d[16];
    __shared__ int s_i[4];
    const Task tk = tasks[blockIdx.x];
    const Member& m = mems[tk.member];
    Ctl* ctl = m.ctl;
    if (!ctl->active) return;
    const int nx = m.nx, ny = m.ny, tid = threadIdx.x, nth = blockDim.x;
    const RowRanges rr = row_ranges(tk.tile, h, ny);
    const int capU = h + 4 > 5 ? h + 4 : 5, capM = h + 2 > 3 ? h + 2 : 3;
    double* sU = (double*)smem;
    float* sMxx = (float*)(sU + (size_t)capU * nx);
    float* sMyy = sMxx + (size_t)capM * nx;
    float* sMxy = sMyy + (size_t)capM * nx;
    float* sR = sMxy + (size_t)capM * nx;
    const double* __restrict__ uprev = (stage == 0) ? uin : m.u[ctl->ibuf];
    const int ik = ctl->ik;
    const float* __restrict__ k1 = m.k14[ik];
    const float* __restrict__ k2 = m.k2;
    const float* __restrict__ k3 = m.k3;

    if (tid == 0) {
        s_plan = plans[m.plan_x];
        const double t = ctl->t, dt = ctl->dt;
        double a1 = 0, a2 = 0, a3 = 0, tr = 0;
        if (stage <= 1) tr = ctl->t_call;
        else if (stage == 2) { tr = t + C2 * dt; a1 = dt * A21; }
        else if (stage == 3) { tr = t + C3 * dt; a2 = dt * A32; }
        else if (stage == 4) { tr = t + dt; a1 = dt * A41; a2 = dt * A42; a3 = dt * A43; }
        const double c1 = 0.25 * (ctl->kcorner[ik][0] + ctl->kcorner[ik][1] + ctl->kcorner[ik][2] + ctl->kcorner[ik][3]) - m.border_v;
        const double c2 = 0.25 * (ctl->kcorner[2][0] + ctl->kcorner[2][1] + ctl->kcorner[2][2] + ctl->kcorner[2][3]) - m.border_v;
        const double c3 = 0.25 * (ctl->kcorner[3][0] + ctl->kcorner[3][1] + ctl->kcorner[3][2] + ctl->kcorner[3][3]) - m.border_v;
        const int cidx[4] = {0, nx - 1, (ny - 1) * nx, (ny - 1) * nx + nx - 1};
        double us = 0.0;
        for (int q = 0; q < 4; q++) {
            double v = uprev[cidx[q]];
            if (a1 != 0.0) v += a1 * (ctl->kcorner[ik][q] - c1);
            if (a2 != 0.0) v += a2 * (ctl->kcorner[2][q] - c2);
            if (a3 != 0.0) v += a3 * (ctl->kcorner[3][q] - c3);
            us += 0.25 * v;
        }
        const int iue = ctl->iue, iuz = ctl->iue_zb;
        s_d[0] = a1; s_d[1] = a2; s_d[2] = a3;
        s_d[3] = c1; s_d[4] = c2; s_d[5] = c3;
        s_d[6] = us - m.border_v;  // corner offset of the stage vector
        s_d[7] = 0.25 * (ctl->ue_corner[iue][0] + ctl->ue_corner[iue][1] + ctl->ue_corner[iue][2] + ctl->ue_corner[iue][3]) - m.border_e;
        s_d[8] = 0.25 * (ctl->ue_corner[iuz][0] + ctl->ue_corner[iuz][1] + ctl->ue_corner[iuz][2] + ctl->ue_corner[iuz][3]) - m.border_e;
        s_d[9] = 0.25 * (ctl->dz_corner[0] + ctl->dz_corner[1] + ctl->dz_corner[2] + ctl->dz_corner[3]) - m.border_g;
        int ii = 0;
        double w = 0.0;
        if (!m.ice_external) {
            const int st = ice_lookup(m.t_ice, m.K, m.ice_flat, tr, &ii, &w);
            if (st != FI_OK && tk.tile == 0) ctl->status = st;
        }
        s_d[10] = w;
        s_i[0] = ii;
        s_i[1] = iue;
        s_i[2] = iuz;
    }
    __syncthreads();
    const double a1 = s_d[0], a2 = s_d[1], a3 = s_d[2], c1 = s_d[3], c2 = s_d[4], c3 = s_d[5], off = s_d[6];

    // phase 1: stage vector rows [loU, hiU) in FP64, corner BC applied
    {
        const int n = (rr.hiU - rr.loU) * nx;
        const size_t base = (size_t)rr.loU * nx;
        for (int e = tid; e < n; e += nth) {
            const size_t g = base + e;
            double v = uprev[g];
            if (a1 != 0.0) v += a1 * ((double)k1[g] - c1);
            if (a2 != 0.0) v += a2 * ((double)k2[g] - c2);
            if (a3 != 0.0) v += a3 * ((double)k3[g] - c3);
            sU[e] = v - off;
        }
    }
    __syncthreads();

    // phase 2a: bending moments on rows [loM, hiM) (u-derivatives in FP64)
    {
        const double dx = m.dx, dy = m.dy, nu = m.nu;
        const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy), i2dx = 1.0 / (2 * dx), idx = 1.0 / dx;
        const double i2dy = 1.0 / (2 * dy), idy = 1.0 / dy;
        const int n = (rr.hiM - rr.loM) * nx;
        for (int e = tid; e < n; e += nth) {
            const int rl = e / nx, x = e - rl * nx, r = rr.loM + rl;
            const double* Ur = sU + (size_t)(r - rr.loU) * nx;
            const int xc = min(max(x, 1), nx - 2);
            const double uxx = (Ur[xc + 1] - 2.0 * Ur[xc] + Ur[xc - 1]) * idx2;
            const int rc = min(max(r, 1), ny - 2);
            const double* U0 = sU + (size_t)(rc - rr.loU) * nx;
            const double uyy = (U0[nx + x] - 2.0 * U0[x] + U0[x - nx]) * idy2;
            // ux on a row: one-sided at the x edges
            auto uxr = [&](const double* R) -> double {
                if (x == 0) return (R[1] - R[0]) * idx;
                if (x == nx - 1) return (R[nx - 1] - R[nx - 2]) * idx;
                return (R[x + 1] - R[x - 1]) * i2dx;
            };
            double uxy;
            if (r == 0) uxy = (uxr(sU + (size_t)(1 - rr.loU) * nx) - uxr(sU + (size_t)(0 - rr.loU) * nx)) * idy;
            else if (r == ny - 1)
                uxy = (uxr(sU + (size_t)(ny - 1 - rr.loU) * nx) - uxr(sU + (size_t)(ny - 2 - rr.loU) * nx)) * idy;
            else uxy = (uxr(Ur + nx) - uxr(Ur - nx)) * i2dy;
            const double D = (double)m.D[(size_t)r * nx + x];
            sMxx[e] = (float)(-D * (nu * uyy + uxx));
            sMyy[e] = (float)(-D * (nu * uxx + uyy));
            sMxy[e] = (float)(-D * (1.0 - nu) * uxy);
        }
    }
    // phase 2b: column anomalies on the own rows; -g sigma_full to sR
    {
        const int n = (rr.y1 - rr.y0) * nx;
        const size_t base = (size_t)rr.y0 * nx;
        const double cue = s_d[7], cuz = s_d[8], cdz = s_d[9], w = s_d[10];
        const float* Ha = m.ice_external ? m.H_ext : m.H_tab + (size_t)s_i[0] * nx * ny;
        const float* Hb = (w != 0.0) ? Ha + (size_t)nx * ny : Ha;
        const float* ue = m.ue[s_i[1]];
        const float* uz = m.ue[s_i[2]];
        const float fw = (float)w;
        // stages 0, 1 and 4 publish the boundary-corrected stage vector (the in-place
        // apply_bc!(u) of the reference) to the scratch half of the state buffer
        double* unew = (stage == 4 || stage <= 1) ? m.u[ctl->ibuf ^ 1] : nullptr;
        for (int e = tid; e < n; e += nth) {
            const size_t g = base + e;
            const double u = sU[(size_t)(rr.y0 - rr.loU) * nx + e];
            const float ha = Ha[g];
            const double H = (double)(fw != 0.0f ? ha + (Hb[g] - ha) * fw : ha);
            const double uev = (double)ue[g] - cue;
            const double zdiff = (double)((m.flags & FLAG_ZBSS) ? m.zbss_ref[g] : m.zbss_scalar) +
                                 ((double)uz[g] - cuz) + u - ((double)m.dz[g] - cdz);
            double haf = H + (zdiff < 0.0 ? zdiff : 0.0) * m.rho_sw_ice;
            haf = haf > 0.0 ? haf : 0.0;
            const double mk = (m.flags & FLAG_MASK) ? (double)m.mask[g] : 1.0;
            const double hafref = (m.flags & FLAG_HAFREF) ? (double)m.H_af_ref[g] : 0.0;
            const double sload = mk * (m.rho_ice * (haf - hafref));
            double sfull = mk * (m.rho_ice * haf + m.rho_litho * uev + m.rho_um * u);
            if (m.flags & FLAG_SIGREF) sfull -= (double)m.sigma_ref[g];
            m.sig_load[g] = (float)sload;
            // sea-surface input: A * sigma_full, or A * (sigma_load + m * sigma_mantle) for a
            // compressible column (sealevel.jl:193-201); sigma_mantle = sigma_full - sigma_load - m sigma_litho
            double geo = sfull;
            if (m.column_compressible) {
                const double uer = (m.flags & FLAG_UEREF) ? (double)m.ue_ref[g] : 0.0;
                geo = sfull - mk * m.rho_litho * (uev - uer);
            }
            m.sig_geo[g] = (float)(m.A * geo);
            sR[e] = (float)(-m.g * sfull);
            if (unew) unew[g] = u;
        }
    }
    __syncthreads();

    // phase 3: moment divergence in FP32 -> f = rhs * K/(2 eta) packed as row pairs
    float2* zb = (float2*)smem;  // aliases sU (dead now)
    const int np = (rr.y1 - rr.y0 + 1) / 2;
    {
        const float idx2 = (float)(1.0 / (m.dx * m.dx)), idy2 = (float)(1.0 / (m.dy * m.dy));
        const float i2dx = (float)(1.0 / (2 * m.dx)), idx = (float)(1.0 / m.dx);
        const float i2dy = (float)(1.0 / (2 * m.dy)), idy = (float)(1.0 / m.dy);
        const int n = np * nx;
        for (int e = tid; e < n; e += nth) {
            const int p = e / nx, x = e - p * nx;
            float f2[2] = {0.0f, 0.0f};
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int r = rr.y0 + 2 * p + q;
                if (r >= rr.y1) break;
                const float* Mx = sMxx + (size_t)(r - rr.loM) * nx;
                const int xc = min(max(x, 1), nx - 2);
                const float mxx = (Mx[xc + 1] - 2.0f * Mx[xc] + Mx[xc - 1]) * idx2;
                const int rc = min(max(r, 1), ny - 2);
                const float* My0 = sMyy + (size_t)(rc - rr.loM) * nx;
                const float myy = (My0[nx + x] - 2.0f * My0[x] + My0[x - nx]) * idy2;
                auto dxr = [&](const float* R) -> float {
                    if (x == 0) return (R[1] - R[0]) * idx;
                    if (x == nx - 1) return (R[nx - 1] - R[nx - 2]) * idx;
                    return (R[x + 1] - R[x - 1]) * i2dx;
                };
                const float* Mr = sMxy + (size_t)(r - rr.loM) * nx;
                float mxy;
                if (r == 0) mxy = (dxr(sMxy + (size_t)(1 - rr.loM) * nx) - dxr(sMxy + (size_t)(0 - rr.loM) * nx)) * idy;
                else if (r == ny - 1)
                    mxy = (dxr(sMxy + (size_t)(ny - 1 - rr.loM) * nx) - dxr(sMxy + (size_t)(ny - 2 - rr.loM) * nx)) * idy;
                else mxy = (dxr(Mr + nx) - dxr(Mr - nx)) * i2dy;
                const size_t g = (size_t)r * nx + x;
                const float rhs = sR[(size_t)(r - rr.y0) * nx + x] + (mxx + (2.0f * mxy + myy));
                f2[q] = rhs * m.visc_fac[g];
            }
            zb[(size_t)p * nx + x] = make_float2(f2[0], f2[1]);
        }
    }
    __syncthreads();
    float2* res = fft_batch<false, float>(zb, zb + (size_t)np * nx, s_plan, np, nx);
    // phase 5: split the pair spectra, store the half spectrum rows
    {
        const int NH = m.NH;
        const int n = np * NH;
        for (int e = tid; e < n; e += nth) {
            const int p = e / NH, kx = e - p * NH;
            const float2 Z = res[(size_t)p * nx + kx];
            const float2 Zc = res[(size_t)p * nx + (kx == 0 ? 0 : nx - kx)];
            const int ra = rr.y0 + 2 * p;
            m.S[(size_t)ra * m.sp + kx] = make_float2(0.5f * (Z.x + Zc.x), 0.5f * (Z.y - Zc.y));
            if (ra + 1 < rr.y1) m.S[(size_t)(ra + 1) * m.sp + kx] = make_float2(0.5f * (Z.y + Zc.y), -0.5f * (Z.x - Zc.x));
        }
    }
}

// ---------------------------------------------------------------------------
// k_cols: column FFT, spectral multiply, inverse column FFT (in place on S)
// ---------------------------------------------------------------------------
size_t cols_smem(int ny, int B) { return (size_t)2 * B * ny * sizeof(float2); }

__global__ void __launch_bounds__(256)
k_cols(const Member* __restrict__ mems, const Task* __restrict__ tasks, const FftPlan* __restrict__ plans, int B) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ FftPlan s_plan;
    const Task tk = tasks[blockIdx.x];
    const Member& m = mems[tk.member];
    if (!m.ctl->active) return;
    const int ny = m.ny, tid = threadIdx.x, nth = blockDim.x;
    const int kx0 = tk.tile * B;
    const int nb = min(B, m.NH - kx0);
    if (tid == 0) s_plan = plans[m.plan_y];
    float2* b0 = (float2*)smem;
    float2* b1 = b0 + (size_t)B * ny;
    const int n = nb * ny;
    for (int e = tid; e < n; e += nth) {
        const int y = e / nb, b = e - y * nb;
        b0[(size_t)b * ny + y] = m.S[(size_t)y * m.sp + kx0 + b];
    }
    __syncthreads();
    float2* r = fft_batch<false, float>(b0, b1, s_plan, nb, ny);
    float2* o = (r == b0) ? b1 : b0;
    for (int e = tid; e < n; e += nth) {
        const int b = e / ny, ky = e - b * ny;
        const float s = __ldg(&m.mult[(size_t)(kx0 + b) * ny + ky]);
        const float2 v = r[e];
        r[e] = make_float2(v.x * s, v.y * s);
    }
    __syncthreads();
    float2* q = fft_batch<true, float>(r, o, s_plan, nb, ny);
    for (int e = tid; e < n; e += nth) {
        const int y = e / nb, b = e - y * nb;
        m.S[(size_t)y * m.sp + kx0 + b] = q[(size_t)b * ny + y];
    }
}

// ---------------------------------------------------------------------------
// k_rows_inv: inverse real row FFT; corner offsets; stage-4 error norm + controller
// ---------------------------------------------------------------------------
size_t rows_inv_smem(int nx, int h) { return (size_t)2 * ((h + 1) / 2) * nx * sizeof(float2); }

__device__ void finish_attempt(const Member& m, Ctl* c, double EEst, cudaGraphConditionalHandle h_gate,
                               cudaGraphConditionalHandle h_loop) {
    controller_update(c, EEst, m.tout);
    int active = (c->status == FI_OK);
    if (c->accept_step) {
        c->nsteps_seg += 1;
        if (c->pending_output || !(c->t < c->t_stop)) active = 0;
    } else {
        c->nsteps_seg += 1;
    }
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

__global__ void __launch_bounds__(256)
k_rows_inv(const Member* __restrict__ mems, const Task* __restrict__ tasks, const FftPlan* __restrict__ plans,
           int stage, int h, float* vout, double* cout, cudaGraphConditionalHandle h_gate,
           cudaGraphConditionalHandle h_loop) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ FftPlan s_plan;
    __shared__ double s_red[32 * 4];
    __shared__ double s_c[8];
    __shared__ int s_last;
    const Task tk = tasks[blockIdx.x];
    const Member& m = mems[tk.member];
    Ctl* ctl = m.ctl;
    if (!ctl->active) return;
    const int nx = m.nx, ny = m.ny, NH = m.NH, tid = threadIdx.x, nth = blockDim.x;
    const int y0 = tk.tile * h, y1 = min(y0 + h, ny);
    const int np = (y1 - y0 + 1) / 2;
    const int ik = ctl->ik;
    int slot;
    float* dst;
    if (stage == 0) { slot = -1; dst = vout; }
    else if (stage == 1) { slot = ik; dst = m.k14[ik]; }
    else if (stage == 2) { slot = 2; dst = m.k2; }
    else if (stage == 3) { slot = 3; dst = m.k3; }
    else { slot = ik ^ 1; dst = m.k14[ik ^ 1]; }
    if (tid == 0) s_plan = plans[m.plan_x];
    __syncthreads();
    // corner values of this stage's field from spectrum rows 0 and ny-1
    {
        double v[4] = {0, 0, 0, 0};
        const float* twr = (const float*)s_plan.tw32;
        row_corner_partial(m.S, nx, twr, &v[0], &v[1]);
        row_corner_partial(m.S + (size_t)(ny - 1) * m.sp, nx, twr, &v[2], &v[3]);
        block_sum<4>(v, s_red);
        if (tid == 0) { s_c[0] = v[0]; s_c[1] = v[1]; s_c[2] = v[2]; s_c[3] = v[3]; }
    }
    // build the pair spectra z[k] = A[k] + i B[k] on the full circle
    float2* zb = (float2*)smem;
    {
        const int n = np * nx;
        for (int e = tid; e < n; e += nth) {
            const int p = e / nx, k = e - p * nx;
            const int ra = y0 + 2 * p;
            const bool hasb = ra + 1 < y1;
            const int kk = (k < NH) ? k : nx - k;
            const float2 A = m.S[(size_t)ra * m.sp + kk];
            const float2 Bv = hasb ? m.S[(size_t)(ra + 1) * m.sp + kk] : make_float2(0.0f, 0.0f);
            float2 z;
            if (k < NH) z = make_float2(A.x - Bv.y, A.y + Bv.x);
            else z = make_float2(A.x + Bv.y, -A.y + Bv.x);  // conj(A) + i conj(B)
            zb[e] = z;
        }
    }
    __syncthreads();
    float2* res = fft_batch<true, float>(zb, zb + (size_t)np * nx, s_plan, np, nx);
    const double cs = 0.25 * (s_c[0] + s_c[1] + s_c[2] + s_c[3]) - m.border_v;
    double acc = 0.0;
    {
        const int n = np * nx;
        const double dt = ctl->dt, abstol = ctl->abstol, reltol = ctl->reltol;
        const double* up = m.u[ctl->ibuf];
        const double* un = m.u[ctl->ibuf ^ 1];
        const float* k1 = m.k14[ik];
        double cc1 = 0, cc2 = 0, cc3 = 0;
        if (stage == 4) {
            cc1 = 0.25 * (ctl->kcorner[ik][0] + ctl->kcorner[ik][1] + ctl->kcorner[ik][2] + ctl->kcorner[ik][3]) - m.border_v;
            cc2 = 0.25 * (ctl->kcorner[2][0] + ctl->kcorner[2][1] + ctl->kcorner[2][2] + ctl->kcorner[2][3]) - m.border_v;
            cc3 = 0.25 * (ctl->kcorner[3][0] + ctl->kcorner[3][1] + ctl->kcorner[3][2] + ctl->kcorner[3][3]) - m.border_v;
        }
        for (int e = tid; e < n; e += nth) {
            const int p = e / nx, x = e - p * nx;
            const float2 z = res[e];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int r = y0 + 2 * p + q;
                if (r >= y1) break;
                const size_t g = (size_t)r * nx + x;
                const float v = q == 0 ? z.x : z.y;
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
            for (int q = 0; q < 4; q++) cdst[q] = s_c[q];
            ctl->nf += 1;
            if (stage == 2 || stage == 3) {
                const double cn = (stage == 2) ? C3 : 1.0;
                const int g = gate_eval(m, ctl, ctl->t + cn * ctl->dt);
                if (h_gate) cudaGraphSetConditional(h_gate, g);
            }
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
        if (s_last && tid == 0) {
            __threadfence();
            const int ntiles = (ny + h - 1) / h;
            double sum = 0.0;
            for (int i = 0; i < ntiles; i++) sum += ((volatile double*)m.partial)[i];
            ctl->arrive = 0;
            for (int q = 0; q < 4; q++) ctl->kcorner[slot][q] = s_c[q];
            ctl->nf += 1;
            const double EEst = sqrt(sum / ((double)nx * ny));
            finish_attempt(m, ctl, EEst, h_gate, h_loop);
        }
    }
}

// ---------------------------------------------------------------------------
// Sparse update: padded linear convolutions of the elastic (channel A) and
// sea-surface (channel B) loads, crop + extended-space corner BC.
// ---------------------------------------------------------------------------
// Row pairs of the same channel share one complex FFT: packing the elastic and the
// sea-surface channel together would mix their FP32 rounding (their inputs differ by
// the cell area, ~1e9).
size_t conv_rows_smem(int Mx, int h) { return (size_t)2 * 2 * ((h + 1) / 2) * Mx * sizeof(float2); }

__global__ void __launch_bounds__(256)
k_conv_rows(const Member* __restrict__ mems, const Task* __restrict__ tasks, const FftPlan* __restrict__ plans,
            int h) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ FftPlan s_plan;
    const Task tk = tasks[blockIdx.x];
    const Member& m = mems[tk.member];
    Ctl* ctl = m.ctl;
    if (!ctl->active || !ctl->gate) return;
    const int nx = m.nx, ny = m.ny, Mx = m.Mx, MH = m.MH, tid = threadIdx.x, nth = blockDim.x;
    const int y0 = tk.tile * h, y1 = min(y0 + h, ny);
    const int np = (y1 - y0 + 1) / 2;
    const int nch = m.elastic_on + m.geoid_on;
    if (nch == 0) return;
    if (tid == 0) s_plan = plans[m.plan_Mx];
    const float* in[2];
    float2* out[2];
    int c = 0;
    if (m.elastic_on) { in[c] = m.sig_load; out[c] = m.SA; c++; }  // * K^2, K == 1
    if (m.geoid_on) { in[c] = m.sig_geo; out[c] = m.SB; c++; }
    const int nt = nch * np;
    float2* zb = (float2*)smem;
    const int n = nt * Mx;
    for (int e = tid; e < n; e += nth) {
        const int tr = e / Mx, x = e - tr * Mx;
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        float2 z = make_float2(0.0f, 0.0f);
        if (x < nx) {
            z.x = in[ch][(size_t)ra * nx + x];
            if (ra + 1 < y1) z.y = in[ch][(size_t)(ra + 1) * nx + x];
        }
        zb[e] = z;
    }
    __syncthreads();
    float2* res = fft_batch<false, float>(zb, zb + (size_t)nt * Mx, s_plan, nt, Mx);
    const int n2 = nt * MH;
    for (int e = tid; e < n2; e += nth) {
        const int tr = e / MH, kx = e - tr * MH;
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        const float2 Z = res[(size_t)tr * Mx + kx];
        const float2 Zc = res[(size_t)tr * Mx + (kx == 0 ? 0 : Mx - kx)];
        out[ch][(size_t)ra * m.msp + kx] = make_float2(0.5f * (Z.x + Zc.x), 0.5f * (Z.y - Zc.y));
        if (ra + 1 < y1) out[ch][(size_t)(ra + 1) * m.msp + kx] = make_float2(0.5f * (Z.y + Zc.y), -0.5f * (Z.x - Zc.x));
    }
}

size_t conv_cols_smem(int My, int B) { return (size_t)2 * 2 * B * My * sizeof(float2); }

__global__ void __launch_bounds__(256)
k_conv_cols(const Member* __restrict__ mems, const Task* __restrict__ tasks, const FftPlan* __restrict__ plans,
            int B) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ FftPlan s_plan;
    const Task tk = tasks[blockIdx.x];
    const Member& m = mems[tk.member];
    Ctl* ctl = m.ctl;
    if (!ctl->active || !ctl->gate) return;
    const int ny = m.ny, My = m.My, tid = threadIdx.x, nth = blockDim.x;
    const int kx0 = tk.tile * B;
    const int nb = min(B, m.MH - kx0);
    if (tid == 0) s_plan = plans[m.plan_My];
    // batch layout: [channel][b][y]; channel 0 = A (elastic), 1 = B (sea surface)
    float2* b0 = (float2*)smem;
    float2* b1 = b0 + (size_t)2 * B * My;
    const int nt = 2 * nb;
    const int n = nt * My;
    for (int e = tid; e < n; e += nth) {
        const int tr = e / My, y = e - tr * My;
        const int ch = tr / nb, b = tr - ch * nb;
        float2 v = make_float2(0.0f, 0.0f);
        if (y < ny) v = (ch == 0 ? m.SA : m.SB)[(size_t)y * m.msp + kx0 + b];
        b0[e] = v;
    }
    __syncthreads();
    float2* r = fft_batch<false, float>(b0, b1, s_plan, nt, My);
    float2* o = (r == b0) ? b1 : b0;
    for (int e = tid; e < n; e += nth) {
        const int tr = e / My, ky = e - tr * My;
        const int ch = tr / nb, b = tr - ch * nb;
        const float2 gk = __ldg(&(ch == 0 ? m.GA : m.GB)[(size_t)(kx0 + b) * My + ky]);
        r[e] = cmul(r[e], gk);
    }
    __syncthreads();
    float2* q = fft_batch<true, float>(r, o, s_plan, nt, My);
    // keep the crop window rows j1..j1+ny-1 and the two corner rows 0, 2ny-2
    const int nrow = ny + 2;
    const int n3 = nt * nrow;
    for (int e = tid; e < n3; e += nth) {
        const int tr = e / nrow, ry = e - tr * nrow;
        const int ch = tr / nb, b = tr - ch * nb;
        const int y = ry < ny ? m.j1 + ry : (ry == ny ? 0 : 2 * ny - 2);
        (ch == 0 ? m.TA : m.TB)[(size_t)ry * m.msp + kx0 + b] = q[(size_t)tr * My + y];
    }
}

__global__ void __launch_bounds__(256)
k_conv_rows_inv(const Member* __restrict__ mems, const Task* __restrict__ tasks, const FftPlan* __restrict__ plans,
                int h) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ FftPlan s_plan;
    const Task tk = tasks[blockIdx.x];
    const Member& m = mems[tk.member];
    Ctl* ctl = m.ctl;
    if (!ctl->active || !ctl->gate) return;
    const int nx = m.nx, ny = m.ny, Mx = m.Mx, MH = m.MH, tid = threadIdx.x, nth = blockDim.x;
    const int nrow = ny + 2;  // crop rows j1..j1+ny-1, then corner rows 0 and 2ny-2
    const int y0 = tk.tile * h, y1 = min(y0 + h, nrow);
    const int np = (y1 - y0 + 1) / 2;
    const int iue = ctl->iue;
    if (!m.elastic_on) {
        // RigidLithosphere: ue = 0 (src/deformation.jl:186-189)
        for (int e = tid; e < (y1 - y0) * nx; e += nth) {
            const int ry = y0 + e / nx;
            if (ry < ny) m.ue[iue][(size_t)ry * nx + e % nx] = 0.0f;
        }
        if (tid == 0 && y1 > ny)
            for (int q = 0; q < 4; q++) ctl->ue_corner[iue][q] = 0.0;
    }
    const int nch = m.elastic_on + m.geoid_on;
    if (nch == 0) return;
    if (tid == 0) s_plan = plans[m.plan_Mx];
    const float2* src[2];
    float* dst[2];
    double* corner[2];
    int c = 0;
    if (m.elastic_on) { src[c] = m.TA; dst[c] = m.ue[iue]; corner[c] = ctl->ue_corner[iue]; c++; }
    if (m.geoid_on) { src[c] = m.TB; dst[c] = m.dz; corner[c] = ctl->dz_corner; c++; }
    const int nt = nch * np;
    float2* zb = (float2*)smem;
    const int n = nt * Mx;
    for (int e = tid; e < n; e += nth) {
        const int tr = e / Mx, k = e - tr * Mx;
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        const int kk = (k < MH) ? k : Mx - k;
        const float2 A = src[ch][(size_t)ra * m.msp + kk];
        const float2 Bv = (ra + 1 < y1) ? src[ch][(size_t)(ra + 1) * m.msp + kk] : make_float2(0.0f, 0.0f);
        zb[e] = (k < MH) ? make_float2(A.x - Bv.y, A.y + Bv.x) : make_float2(A.x + Bv.y, -A.y + Bv.x);
    }
    __syncthreads();
    float2* res = fft_batch<true, float>(zb, zb + (size_t)nt * Mx, s_plan, nt, Mx);
    const int n2 = nt * nx;
    for (int e = tid; e < n2; e += nth) {
        const int tr = e / nx, x = e - tr * nx;
        const int ch = tr / np, p = tr - ch * np;
        const float2 z = res[(size_t)tr * Mx + m.i1 + x];
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int ry = y0 + 2 * p + q;
            if (ry < ny && ry < y1) dst[ch][(size_t)ry * nx + x] = q == 0 ? z.x : z.y;
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
__device__ __forceinline__ double corner_off(const double* c, double border) {
    return 0.25 * (c[0] + c[1] + c[2] + c[3]) - border;
}

__global__ void kf_initdt_norms(const double* u, const float* v, const double* vc, double border, double abstol,
                                double reltol, double* partial, size_t n) {
    __shared__ double red[64];
    const double c = corner_off(vc, border);
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
    const double c = corner_off(vc, border);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        u1[i] = u[i] + dt0 * ((double)v[i] - c);
}

__global__ void kf_initdt_d2(const double* u, const float* v0, const double* c0p, const float* v1,
                             const double* c1p, double border, double abstol, double reltol, double* partial,
                             size_t n) {
    __shared__ double red[64];
    const double c0 = corner_off(c0p, border), c1 = corner_off(c1p, border);
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
