// fi_plain.cu -- the plain FP64 form: one kernel per operation of the reference
// right-hand side (the broadcast / stencil structure of src/simulation.jl:335-393,
// src/deformation.jl:91-131 and src/derivatives.jl:48-191), complex 2D FFTs as in
// the reference's c2c plans, a host-side step controller.  It is the comparison
// baseline of the fused FP32 form and a second, independent implementation.
#include "fi_device.cuh"
#include "fi_plain.h"

namespace fi {

#define GRID_STRIDE(i, n) for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)(n); \
                               i += (size_t)gridDim.x * blockDim.x)

__global__ void kp_corner_off(const double* X, int nx, int ny, double border, double* off) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        // sum(W .* X) with W = 1/4 at the corners (boundary_conditions.jl:144-148, 199-207)
        const double s = 0.25 * X[0] + 0.25 * X[nx - 1] + 0.25 * X[(size_t)(ny - 1) * nx] +
                         0.25 * X[(size_t)(ny - 1) * nx + nx - 1];
        *off = s - border;
    }
}

__global__ void kp_sub_off(double* X, size_t n, const double* off) {
    const double o = *off;
    GRID_STRIDE(i, n) X[i] -= o;
}

__global__ void kp_copy(double* dst, const double* src, size_t n) { GRID_STRIDE(i, n) dst[i] = src[i]; }

__global__ void kp_bedrock(const double* u, const double* ue, const double* z_b_ref, const double* u_ref,
                           double* now_u, double* z_b, double* s_m, double rho_um, size_t n) {
    GRID_STRIDE(i, n) {
        now_u[i] = u[i];
        z_b[i] = z_b_ref[i] + ue[i] + u[i];
        s_m[i] = rho_um * (u[i] - u_ref[i]);
    }
}

__global__ void kp_ice(const double* Ha, const double* Hb, double dti, double tt, int exact, double* H, size_t n) {
    GRID_STRIDE(i, n) H[i] = exact ? Ha[i] : Ha[i] + (Hb[i] - Ha[i]) / dti * tt;
}

__global__ void kp_haf_ice(const double* H, const double* z_b, const double* z_ss, const double* H_af_ref,
                           double* H_af, double* s_i, double rho_sw_ice, double rho_ice, size_t n) {
    GRID_STRIDE(i, n) {
        double m = z_b[i] - z_ss[i];
        if (m > 0) m = 0;
        double v = H[i] + m * rho_sw_ice;
        v = v > 0 ? v : 0.0;
        H_af[i] = v;
        s_i[i] = rho_ice * (v - H_af_ref[i]);
    }
}

__global__ void kp_litho(const double* ue, const double* ue_ref, double* s_l, double rho_l, size_t n) {
    GRID_STRIDE(i, n) s_l[i] = rho_l * (ue[i] - ue_ref[i]);
}

__global__ void kp_geo_in(const double* s_load, const double* s_full, const double* s_m, const double* mask,
                          int compressible, double A, double* out, size_t n) {
    GRID_STRIDE(i, n) out[i] = compressible ? A * (s_load[i] + mask[i] * s_m[i]) : A * s_full[i];
}

__global__ void kp_zss(const double* z_ss_ref, const double* dz, double z_bsl, double* z_ss, size_t n) {
    GRID_STRIDE(i, n) z_ss[i] = z_ss_ref[i] + dz[i] + z_bsl;
}

__global__ void kp_load_full(const double* s_i, const double* s_sw, const double* s_l, const double* s_m,
                             const double* mask, double* s_load, double* s_full, size_t n) {
    GRID_STRIDE(i, n) {
        const double ld = mask[i] * (s_i[i] + s_sw[i] + 0.0);  // the sediment anomaly is zero
        s_load[i] = ld;
        s_full[i] = ld + mask[i] * (s_l[i] + s_m[i]);
    }
}

// block partial sums of H_af A, H_ice A and max(z_ss - z_b, 0) A (update_V_af!,
// update_V_den!, update_V_pov!, src/sealevel.jl:275-332), three per block
__global__ void kp_volumes(const double* H_af, const double* H, const double* z_ss, const double* z_b, double A,
                           double* partial, size_t n) {
    __shared__ double red[96];
    double a = 0.0, d = 0.0, p = 0.0;
    GRID_STRIDE(i, n) {
        a += H_af[i] * A;
        d += H[i] * A;
        const double w = z_ss[i] - z_b[i];
        p += (w > 0 ? w : 0.0) * A;
    }
    double v[3] = {a, d, p};
    block_sum<3>(v, red);
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++) partial[3 * blockIdx.x + q] = v[q];
}

// update_maskgrounded!, update_maskocean!, watercolumn! and columnanom_water!
// (src/topography.jl:1-28, src/loads.jl:56-85)
__global__ void kp_sealevel(const double* H, const double* H_af, const double* z_ss, const double* z_b,
                            const double* z_ss_ref, const double* mask, int interactive, double rho_sw,
                            double rho_i_sw, double* mgr, double* moc, double* hwater, double* s_sw, size_t n) {
    GRID_STRIDE(i, n) {
        const bool gr = H_af[i] > 0;
        const double w = z_ss[i] - z_b[i];
        const bool oc = w > 0 && !gr;
        const double wc = w > 0 ? w : 0.0;
        mgr[i] = gr;
        moc[i] = oc;
        hwater[i] = (H[i] <= 1 ? wc : 0.0) + ((!gr && H[i] > 1) ? wc - H[i] * rho_i_sw : 0.0);
        s_sw[i] = interactive ? rho_sw * (z_ss[i] - z_ss_ref[i]) * (oc ? 1.0 : 0.0) * mask[i] : 0.0;
    }
}

__global__ void kp_rhs_init(const double* s_full, double g, double* rhs, size_t n) {
    GRID_STRIDE(i, n) rhs[i] = -g * s_full[i];
}

__global__ void kp_dxx(double* du, const double* u, int nx, int ny, double Dx) {
    GRID_STRIDE(e, (size_t)nx * ny) {
        const int i = (int)(e % nx);
        const size_t r = e - i;
        const int c = i < 1 ? 1 : (i > nx - 2 ? nx - 2 : i);
        du[e] = (u[r + c + 1] - 2 * u[r + c] + u[r + c - 1]) / (Dx * Dx);
    }
}

__global__ void kp_dyy(double* du, const double* u, int nx, int ny, double Dy) {
    GRID_STRIDE(e, (size_t)nx * ny) {
        const int i = (int)(e % nx), j = (int)(e / nx);
        const int c = j < 1 ? 1 : (j > ny - 2 ? ny - 2 : j);
        if (j > 0 && j < ny - 1)
            du[e] = (u[(size_t)(c + 1) * nx + i] - 2 * u[(size_t)c * nx + i] + u[(size_t)(c - 1) * nx + i]) / (Dy * Dy);
        else if (j == 0)
            du[e] = (u[(size_t)2 * nx + i] - 2 * u[(size_t)nx + i] + u[i]) / (Dy * Dy);
        else
            du[e] = (u[(size_t)(ny - 1) * nx + i] - 2 * u[(size_t)(ny - 2) * nx + i] + u[(size_t)(ny - 3) * nx + i]) /
                    (Dy * Dy);
    }
}

__global__ void kp_dx(double* du, const double* u, int nx, int ny, double Dx) {
    GRID_STRIDE(e, (size_t)nx * ny) {
        const int i = (int)(e % nx);
        if (i == 0) du[e] = (u[e + 1] - u[e]) / Dx;
        else if (i == nx - 1) du[e] = (u[e] - u[e - 1]) / Dx;
        else du[e] = (u[e + 1] - u[e - 1]) / (2 * Dx);
    }
}

__global__ void kp_dy(double* du, const double* u, int nx, int ny, double Dy) {
    GRID_STRIDE(e, (size_t)nx * ny) {
        const int j = (int)(e / nx);
        if (j == 0) du[e] = (u[e + nx] - u[e]) / Dy;
        else if (j == ny - 1) du[e] = (u[e] - u[e - nx]) / Dy;
        else du[e] = (u[e + nx] - u[e - nx]) / (2 * Dy);
    }
}

__global__ void kp_moments(const double* bxx, const double* byy, const double* bxy, const double* D, double nu,
                           double* Mxx, double* Myy, double* Mxy, size_t n) {
    GRID_STRIDE(i, n) {
        Mxx[i] = -D[i] * (nu * byy[i] + bxx[i]);
        Myy[i] = -D[i] * (nu * bxx[i] + byy[i]);
        Mxy[i] = -D[i] * (1 - nu) * bxy[i];
    }
}

__global__ void kp_rhs_acc(double* rhs, const double* bxx, const double* byy, const double* bxy, size_t n) {
    GRID_STRIDE(i, n) rhs[i] += bxx[i] + (2 * bxy[i] + byy[i]);
}

__global__ void kp_fftin(const double* rhs, const double* eta, double2* f, size_t n) {
    GRID_STRIDE(i, n) f[i] = make_double2(rhs[i] * 1.0 / (2 * eta[i]), 0.0);
}

__global__ void kp_spec(double2* f, const double* spinv, size_t n) {
    GRID_STRIDE(i, n) {
        const double s = spinv[i];
        f[i].x *= s;
        f[i].y *= s;
    }
}

__global__ void kp_real_spy(const double2* f, double spy, double* dudt, size_t n) {
    GRID_STRIDE(i, n) dudt[i] = f[i].x * spy;
}

__global__ void kp_cmul(double2* P, const double2* G, size_t n) {
    GRID_STRIDE(i, n) {
        const double2 a = P[i], b = G[i];
        P[i] = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    }
}

__global__ void kp_crop(const double2* P, int Mx, int cx, int cy, double* out) {
    GRID_STRIDE(e, (size_t)cx * cy) {
        const int i = (int)(e % cx), j = (int)(e / cx);
        out[e] = P[(size_t)j * Mx + i].x;
    }
}

__global__ void kp_window(const double* cropped, int cx, int i1, int j1, int nx, int ny, double* out) {
    GRID_STRIDE(e, (size_t)nx * ny) {
        const int i = (int)(e % nx), j = (int)(e / nx);
        out[e] = cropped[(size_t)(j1 + j) * cx + i1 + i];
    }
}

__global__ void kp_zero(double* X, size_t n) { GRID_STRIDE(i, n) X[i] = 0.0; }

// integrator helpers (perform_step!(integrator, ::BS3Cache))
__global__ void kp_stage(double* out, const double* uprev, double a, const double* k, size_t n) {
    GRID_STRIDE(i, n) out[i] = uprev[i] + a * k[i];
}

__global__ void kp_stage4(double* out, const double* uprev, double dt, const double* k1, const double* k2,
                          const double* k3, size_t n) {
    GRID_STRIDE(i, n) out[i] = uprev[i] + dt * (A41 * k1[i] + A42 * k2[i] + A43 * k3[i]);
}

__global__ void kp_err(const double* uprev, const double* u, const double* k1, const double* k2, const double* k3,
                       const double* k4, double dt, double abstol, double reltol, double* partial, size_t n) {
    __shared__ double red[32];
    double acc = 0.0;
    GRID_STRIDE(i, n) {
        const double ut = dt * (BT1 * k1[i] + BT2 * k2[i] + BT3 * k3[i] + BT4 * k4[i]);
        const double a = fabs(uprev[i]), b = fabs(u[i]);
        const double r = ut / (abstol + (a > b ? a : b) * reltol);
        acc += r * r;
    }
    double v[1] = {acc};
    block_sum<1>(v, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

// sums of squares for the initial-dt heuristic: s0 = sum (a/sk)^2, s1 = sum (b/sk)^2
__global__ void kp_norms2(const double* a, const double* b, const double* sk_base, double abstol, double reltol,
                          double* partial, size_t n) {
    __shared__ double red[64];
    double s0 = 0.0, s1 = 0.0;
    GRID_STRIDE(i, n) {
        const double sk = abstol + fabs(sk_base[i]) * reltol;
        const double x = a[i] / sk, y = b[i] / sk;
        s0 += x * x;
        s1 += y * y;
    }
    double v[2] = {s0, s1};
    block_sum<2>(v, red);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = v[0]; partial[2 * blockIdx.x + 1] = v[1]; }
}

__global__ void kp_initdt_terms(const double* f0, const double* f1, const double* sk_base, double abstol,
                                double reltol, double* partial, size_t n) {
    __shared__ double red[64];
    double s0 = 0.0, eq = 1.0;
    GRID_STRIDE(i, n) {
        const double sk = abstol + fabs(sk_base[i]) * reltol;
        const double x = (f1[i] - f0[i]) / sk;
        s0 += x * x;
        if (f1[i] != f0[i]) eq = 0.0;
    }
    double v[2] = {s0, eq};
    block_sum<2>(v, red);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = v[0]; partial[2 * blockIdx.x + 1] = v[1]; }
}

// ELRA (src/deformation.jl:29-45): the convolution input -(load + litho) g K^2 and
// dudt = (u_eq - u) / tau
__global__ void kp_elra_in(const double* s_load, const double* s_l, double g, double* out, size_t n) {
    GRID_STRIDE(i, n) out[i] = -(s_load[i] + s_l[i]) * g;
}
__global__ void kp_elra_dudt(const double* u_eq, const double* u, const double* tau, double* dudt, size_t n) {
    GRID_STRIDE(i, n) dudt[i] = 1.0 / tau[i] * (u_eq[i] - u[i]);
}

// Laterally-constant Maxwell step (src/deformation.jl:52-89): F = -(load + litho) g,
// U = u as complex inputs; then U <- ((nabla - dt/2 beta) U + dt F) / (nabla + dt/2 beta)
// with nabla = 2 eta |k| R and beta = rho_m g + D |k|^4, elementwise as the reference
// broadcasts them; then u = Re(ifft(U)).
__global__ void kp_lc_in(const double* s_load, const double* s_l, double g, const double* u, double2* F, double2* U,
                         size_t n) {
    GRID_STRIDE(i, n) {
        F[i] = make_double2(-(s_load[i] + s_l[i]) * g, 0.0);
        U[i] = make_double2(u[i], 0.0);
    }
}
__global__ void kp_lc_step(double2* U, const double2* F, const double* eta, const double* pd, const double* R,
                           const double* D, double rho_m_g, double dt, size_t n) {
    GRID_STRIDE(i, n) {
        const double k = pd[i];
        const double nab = 2.0 * eta[i] * k * R[i];
        const double beta = rho_m_g + D[i] * k * k * k * k;
        const double a = nab - dt / 2 * beta, b = nab + dt / 2 * beta;
        U[i] = make_double2((a * U[i].x + dt * F[i].x) / b, (a * U[i].y + dt * F[i].y) / b);
    }
}
__global__ void kp_real(const double2* U, double* u, size_t n) { GRID_STRIDE(i, n) u[i] = U[i].x; }

// Output staging of the FP32 form: out = [u | ue - cue | dudt - cdu | dz - cdz] in FP64
// (fields whose source is null are skipped).
__global__ void k_out_stage(const double* u, const float* ue, double cue, const float* dudt, double cdu,
                            const float* dz, double cdz, double* out, size_t n) {
    GRID_STRIDE(i, n) {
        if (u) out[i] = u[i];
        if (ue) out[n + i] = (double)ue[i] - cue;
        if (dudt) out[2 * n + i] = (double)dudt[i] - cdu;
        if (dz) out[3 * n + i] = (double)dz[i] - cdz;
    }
}

}  // namespace fi
