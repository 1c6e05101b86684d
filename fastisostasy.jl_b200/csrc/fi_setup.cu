// fi_setup.cu -- FP64 device set-up: 2D transforms, spectral factors, Green's
// functions and convolution-kernel spectra (GIATools, src/tools.jl:49-97).
#include <math.h>

#include "fi_device.cuh"
#include "fi_kernels.h"

namespace fi {

// ---------------------------------------------------------------------------
// FP64 complex 2D transform passes (x fastest, row pitch `pitch`), in place
// ---------------------------------------------------------------------------
size_t fft64_rows_smem(int nx, int rpb) { return (size_t)2 * rpb * nx * sizeof(double2); }
size_t fft64_cols_smem(int ny, int cpb) { return (size_t)2 * cpb * ny * sizeof(double2); }

__global__ void __launch_bounds__(256)
k_fft64_rows(double2* a, int nx, int ny, int pitch, const FftPlan* plans, int plan, int inverse, int rpb) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ FftPlan s_plan;
    const int y0 = blockIdx.x * rpb, nr = min(rpb, ny - y0);
    if (nr <= 0) return;
    if (threadIdx.x == 0) s_plan = plans[plan];
    double2* b0 = (double2*)smem;
    double2* b1 = b0 + (size_t)rpb * nx;
    for (int e = threadIdx.x; e < nr * nx; e += blockDim.x) {
        const int r = e / nx, x = e - r * nx;
        b0[e] = a[(size_t)(y0 + r) * pitch + x];
    }
    __syncthreads();
    double2* res = inverse ? fft_batch<true, double>(b0, b1, s_plan, nr, nx)
                           : fft_batch<false, double>(b0, b1, s_plan, nr, nx);
    for (int e = threadIdx.x; e < nr * nx; e += blockDim.x) {
        const int r = e / nx, x = e - r * nx;
        a[(size_t)(y0 + r) * pitch + x] = res[e];
    }
}

__global__ void __launch_bounds__(256)
k_fft64_cols(double2* a, int nx, int ny, int pitch, const FftPlan* plans, int plan, int inverse, int cpb,
             double scale) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ FftPlan s_plan;
    const int x0 = blockIdx.x * cpb, nc = min(cpb, nx - x0);
    if (nc <= 0) return;
    if (threadIdx.x == 0) s_plan = plans[plan];
    double2* b0 = (double2*)smem;
    double2* b1 = b0 + (size_t)cpb * ny;
    for (int e = threadIdx.x; e < nc * ny; e += blockDim.x) {
        const int y = e / nc, c = e - y * nc;
        b0[(size_t)c * ny + y] = a[(size_t)y * pitch + x0 + c];
    }
    __syncthreads();
    double2* res = inverse ? fft_batch<true, double>(b0, b1, s_plan, nc, ny)
                           : fft_batch<false, double>(b0, b1, s_plan, nc, ny);
    for (int e = threadIdx.x; e < nc * ny; e += blockDim.x) {
        const int y = e / nc, c = e - y * nc;
        double2 v = res[(size_t)c * ny + y];
        v.x *= scale;
        v.y *= scale;
        a[(size_t)y * pitch + x0 + c] = v;
    }
}

// ---------------------------------------------------------------------------
// |k| (src/domain.jl:151-155, src/derivatives.jl:201-223), the channel scaling
// R(|k|) of FreqDomainViscosityLumping (src/material.jl:232-278) and
// scaled_pseudodiff_inv = 1/(R |k|) (src/solidearth.jl:222), all in FP64.
// mult[kx][ky] = spy / (nx ny R |k|) for the half spectrum, DC set to zero: the
// DC mode only adds a constant that the corner BC of dudt removes exactly.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fftint_d(int i, int N) { return (double)(i <= N / 2 ? i : N - i); }

__device__ __forceinline__ double channel_scaling_d(double kappa, double T, double r) {
    const double C = cosh(T * kappa), S = sinh(T * kappa);
    double num = 0.0, den = 0.0;
    num += 2 * r * C * S;
    num += (1 - r * r) * T * T * kappa * kappa;
    num += r * r * S * S + C * C;
    den += (r + 1 / r) * C * S;
    den += (r - 1 / r) * T * kappa;
    den += S * S + C * C;
    return num / den;
}

__global__ void k_spectral_factors(int nx, int ny, double Wx, double Wy, int nch, const double* ratio,
                                   const double* thick, const double* R_given, double spy, double* pseudodiff,
                                   double* Rout, double* spinv, float* mult, int NH) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nx * ny) return;
    const int i = e % nx, j = e / nx;
    const double mux = M_PI / Wx, muy = M_PI / Wy;
    double pd;
    if (e == 0) {
        const double a = mux * 1.0, b = muy * 1.0;  // pseudodiff[2,1], pseudodiff[1,2]
        pd = 1e-3 * ((b + a) / 2);
    } else {
        const double a = mux * fftint_d(i, nx), b = muy * fftint_d(j, ny);
        pd = sqrt(a * a + b * b);
    }
    double R = 1.0;
    if (R_given) {
        R = R_given[e];
    } else {
        for (int l = 0; l < nch; l++) R *= channel_scaling_d(pd, thick[l], ratio[l]);
    }
    pseudodiff[e] = pd;
    Rout[e] = R;
    const double si = 1.0 / (R * pd);
    spinv[e] = si;
    if (i < NH) mult[(size_t)i * ny + j] = (e == 0) ? 0.0f : (float)(spy * si / ((double)nx * ny));
}

// ---------------------------------------------------------------------------
// Elastic Green's function: get_elastic_green (src/material.jl:340-364) with the
// 4-point Gauss-Legendre quadrature2D (src/utils.jl:118-177) of
// get_loadgreen (src/material.jl:318-332) over each cell.
// ---------------------------------------------------------------------------
__device__ double loadgreen_d(double r, const double* rm, const double* GE, int n) {
    if (r < 0.01) return GE[0] / (rm[1] * 1e12);
    if (r > rm[n - 1]) return 0.0;
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (rm[mid] <= r) lo = mid; else hi = mid;
    }
    const double w = (r - rm[lo]) / (rm[hi] - rm[lo]);
    const double v = (1.0 - w) * GE[lo] + w * GE[hi];
    return v / (r * 1e12);
}

__global__ void k_elastic_green(double* G, int nx, int ny, int mx, int my, double dx, double dy, const double* rm,
                                const double* GE, int n) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nx * ny) return;
    const int i = e % nx, j = e / nx;
    const double a = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
    const double b = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
    const double wa = (18.0 + sqrt(30.0)) / 36.0, wb = (18.0 - sqrt(30.0)) / 36.0;
    const double qx[4] = {-b, -a, a, b};
    const double qw[4] = {wb, wa, wa, wb};
    const int p = i - mx, q = j - my;
    const double x1 = p * dx, x2 = (p + 1) * dx, y1 = q * dy, y2 = (q + 1) * dy;
    const double mxx = 2.0 / (x2 - x1), pxx = -1.0 - mxx * x1;
    const double myy = 2.0 / (y2 - y1), pyy = -1.0 - myy * y1;
    double sum = 0.0;
    for (int u = 0; u < 4; u++)
        for (int v = 0; v < 4; v++) {
            const double xx = (qx[u] - pxx) / mxx, yy = (qx[v] - pyy) / myy;
            sum = sum + loadgreen_d(sqrt(xx * xx + yy * yy), rm, GE, n) * qw[u] * qw[v] / mxx / myy;
        }
    G[e] = sum;
}

// Sea-surface Green's function (get_dz_ss_green, src/sealevel.jl:208-219)
__global__ void k_geoid_green(double* G, int nx, int ny, double Wx, double Wy, double dx, double dy,
                              double r_pole, double mE) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nx * ny) return;
    const int i = e % nx, j = e / nx;
    const double x = -Wx + (i + 1) * dx, y = -Wy + (j + 1) * dy;
    const double R = sqrt(x * x + y * y);
    const double cap = r_pole / (2.0 * mE * sin((dx / 2) / (2.0 * r_pole)));
    double g = r_pole / (2.0 * mE * sin(R / (2.0 * r_pole)));
    if (!(g <= cap)) g = cap;
    G[e] = g;
}

// zero-padded copy into an Mx-by-My complex plane (_pad!, src/convolutions.jl:1-15)
__global__ void k_pad_real(const double* in, int nx, int ny, double2* P, int Mx, int My) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)Mx * My) return;
    const int i = (int)(e % Mx), j = (int)(e / Mx);
    double2 v = make_double2(0.0, 0.0);
    if (i < nx && j < ny) v.x = in[(size_t)j * nx + i];
    P[e] = v;
}

// kx-major FP32 half spectrum scaled by 1/(Mx My): out[kx][ky] = P[ky][kx] * scale
__global__ void k_half_spectrum32(const double2* P, int Mx, int My, int MH, double scale, float2* out) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)MH * My) return;
    const int kx = (int)(e / My), ky = (int)(e % My);
    const double2 v = P[(size_t)ky * Mx + kx];
    out[e] = make_float2((float)(v.x * scale), (float)(v.y * scale));
}

}  // namespace fi
