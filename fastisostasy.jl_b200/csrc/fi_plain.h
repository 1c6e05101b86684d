// fi_plain.h -- kernels of the plain FP64 form (fi_plain.cu).
#pragma once
#include <cuda_runtime.h>

namespace fi {
__global__ void kp_corner_off(const double* X, int nx, int ny, double border, double* off);
__global__ void kp_sub_off(double* X, size_t n, const double* off);
__global__ void kp_copy(double* dst, const double* src, size_t n);
__global__ void kp_bedrock(const double* u, const double* ue, const double* z_b_ref, const double* u_ref,
                           double* now_u, double* z_b, double* s_m, double rho_um, size_t n);
__global__ void kp_ice(const double* Ha, const double* Hb, double dti, double tt, int exact, double* H, size_t n);
__global__ void kp_haf_ice(const double* H, const double* z_b, const double* z_ss, const double* H_af_ref,
                           double* H_af, double* s_i, double rho_sw_ice, double rho_ice, size_t n);
__global__ void kp_litho(const double* ue, const double* ue_ref, double* s_l, double rho_l, size_t n);
__global__ void kp_geo_in(const double* s_load, const double* s_full, const double* s_m, const double* mask,
                          int compressible, double A, double* out, size_t n);
__global__ void kp_zss(const double* z_ss_ref, const double* dz, double z_bsl, double* z_ss, size_t n);
__global__ void kp_load_full(const double* s_i, const double* s_sw, const double* s_l, const double* s_m,
                             const double* mask, double* s_load, double* s_full, size_t n);
__global__ void kp_volumes(const double* H_af, const double* H, const double* z_ss, const double* z_b, double A,
                           double* partial, size_t n);
__global__ void kp_sealevel(const double* H, const double* H_af, const double* z_ss, const double* z_b,
                            const double* z_ss_ref, const double* mask, int interactive, double rho_sw,
                            double rho_i_sw, double* mgr, double* moc, double* hwater, double* s_sw, size_t n);
__global__ void kp_rhs_init(const double* s_full, double g, double* rhs, size_t n);
__global__ void kp_dxx(double* du, const double* u, int nx, int ny, double Dx);
__global__ void kp_dyy(double* du, const double* u, int nx, int ny, double Dy);
__global__ void kp_dx(double* du, const double* u, int nx, int ny, double Dx);
__global__ void kp_dy(double* du, const double* u, int nx, int ny, double Dy);
__global__ void kp_moments(const double* bxx, const double* byy, const double* bxy, const double* D, double nu,
                           double* Mxx, double* Myy, double* Mxy, size_t n);
__global__ void kp_rhs_acc(double* rhs, const double* bxx, const double* byy, const double* bxy, size_t n);
__global__ void kp_fftin(const double* rhs, const double* eta, double2* f, size_t n);
__global__ void kp_spec(double2* f, const double* spinv, size_t n);
__global__ void kp_real_spy(const double2* f, double spy, double* dudt, size_t n);
__global__ void kp_cmul(double2* P, const double2* G, size_t n);
__global__ void kp_crop(const double2* P, int Mx, int cx, int cy, double* out);
__global__ void kp_window(const double* cropped, int cx, int i1, int j1, int nx, int ny, double* out);
__global__ void kp_zero(double* X, size_t n);
__global__ void kp_stage(double* out, const double* uprev, double a, const double* k, size_t n);
__global__ void kp_stage4(double* out, const double* uprev, double dt, const double* k1, const double* k2,
                          const double* k3, size_t n);
__global__ void kp_err(const double* uprev, const double* u, const double* k1, const double* k2, const double* k3,
                       const double* k4, double dt, double abstol, double reltol, double* partial, size_t n);
__global__ void kp_norms2(const double* a, const double* b, const double* sk_base, double abstol, double reltol,
                          double* partial, size_t n);
__global__ void kp_initdt_terms(const double* f0, const double* f1, const double* sk_base, double abstol,
                                double reltol, double* partial, size_t n);
__global__ void kp_elra_in(const double* s_load, const double* s_l, double g, double* out, size_t n);
__global__ void kp_elra_dudt(const double* u_eq, const double* u, const double* tau, double* dudt, size_t n);
__global__ void kp_lc_in(const double* s_load, const double* s_l, double g, const double* u, double2* F, double2* U,
                         size_t n);
__global__ void kp_lc_step(double2* U, const double2* F, const double* eta, const double* pd, const double* R,
                           const double* D, double rho_m_g, double dt, size_t n);
__global__ void kp_real(const double2* U, double* u, size_t n);
__global__ void k_out_stage(const double* u, const float* ue, double cue, const float* dudt, double cdu,
                            const float* dz, double cdz, double* out, size_t n);
}  // namespace fi
