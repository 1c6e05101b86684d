/*
 * fi_oracle.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU FP64 restatement of the FastIsostasy.jl LV-ELVA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only
 * as the checker; the product library never links or calls it.
 *
 * The entry points mirror include/fastiso_b200.h with an or_ prefix and share
 * its fi_config struct and field identifiers, so a test drives both the same way.
 */
#ifndef FI_ORACLE_H
#define FI_ORACLE_H
#include "../include/fastiso_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_sim or_sim;

int or_create(const fi_config* cfg, or_sim** out);
int or_set_field(or_sim* s, int32_t field, const double* host, size_t n);
int or_get_field(or_sim* s, int32_t field, double* host, size_t n);
int or_set_ice_history(or_sim* s, int32_t K, const double* t, const double* H);
int or_set_elastic_table(or_sim* s, int32_t n, const double* rm, const double* GE);
int or_set_channel_scaling(or_sim* s, int32_t n, const double* ratio, const double* thick);
int or_init(or_sim* s);
int or_rhs(or_sim* s, double t, double* u_inout, double* dudt_out);
int or_run(or_sim* s, int32_t n_out, const double* t_out, double* out_t,
           double* out_u, double* out_ue, double* out_dudt, double* out_dz_ss);
int or_init_integrator(or_sim* s, int32_t n_tstops, const double* tstops);
int or_step(or_sim* s, double dt);
int or_resume(or_sim* s, double t, int64_t count_sparse, const double* u, const double* ue, const double* dz_ss,
              int32_t n_tstops, const double* tstops);
int or_record_steps(or_sim* s, int64_t cap);
int or_get_step_record(or_sim* s, double* dts, int64_t cap, int64_t* n);
int or_set_step_replay(or_sim* s, int64_t n, const double* dts);
int or_get_stats(or_sim* s, fi_stats* st);
int or_get_sealevel(or_sim* s, fi_sealevel* out);
int or_set_ocean_surface_table(or_sim* s, int32_t n, const double* z, const double* A);
int or_set_bsl_history(or_sim* s, int32_t n, const double* t, const double* z);
const char* or_last_error(const or_sim* s);
void or_destroy(or_sim* s);
void or_set_threads(int32_t n);

/* Known-answer helpers (reference KATs, test/test_derivatives.jl and
 * test/test_convolution.jl). */
int32_t or_nextfastfft(int32_t n);
void or_second_derivatives(int32_t nx, int32_t ny, double Dx, double Dy, const double* u,
                           double* uxx, double* uyy, double* ux, double* uxy);
int or_fft2(int32_t nx, int32_t ny, const double* in_re, const double* in_im,
            double* out_re, double* out_im, int32_t inverse);
int or_conv_full(int32_t nx, int32_t ny, const double* kernel, const double* input,
                 double* out);
/* Standalone BS3 + PI controller on u' = lambda*u (src/integrators.jl:205-217 check). */
int or_bs3_decay(double lambda, double u0, double t1, double reltol, double abstol,
                 int32_t n_out, const double* t_out, double* u_out, int64_t* nsteps);

#ifdef __cplusplus
}
#endif
#endif
