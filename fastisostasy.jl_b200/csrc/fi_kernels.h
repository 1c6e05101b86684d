// fi_kernels.h -- kernel declarations shared by the translation units.
#pragma once
#include <cuda_runtime.h>

#include "fi_internal.cuh"

namespace fi {

// ---- fused FP32 form (fi_fused.cu) ----
__global__ void k_gate(const Member* mems, int nmem, double t, int use_ctl_t);
__global__ void k_rows_fwd(const Member* mems, const Task* tasks, int stage, int h, const double* uin, int inv_prev);
__global__ void k_cols(const Member* mems, const Task* tasks, int B, int next_stage, cudaGraphConditionalHandle h_gate);
__global__ void k_rows_inv(const Member* mems, const Task* tasks, int stage, int h, float* vout, double* cout,
                           cudaGraphConditionalHandle h_gate, cudaGraphConditionalHandle h_loop);
__global__ void k_conv_rows(const Member* mems, const Task* tasks, int h);
__global__ void k_conv_cols(const Member* mems, const Task* tasks, int B);
__global__ void k_conv_rows_inv(const Member* mems, const Task* tasks, int h);
__global__ void k_segment_start(const Member* mems, int nmem, cudaGraphConditionalHandle h_gate,
                                cudaGraphConditionalHandle h_loop);
__global__ void kf_initdt_norms(const double* u, const float* v, const double* vc, double border, double abstol,
                                double reltol, double* partial, size_t n);
__global__ void kf_initdt_u1(double* u1, const double* u, const float* v, const double* vc, double border,
                             double dt0, size_t n);
__global__ void kf_initdt_d2(const double* u, const float* v0, const double* c0p, const float* v1,
                             const double* c1p, double border, double abstol, double reltol, double* partial,
                             size_t n);
size_t rows_fwd_smem(int ws_bytes, int nx, int K);
constexpr int ROW_THREADS = 512;
size_t cols_smem(int ny, int B);
size_t rows_inv_smem(int nx, int h, int ncols);
size_t conv_rows_smem(int Mx, int h);
size_t conv_cols_smem(int My, int B);

// ---- persistent step executor (fi_persist.cu) ----
constexpr long long PERSIST_SPIN_LIMIT = 1LL << 24;  // grid-barrier polls of >= 64 ns each, about 1 s or more
struct PersistArgs {
    const Member* mem;
    unsigned int* bar;  // grid barrier: [0] arrivals, [1] generation, [2] abort
    int h_rows, B_cols, h_conv, B_conv;
    int n_rows, n_cols, n_crow, n_ccol, n_crowi;
    int ws_bytes;       // phase workspace at the front of dynamic shared memory
    int tw_off[4];      // float2 offsets (after the workspace) of the x, y, Mx, My twiddles; -1: global
    int tice_off;       // float2 offset of the ice-time table, -1: read from global memory
    unsigned long long* trace;  // optional phase timeline: [2 * PH_COUNT] sums of ns and counts
    long long polls;            // grid-barrier wait bound (PERSIST_SPIN_LIMIT by default)
    unsigned int bar_extra;     // arrivals a barrier expects beyond the grid (0; > 0 only in
                                // the timeout test, which then sees FI_ERR_TIMEOUT)
    unsigned int pad_;
};
// phases of the persistent executor, as accumulated in PersistArgs::trace
enum {
    PH_CONV_ROWS = 0, PH_CONV_COLS, PH_CONV_ROWS_INV,
    PH_ROWS_FWD2, PH_COLS2, PH_ROWS_FWD3, PH_COLS3, PH_ROWS_FWD4, PH_COLS4, PH_ROWS_INV4, PH_CONTROLLER,
    PH_COUNT
};
// The persistent step kernel whose row and column transforms run the compiled radix
// sequences seqx / seqy (fi_fft.cuh seq_code), built for two blocks per SM (minb 2) or
// one (minb 1, larger register budget); pairs without a compiled kernel get the one
// that runs the plans' runtime passes.
const void* persist_kernel(int seqx, int seqy, int minb);
// fills the shared-memory layout fields of a and returns the dynamic shared memory bytes
size_t persist_layout(int nx, int ny, int Mx, int My, int K, int fwd_bytes, int h_rows, int ncols, int B_cols,
                      int h_conv, int B_conv, PersistArgs* a);

// ---- persistent ensemble executor (fi_ensemble.cu) ----
constexpr int ENS_MAX_MEMBERS = 256;
struct EnsArgs {
    const Member* mems;          // member descriptors (device)
    Ctl* const* ctls;            // their control blocks (device array of pointers)
    int nmem;
    unsigned int* bar;           // grid barrier words
    unsigned long long* counter; // task counter, monotonic within a launch
    int ws_bytes;                // phase workspace
    int tw_cap;                  // float2 slots of the staged twiddle table
    int tice_cap;                // doubles of the staged ice-time table
    unsigned long long* trace;   // optional phase timeline
};
// the ensemble kernel: dispatch 1 runs the compiled radix sequences of the member
// grids where a member's schedule has one, 0 always the plans' runtime passes
const void* ens_kernel(int dispatch);
size_t ens_layout(const Member* host_mems, int n, EnsArgs* a);

// ---- FP64 transforms and set-up (fi_setup.cu) ----
__global__ void k_fft64_rows(double2* a, int nx, int ny, int pitch, const FftPlan* plans, int plan, int inverse,
                             int rows_per_block);
__global__ void k_fft64_cols(double2* a, int nx, int ny, int pitch, const FftPlan* plans, int plan, int inverse,
                             int cols_per_block, double scale);
size_t fft64_rows_smem(int nx, int rows_per_block);
size_t fft64_cols_smem(int ny, int cols_per_block);
__global__ void k_spectral_factors(int nx, int ny, double Wx, double Wy, int nch, const double* ratio,
                                   const double* thick, const double* R_given, double spy, double* pseudodiff,
                                   double* Rout, double* spinv, float* mult, int NH);
__global__ void k_elastic_green(double* G, int nx, int ny, int mx, int my, double dx, double dy, const double* rm,
                                const double* GE, int n);
__global__ void k_geoid_green(double* G, int nx, int ny, double Wx, double Wy, double dx, double dy,
                              double r_pole, double mE);
__global__ void k_pad_real(const double* in, int nx, int ny, double2* P, int Mx, int My);
__global__ void k_half_spectrum32(const double2* P, int Mx, int My, int MH, double scale, float2* out);

}  // namespace fi
