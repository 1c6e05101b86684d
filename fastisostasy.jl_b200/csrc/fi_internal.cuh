// fi_internal.cuh -- device data layout of the LV-ELVA path.
//
// HBM layout per simulation ("member"; a single run is a batch of one):
//   FP64: integrator state u (uprev / unew double buffer, nx*ny each), x fastest.
//   FP32: stage derivatives k1..k4 in physical space (nx*ny each), rigidity D,
//         K/(2 eta_eff), ice snapshots, elastic/sea-surface fields, column-anomaly
//         history for the sparse update.
//   complex64: half spectrum S[y][kx] (kx in [0, nx/2], row pitch sp) shared by
//         the forward row pass, the column pass and the inverse row pass;
//         convolution spectra SA/SB[y][kx] (kx in [0, Mx/2], y < ny) and
//         cropped column output T[ry][kx].
//   spectral multipliers: viscous m[kx][ky] = spy / (nx ny R |k|) with DC = 0,
//         convolution kernels G[kx][ky] = rfft(pad(G)) / (Mx My), kx-major.
// All kernels take a member table and a task list (member, tile) so one launch
// serves one simulation or a mixed-size ensemble.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fi_fft.cuh"

namespace fi {

constexpr int MAX_TSTOPS = 4096;

// BS3 tableau (src/integrators.jl:154-173) and the OrdinaryDiffEq PI controller
// defaults for an order-3 method.
constexpr double A21 = 0.5, A32 = 0.75, A41 = 2.0 / 9.0, A42 = 1.0 / 3.0, A43 = 4.0 / 9.0;
constexpr double C2 = 0.5, C3 = 0.75;
constexpr double BT1 = -5.0 / 72.0, BT2 = 1.0 / 12.0, BT3 = 1.0 / 9.0, BT4 = -1.0 / 8.0;
constexpr double PI_BETA1 = 7.0 / 30.0, PI_BETA2 = 2.0 / 15.0;
constexpr double QMIN = 0.2, QMAX = 10.0, GAMMA = 0.9, QOLDINIT = 1e-4;

// Per-member integrator / diagnostic control block (device resident).
struct Ctl {
    // integrator (OrdinaryDiffEq semantics)
    double t, dt, dtpropose, qold, q11, EEst;
    double t0, t1, dtmax, dtmin, reltol, abstol;
    double t_stop;              // end of the current segment (next tstop)
    double t_call;              // time of a host-driven right-hand side call
    long long iter, naccept, nreject, nf, count_sparse, max_steps;
    int accept_step;
    int status;                 // FI_OK or an FI_ERR_* code
    int active;                 // the step loop runs while 1
    int ibuf;                   // uprev = u[ibuf], unew = u[ibuf ^ 1]
    int ik;                     // k1 = k14[ik], k4 = k14[ik ^ 1]
    int iue, iue_zb;            // ue buffers: current, and the one z_b reads this call
    int gate;                   // sparse update before the next RHS
    int pending_output;         // an output time was passed by the last accepted step
    int kout, nout;             // next output index / number of outputs
    int nsteps_seg;             // accepted+rejected attempts in the current segment
    int pad0;
    // corner values (x=0,y=0), (nx-1,0), (0,ny-1), (nx-1,ny-1) of raw buffers
    double kcorner[4][4];       // slots: 0/1 = k14 pair, 2 = k2, 3 = k3
    double ue_corner[2][4];     // raw convolution corners of the two ue buffers
    double dz_corner[4];
    unsigned int arrive;        // last-block counter of the error-norm reduction
    unsigned int arrive_pad;
    // Step-sequence replay and record (fi_set_step_replay / fi_record_steps): device
    // pointers in the FP32 form, host pointers in the plain form (host controller).
    // Every attempt appends its dt to rec_dt (up to rec_cap), negated when rejected.
    // While a replay runs, attempt i takes |replay_dt[i]| and is accepted iff
    // replay_dt[i] > 0.
    const double* replay_dt;
    double* rec_dt;
    long long replay_n, replay_i, rec_cap, rec_n;
    // barystatic sea level and ocean area (sim.now.z_bsl, sim.sealevel.bsl.A) and the
    // volume terms of the last sparse update (V_af, V_den, V_pov, delta_V)
    double z_bsl, A_bsl, V_af, V_den, V_pov, delta_V;
};

// Shared-memory layout of the forward row phase: byte offsets (16-byte aligned) of the
// staging buffers of one row tile.  An input whose offset is -1 is read in place from
// global memory (the layout is budgeted per member; results do not depend on it).
struct FwdLayout {
    int U;        // stage vector rows [loU, hiU), FP64 (prefetched uprev, updated in place)
    int MS;       // moments (3 x capM rows, FP32), aliased by the inverse-prologue FFT
    int KA, KB, KC;  // k1, k2, k3 rows [loU, hiU) (FP32)
    int S_in;     // previous stage's spectrum rows [loU, hiU) (complex)
    int D;        // rigidity rows [loM, hiM)
    int Ha, Hb, ue, uz, dz, visc, zbss, mask, hafref, sigref, ueref;  // own rows
    int R;        // -g sigma_full of the own rows
    int cpart;    // corner partials of the column tasks (4 doubles each)
    int stage_u;  // 1: uprev rows are copied into U asynchronously; 0: read in place
    int bytes;
};

// Per-member static description + device pointers.
struct Member {
    int nx, ny, NH, sp;         // grid, half-spectrum width nx/2+1, spectrum row pitch
    int Mx, My, MH, msp;        // convolution padded sizes, half width, pitch
    int i1, j1;                 // 0-based crop origin of samesize_conv
    int plan_x, plan_y, plan_Mx, plan_My;
    FftPlan px, py, pMx, pMy;   // copies of the plans (kernels stage them in shared memory)
    int K;                      // ice snapshots
    int ice_external, ice_flat;
    int elastic_on, geoid_on, column_compressible;
    int flags;                  // FLAG_* below
    double dx, dy, A;
    double g, rho_ice, rho_litho, rho_um, nu, rho_sw_ice, spy;
    double border_v, border_e, border_g;
    double dt_sparse;
    float zbss_scalar;
    int ncols;                  // column tasks (corner partials per right-hand side)
    int h_rows, B_cols, h_conv, B_conv;        // tile height / width of each phase
    int n_rows, n_crow, n_ccol, n_crowi;       // task counts (n_cols == ncols)
    FwdLayout fl;               // forward row phase staging layout
    // state
    double* u[2];               // FP64 state double buffer
    float* k14[2];              // k1 / k4 physical (raw, before the corner offset)
    float* k2;
    float* k3;
    // parameters
    const float* D;             // litho rigidity
    const float* visc_fac;      // K / (2 eta_eff)
    const float* mult;          // viscous spectral multiplier [kx][ky]
    const float* mask;          // maskactive (null = all ones)
    const float* H_af_ref;      // null = 0
    const float* sigma_ref;     // m (rho_i H_af_ref + rho_l ue_ref + rho_m u_ref), null = 0
    const float* zbss_ref;      // z_b_ref - z_ss_ref - z_bsl, null = zbss_scalar
    const float* ue_ref;        // null = 0 (compressible-column sea-surface input only)
    const double* t_ice;        // K times
    const float* H_tab;         // K * nx*ny snapshots
    float* H_ext;               // external ice (FI_ICE_EXTERNAL)
    float* ue[2];               // raw elastic displacement (before the corner offset)
    float* dz;                  // raw sea-surface perturbation
    float* sig_load;            // columnanoms.load of the last RHS call
    float* sig_geo;             // sea-surface convolution input of the last RHS call
    float2* S[2];               // viscous half spectrum [ny][sp], double-buffered (stage 3 uses S[1])
    float2* SA;                 // convolution spectrum, channel A [ny][msp]
    float2* SB;                 // convolution spectrum, channel B [ny][msp]
    float2* TA;                 // cropped column output, channel A [ny+2][msp]
    float2* TB;
    const float2* GA;           // kernel spectrum channel A [MH][My] (kx-major)
    const float2* GB;
    double* partial;            // error-norm partial sums per row tile
    double* cpart;              // corner partials [ncols][4] of the last column pass
    const double* tout;         // output times (nout_condition), ctl->nout entries
    Ctl* ctl;
    // sea level beyond the surface (src/loads.jl:56-85, src/topography.jl:1-28): the
    // seawater column anomaly of InteractiveSealevelLoad and the masks / water column
    // of the last sparse update; an ImposedBSL history
    int sl_interactive;         // sealevel.load isa InteractiveSealevelLoad
    int bsl_imposed;            // z_bsl(t) from bslh_t / bslh_z at each sparse update
    int n_bslh, pad_sl;
    double bsl_ref_z;           // ReferenceBSL z (the z_bsl folded into zbss_ref)
    double rho_sw;              // seawater density
    const double* bslh_t;
    const double* bslh_z;
    float* sw;                  // columnanoms.seawater
    float* mgr;                 // maskgrounded (0/1)
    float* moc;                 // maskocean (0/1)
    float* hwater;              // H_water
};

enum {
    FLAG_MASK = 1,
    FLAG_HAFREF = 2,
    FLAG_SIGREF = 4,
    FLAG_ZBSS = 8,
    FLAG_UEREF = 16,
};

struct Task {
    int member;
    int tile;
};

static_assert(sizeof(Member) % 8 == 0, "Member is copied as 8-byte words");
static_assert(sizeof(Ctl) % 8 == 0, "Ctl is copied as 8-byte words");
constexpr int TICE_MAX = 4096;  // ice-time tables up to this length are searched in shared memory

}  // namespace fi
