/*
 * fastiso_b200.h -- C ABI of the B200-native LV-ELVA hot path of FastIsostasy.jl.
 *
 * The library replaces the laterally-variable ELVA (elastic lithosphere, viscous
 * asthenosphere) right-hand side and the adaptive BS3 integrator that drives it:
 *
 *   update_diagnostics!(dudt, u, sim, t)          src/simulation.jl:335-393
 *   update_dudt!(.., ::MaxwellMantle, ::LaterallyVariableLithosphere)
 *                                                 src/deformation.jl:91-103
 *   update_deformation_rhs!                       src/deformation.jl:110-131
 *   update_elasticresponse!                       src/deformation.jl:175-184
 *   update_dz_ss!(::LaterallyVariableSeaSurface)  src/sealevel.jl:173-201
 *   samesize_conv!/conv!                          src/convolutions.jl:94-154
 *   run!(sim) -> solve(prob, BS3(); reltol)       src/simulation.jl:236-262
 *   init_integrator / step!(integrator, dt, true) src/simulation.jl:293-322
 *
 * All arrays crossing this boundary are host arrays of double in the Julia
 * column-major layout of the reference (element (i,j) at i + j*nx, x fastest,
 * dimension 1 = x; test/test_dimensions.jl:14-19).  The caller owns every host
 * buffer; each call copies in or out and keeps no pointer past its return.
 * The library owns its device memory, streams and CUDA graphs for the lifetime
 * of a handle.  A handle is not thread-safe; distinct handles may be used from
 * distinct host threads.  Every entry point returns FI_OK (0) or an FI_ERR_*
 * code; fi_last_error() returns the message of the last failure on a handle.
 */
#ifndef FASTISO_B200_H
#define FASTISO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FI_ABI_VERSION 2

/* ---- status codes (error(...) calls of the reference become these) ---- */
enum {
    FI_OK = 0,
    FI_ERR_ARG = 1,            /* invalid argument or size */
    FI_ERR_CUDA = 2,           /* CUDA runtime error */
    FI_ERR_NONFINITE = 3,      /* NaN/Inf in the error norm or state */
    FI_ERR_DT_UNDERFLOW = 4,   /* adaptive dt fell below dtmin */
    FI_ERR_FORCING_RANGE = 5,  /* "TimeInterpolation2D out of range." (src/interpolations.jl:51-58) */
    FI_ERR_TIMEOUT = 6,        /* a bounded device wait gave up */
    FI_ERR_STATE = 7,          /* call out of lifecycle order */
    FI_ERR_UNSUPPORTED = 8,    /* option outside the LV-ELVA path */
    FI_ERR_MAXITERS = 9        /* step budget exhausted */
};

/* ---- compute form ---- */
enum {
    FI_FORM_FP32 = 0,  /* fused kernels: FP32 FFTs, stencils and spectral multiplies,
                          FP64 state, first stencil and controller; CUDA graph */
    FI_FORM_FP64 = 1   /* plain form: one FP64 kernel per operation, host-driven loop */
};

/* ---- tags of the reference (src/solidearth.jl:13-109, src/sealevel.jl:114-130) ---- */
enum { FI_LITHO_LATERALLY_VARIABLE = 0, FI_LITHO_RIGID = 1, FI_LITHO_LATERALLY_CONSTANT = 2 };
/* solidearth.mantle (src/solidearth.jl:40-75): MaxwellMantle (the LV-ELVA default),
 * RelaxedMantle (ELRA: dudt = (u_eq - u) / tau with u_eq the Kelvin-function
 * convolution of the load, src/deformation.jl:29-45), RigidMantle (dudt = 0). */
enum { FI_MANTLE_MAXWELL = 0, FI_MANTLE_RELAXED = 1, FI_MANTLE_RIGID = 2 };
/* opts.diffeq.alg: BS3 (adaptive) or Euler with the fixed step dt_min, which the
 * laterally-constant Maxwell form needs (src/simulation.jl:236-262). */
enum { FI_ALG_BS3 = 0, FI_ALG_EULER = 1 };
enum { FI_SEA_SURFACE_LATERALLY_CONSTANT = 0, FI_SEA_SURFACE_LATERALLY_VARIABLE = 1 };
enum { FI_COLUMN_INCOMPRESSIBLE = 0, FI_COLUMN_COMPRESSIBLE = 1 };
enum { FI_ICE_TIME_INTERPOLATED = 0, FI_ICE_EXTERNAL = 1 };

/* Scalars of RegionalDomain, PhysicalConstants, SolidEarth, RegionalSeaLevel and
 * SolverOptions that the hot path reads.  fi_config_default() fills the
 * reference defaults (src/constants.jl:16-28, src/solidearth.jl:115-121,
 * src/simulation.jl:11-26). */
typedef struct fi_config {
    int32_t nx, ny;                 /* RegionalDomain(Wx, Wy, nx, ny), src/domain.jl:76 */
    double Wx, Wy;                  /* half-widths (m) */
    /* PhysicalConstants */
    double mE, r_pole, g, seconds_per_year;
    double rho_ice, rho_water, rho_seawater;
    /* SolidEarth scalars */
    double rho_litho, rho_uppermantle, litho_poissonratio;
    int32_t lithosphere;            /* FI_LITHO_* (Rigid => ue = 0, deformation.jl:186-189) */
    int32_t lithosphere_column;     /* FI_COLUMN_* (sealevel.jl:193-201) */
    /* RegionalSeaLevel with ConstantBSL and NoSealevelLoad */
    int32_t sea_surface;            /* FI_SEA_SURFACE_* */
    double z_bsl;                   /* ConstantBSL level (m) */
    /* boundary conditions: BoundaryConditions(...) x_border of the three CornerBCs */
    double bc_viscous_border, bc_elastic_border, bc_sea_surface_border;
    int32_t ice_mode;               /* FI_ICE_* */
    int32_t ice_flat_bc;            /* TimeInterpolation2D flat_bc */
    /* SolverOptions / DiffEqOptions */
    double t0, t1;                  /* t_span */
    double reltol, abstol;          /* reltol = Float64(1f-5), abstol = 1e-6 */
    double dt_sparse_diagnostics;   /* 10 yr */
    int64_t max_steps;              /* step-attempt budget per run/step call (0 = unlimited) */
    int32_t form;                   /* FI_FORM_* */
    int32_t device;                 /* CUDA device ordinal the handle runs on */
    /* RegionalSeaLevel beyond its surface (src/sealevel.jl:114-130,
     * src/barystatic_sealevel.jl): the sea-level load, the barystatic sea level
     * (BSL) and its update, the volume contributions.  Defaults: NoSealevelLoad,
     * ConstantBSL, InternalBSLUpdate, Goelzer volume and density contributions, no
     * adjustment contribution.  z_bsl above is the ReferenceBSL level ref.z. */
    int32_t sealevel_load;          /* FI_SEALEVEL_LOAD_* */
    int32_t bsl_mode;               /* FI_BSL_* */
    int32_t bsl_update;             /* FI_BSL_UPDATE_* */
    int32_t volume_contribution;    /* FI_CONTRIB_NONE or FI_CONTRIB_GOELZER */
    int32_t density_contribution;   /* FI_CONTRIB_NONE or FI_CONTRIB_GOELZER */
    int32_t adjustment_contribution;/* FI_CONTRIB_NONE or FI_CONTRIB_GOELZER */
    double bsl_ref_A;               /* ReferenceBSL ocean area ref.A (m^2), A_OCEAN_PD = 3.625e14 */
    /* rheology and integrator beyond the LV-ELVA path (the plain FP64 form runs them) */
    int32_t mantle;                 /* FI_MANTLE_* */
    int32_t alg;                    /* FI_ALG_* */
    double dt_min;                  /* DiffEqOptions dt_min (yr) of FI_ALG_EULER */
} fi_config;

/* sealevel.load (src/loads.jl:1-27) */
enum { FI_SEALEVEL_LOAD_NONE = 0, FI_SEALEVEL_LOAD_INTERACTIVE = 1 };
/* sealevel.bsl (src/barystatic_sealevel.jl:100-200): ConstantBSL; ConstantOceanSurfaceBSL
 * (z += dV / ref.A); PiecewiseConstantBSL (z += dV / A, then A = A_itp(z) from the table
 * of fi_set_ocean_surface_table); ImposedBSL (z = z_itp(t) from fi_set_bsl_history). */
enum { FI_BSL_CONSTANT = 0, FI_BSL_CONSTANT_OCEAN_SURFACE = 1, FI_BSL_PIECEWISE_CONSTANT = 2, FI_BSL_IMPOSED = 3 };
/* sealevel.update_bsl: InternalBSLUpdate / ExternalBSLUpdate (delta_V only) */
enum { FI_BSL_UPDATE_INTERNAL = 0, FI_BSL_UPDATE_EXTERNAL = 1 };
/* volume / density / adjustment contributions (src/sealevel.jl:260-332) */
enum { FI_CONTRIB_NONE = 0, FI_CONTRIB_GOELZER = 1 };

/* Fields addressable by fi_set_field / fi_get_field.  All are nx*ny doubles. */
enum {
    FI_FIELD_LITHO_RIGIDITY = 0,      /* SolidEarth.litho_rigidity D (set, required) */
    FI_FIELD_EFFECTIVE_VISCOSITY = 1, /* SolidEarth.effective_viscosity (set, required) */
    FI_FIELD_PSEUDODIFF_SCALING = 2,  /* SolidEarth.pseudodiff_scaling R, spectral index
                                         (set optional; default from channel layers or 1) */
    FI_FIELD_MASKACTIVE = 3,          /* SolidEarth.maskactive as 0/1 (set optional) */
    FI_FIELD_U_REF = 4,               /* Simulation(...; u_ref) */
    FI_FIELD_UE_REF = 5,              /* Simulation(...; ue_ref) */
    FI_FIELD_DZ_SS_REF = 6,           /* Simulation(...; dz_ss_ref) */
    FI_FIELD_Z_B_REF = 7,             /* Simulation(...; z_b_ref), default 1e6 */
    FI_FIELD_U = 8,                   /* sim.now.u (get; set before fi_init overrides u_ref copy) */
    FI_FIELD_UE = 9,                  /* sim.now.ue */
    FI_FIELD_DUDT = 10,               /* sim.now.dudt */
    FI_FIELD_DZ_SS = 11,              /* sim.now.dz_ss */
    FI_FIELD_H_ICE = 12,              /* sim.now.H_ice (set for FI_ICE_EXTERNAL) */
    FI_FIELD_Z_SS = 13,               /* sim.now.z_ss */
    FI_FIELD_Z_B = 14,                /* sim.now.z_b */
    FI_FIELD_ELASTIC_GREEN = 15,      /* GIATools elastic Green's function (get) */
    FI_FIELD_DZ_SS_GREEN = 16,        /* GIATools sea-surface Green's function (get) */
    FI_FIELD_PSEUDODIFF = 17,         /* RegionalDomain.pseudodiff (get) */
    FI_FIELD_SCALED_PSEUDODIFF_INV = 18, /* SolidEarth.scaled_pseudodiff_inv (get) */
    FI_FIELD_COLUMNANOM_LOAD = 19,    /* sim.now.columnanoms.load (get) */
    FI_FIELD_COLUMNANOM_FULL = 20,    /* sim.now.columnanoms.full (get) */
    FI_FIELD_H_AF = 21,               /* sim.now.H_af (get) */
    FI_FIELD_MASKGROUNDED = 22,       /* sim.now.maskgrounded as 0/1 (get) */
    FI_FIELD_MASKOCEAN = 23,          /* sim.now.maskocean as 0/1 (get) */
    FI_FIELD_H_WATER = 24,            /* sim.now.H_water (get) */
    FI_FIELD_COLUMNANOM_SEAWATER = 25,/* sim.now.columnanoms.seawater (get) */
    FI_FIELD_TAU = 26,                /* SolidEarth.tau, ELRA relaxation time in yr (set; default 855) */
    FI_FIELD_U_EQ = 27,               /* sim.now.u_eq, ELRA equilibrium displacement (get) */
    FI_NUM_FIELDS = 28
};

/* Barystatic sea level and the volume terms of the last sparse update (sim.now.z_bsl,
 * sim.sealevel.bsl.A, sim.now.V_af / V_den / V_pov / delta_V).  The FP32 form keeps the
 * volumes only when they can act on the solution (an interactive sea-level load or a
 * BSL other than ConstantBSL); otherwise `tracked` is 0 and they read 0. */
typedef struct fi_sealevel {
    double z_bsl, A_bsl;
    double V_af, V_den, V_pov, delta_V;
    int32_t tracked;
    int32_t pad;
} fi_sealevel;

typedef struct fi_stats {
    double t;                 /* integrator time (yr) */
    double dt;                /* proposed next dt (yr) */
    int64_t nf;               /* RHS evaluations (update_diagnostics! calls) */
    int64_t naccept, nreject; /* step attempts */
    int64_t nsparse;          /* sparse elastic / sea-surface updates (count_sparse_updates) */
    int32_t status;           /* FI_OK or the device status code */
    int32_t form;
    double gpu_ms;            /* device time of integration calls so far (CUDA events on
                                 the handle's stream), ms */
    double last_gpu_ms;       /* device time of the last fi_run / fi_step call, ms */
    int64_t segments;         /* step-loop launches (one per output segment) */
    int32_t executor;         /* FP32 step executor: FI_EXEC_* */
    int32_t grid;             /* blocks of the persistent executor (0 otherwise) */
} fi_stats;

/* Step executors of the FP32 form; the environment variable FI_EXECUTOR
 * (persist | graph | loop) read by fi_create selects one, default persist.
 * persist: one cooperative persistent kernel per output segment; graph: a CUDA
 * graph with conditional nodes, one kernel per phase; loop: the same kernels
 * launched from a host loop.  All three compute bitwise identical results. */
enum { FI_EXEC_PERSIST = 0, FI_EXEC_GRAPH = 1, FI_EXEC_LOOP = 2 };

typedef struct fi_handle fi_handle;

/* Fill cfg with the reference defaults for a domain of 2Wx x 2Wy and nx x ny cells. */
void fi_config_default(fi_config* cfg, int32_t nx, int32_t ny, double Wx, double Wy);

/* Simulation(domain, bcs, sealevel, solidearth, t_span; ...) -- src/simulation.jl:105-156.
 * Allocates device state; fields are set afterwards. */
int fi_create(const fi_config* cfg, fi_handle** out);

/* Copy a host field (nx*ny doubles) to / from the device. */
int fi_set_field(fi_handle* h, int32_t field, const double* host, size_t n);
int fi_get_field(fi_handle* h, int32_t field, double* host, size_t n);

/* TimeInterpolatedIceThickness(t_vec, H_vec, domain) -- src/boundary_conditions.jl:36-40.
 * K snapshots, H is K*nx*ny doubles, t strictly increasing. */
int fi_set_ice_history(fi_handle* h, int32_t K, const double* t, const double* H);

/* get_greenintegrand_coeffs -> build_greenintegrand -> get_elastic_green
 * (src/dataloaders.jl:257-273, src/material.jl:299-364, src/tools.jl:64-71):
 * the elastic Green's function is integrated in FP64 on the device from the
 * Farrell (1972) table (distance rm in m, coefficients GE), n entries. */
int fi_set_elastic_table(fi_handle* h, int32_t n, const double* rm, const double* GE);

/* FreqDomainViscosityLumping channel scaling (src/material.jl:154-179, 232-278):
 * n channels, each with its mask-mean viscosity ratio and mean thickness (m).
 * R(|k|) is evaluated in FP64 on the device.  Without this call (or a
 * FI_FIELD_PSEUDODIFF_SCALING field) R = 1, the one-layer case. */
int fi_set_channel_scaling(fi_handle* h, int32_t n, const double* visc_ratio_mean,
                           const double* channel_thickness_mean);

/* ReferenceBSL(z).A_itp (src/barystatic_sealevel.jl:36-42): the ocean surface area A(z)
 * of PiecewiseConstantBSL, n strictly increasing levels z (m) with areas A (m^2) --
 * the caller's copy of the table the reference downloads (unbiased so that A(0) is
 * A_OCEAN_PD); linear inside, and z outside [z_0, z_{n-1}] is FI_ERR_FORCING_RANGE. */
int fi_set_ocean_surface_table(fi_handle* h, int32_t n, const double* z, const double* A);

/* ImposedBSL(t_vec, z_vec) (src/barystatic_sealevel.jl:172-181): z_bsl(t) linear in time. */
int fi_set_bsl_history(fi_handle* h, int32_t n, const double* t, const double* z);

/* No counterpart in the reference: tile shape of the FP32 kernels, between fi_create
 * and fi_init.  h_rows: rows per row task (row FFTs, stencils), B_cols: spectral
 * columns per column task, both in [1, 16].  Small tiles favour a single simulation
 * (latency), tall tiles an ensemble (throughput); fastiso_b200.autotune measures them.
 * Results agree to FP32 rounding across tile shapes (the row FFTs pair halo rows
 * differently). */
int fi_set_tiles(fi_handle* h, int32_t h_rows, int32_t B_cols);

/* No counterpart in the reference (which calls FFTW/CUFFT plans): the radix schedule of
 * the library's transforms of length L (nx, ny or the padded convolution lengths Mx,
 * My), between fi_create and fi_init.  radices[0..n) are the Stockham passes in order;
 * they must multiply to L.  Radices 2, 3, 4, 5, 7 and 8 run register butterflies,
 * any other factor a generic O(R^2) pass.  The default is radix 8 while possible, then
 * 4, 2, 7, 5, 3.  fastiso_b200.autotune measures schedules.  Results agree to rounding
 * across schedules.  fi_get_fft_schedule writes the current one (at most 20 passes). */
int fi_set_fft_schedule(fi_handle* h, int32_t L, int32_t n, const int32_t* radices);
int fi_get_fft_schedule(fi_handle* h, int32_t L, int32_t* n, int32_t* radices);

/* Reference state + init_problem! (src/simulation.jl:129-156, 305-312): builds the
 * Green's functions and spectral factors, the reference state, and performs the
 * first RHS evaluation (which forces the sparse update). */
int fi_init(fi_handle* h);

/* One update_diagnostics!(dudt, u, sim, t) call with all its side effects on the
 * state (sparse update gate, column anomalies).  u is modified in place by the
 * viscous corner boundary condition exactly as in the reference. */
int fi_rhs(fi_handle* h, double t, double* u_inout, double* dudt_out);

/* No counterpart in the reference: fi_rhs for callers that may not allocate
 * memory, e.g. a coupled ice-sheet model that keeps its state in device
 * arrays and runs with device memory fully reserved by its own pool, or that
 * cannot afford the device-wide synchronisation of cudaMalloc/cudaFree inside
 * its time loop.  u_dev / dudt_dev are DEVICE pointers (nx*ny doubles, layout as
 * for fi_set_field) on the handle's device; same results and side effects as
 * fi_rhs.  FP32 form only.  On success the call allocates nothing, on the device
 * or the host: its result scratch is a static device array of
 * FI_NOALLOC_MAX_CELLS * 4 + 256 bytes (4 MiB) per device, and grids with more
 * than FI_NOALLOC_MAX_CELLS cells are rejected with FI_ERR_ARG.  The first call
 * on each device looks up the scratch address once (cudaGetSymbolAddress, that
 * device current); make that first call before any stream capture starts.  All
 * handles on a device share the scratch: calls that overlap in time on one
 * device (from several host threads) race on it and must be serialised by the
 * caller.  The call returns after its device work has finished.  The cached
 * scratch address belongs to the device's primary context: like every handle, it
 * does not survive cudaDeviceReset (create new handles after a reset, and do not
 * call fi_rhs_noalloc again in that process). */
#define FI_NOALLOC_MAX_CELLS (1024 * 1024)
int fi_rhs_noalloc(fi_handle* h, double t, double* u_dev, double* dudt_dev);

/* run!(sim) with NativeOutput times t_out (src/simulation.jl:236-262): integrates
 * t0 -> t1 with BS3 and the reference tolerances; at each output (same callback
 * semantics as nout_condition/nout_affect!) copies u, ue, dudt and dz_ss into
 * out_* (n_out*nx*ny each, any may be NULL) and the output time into out_t. */
int fi_run(fi_handle* h, int32_t n_out, const double* t_out, double* out_t,
           double* out_u, double* out_ue, double* out_dudt, double* out_dz_ss);

/* init_integrator(sim) (src/simulation.jl:293-303) with tstops; then
 * fi_step(h, dt) = step!(integrator, dt, true) (src/simulation.jl:319-322). */
int fi_init_integrator(fi_handle* h, int32_t n_tstops, const double* tstops);
int fi_step(fi_handle* h, double dt);

/* No counterpart in the reference (whose step sequence is OrdinaryDiffEq's own):
 * record and replay of the accepted step sizes, to separate the arithmetic error of
 * one compute form from the effect of a different accept/reject sequence.
 * fi_record_steps(h, cap): from now on the dt of every accepted step is stored (the
 * first cap of them; cap = 0 stops recording).  fi_get_step_record copies up to cap
 * stored values into dts and writes into *n how many steps were accepted since
 * recording started (more than stored when the record overflowed).
 * fi_set_step_replay(h, n, dts): the next n step attempts take exactly the step
 * sizes dts[0..n) and are all accepted (no error control); afterwards the adaptive
 * controller resumes from the last step.  Both need fi_init_integrator; a run that
 * replays the record of another handle with the same inputs and tstops visits the
 * same times, so the two solutions can be compared at every output. */
int fi_record_steps(fi_handle* h, int64_t cap);
int fi_get_step_record(fi_handle* h, double* dts, int64_t cap, int64_t* n);
int fi_set_step_replay(fi_handle* h, int64_t n, const double* dts);

/* Counters of the integrator and the RHS. */
int fi_get_stats(fi_handle* h, fi_stats* st);

/* sim.now.z_bsl, bsl.A and the volume terms of the last sparse update. */
int fi_get_sealevel(fi_handle* h, fi_sealevel* out);

/* Checkpoint: the full integrator + diagnostic state, behind a header that names the
 * library's checkpoint version, the compute form and the grid.  fi_checkpoint with
 * buf == NULL writes the needed size into *size.  fi_restore checks the header, the
 * size and the tstop count against the handle before it changes anything: a
 * checkpoint of another form, grid or version, a truncated buffer or a corrupt count
 * is rejected with FI_ERR_ARG and leaves the handle as it was.  A recording or replay
 * installed on the handle (fi_record_steps, fi_set_step_replay) is kept. */
int fi_checkpoint(fi_handle* h, void* buf, size_t* size);
int fi_restore(fi_handle* h, const void* buf, size_t size);

/* Diagnostics (no counterpart in the reference): times each fused FP32 kernel with
 * CUDA events over `reps` back-to-back launches on the handle's stream and writes the
 * mean ms per launch of k_rows_fwd (stage 2), k_cols, k_rows_inv (stage 2),
 * k_conv_rows, k_conv_cols and k_conv_rows_inv into ms[0..5].  It overwrites the
 * handle's state; use a separate handle. */
int fi_time_kernels(fi_handle* h, int32_t reps, double* ms);

/* Diagnostics (no counterpart in the reference): phase timeline of the persistent
 * FP32 executor.  fi_trace_phases(h, 1) clears the sums and starts recording,
 * fi_trace_phases(h, 0) stops.  fi_get_phase_trace writes FI_NUM_PHASES sums of
 * time (ms, as seen by block 0: the phase's slowest block plus the grid barrier)
 * and counts, in the order conv rows, conv columns, conv rows-inverse, rows(2),
 * columns(2), rows(3), columns(3), rows(4), columns(4), rows-inverse(4) + error
 * norm, controller. */
#define FI_NUM_PHASES 11
int fi_trace_phases(fi_handle* h, int32_t on);
int fi_get_phase_trace(fi_handle* h, double* ms, int64_t* counts);

/* ---- batched ensembles: no counterpart in the reference (its only batching is the
 * host-threaded ensemble of ext/FastIsostasyEnsembleKalmanProcessesExt.jl:107-122).
 * An ensemble groups initialised FP32 handles on one device, each with its own grid,
 * fields, tolerances and integrator (fi_init_integrator called).  fi_ensemble_step(e,
 * dt, status) is step!(integrator_m, dt, true) for every member m, all members
 * advancing together in one persistent cooperative kernel per segment; status[m]
 * (n entries, may be NULL) receives each member's FI_* code, and a failing member does not stop the others.
 * fi_ensemble_last_gpu_ms: device time of the last fi_ensemble_step (first start to
 * last end over the members' streams).  The ensemble does not own its members. */
typedef struct fi_ensemble fi_ensemble;
int fi_ensemble_create(fi_handle* const* members, int32_t n, fi_ensemble** out);
int fi_ensemble_step(fi_ensemble* e, double dt, int32_t* status);
double fi_ensemble_last_gpu_ms(const fi_ensemble* e);
/* Phase timeline of the persistent ensemble executor (FI_ERR_UNSUPPORTED for the
 * stream executor): on = 1 clears and starts recording, 0 stops, -1 leaves it; ms and
 * counts (FI_NUM_PHASES each, may be NULL) receive the sums as fi_get_phase_trace.
 * FI_ENS_EXECUTOR=streams (read by fi_ensemble_create) selects the stream executor:
 * one CUDA graph per member on its own stream. */
int fi_ensemble_trace(fi_ensemble* e, int32_t on, double* ms, int64_t* counts);
void fi_ensemble_destroy(fi_ensemble* e);

/* ---- Fourier-neural-operator surrogate (no counterpart in the reference) ----
 * fi_fno_gemm: C[z] = A[z] * B[z]^T for z < batch on the 5th-generation tensor cores
 * (tcgen05, BF16 inputs, FP32 accumulation in tensor memory), the channel-mixing and
 * truncated-DFT kernel of the surrogate, exposed for testing.  Device pointers; A is
 * M x K and B is N x K with K-contiguous rows (pitches lda, ldb, elements), C is M x N
 * FP32 (pitch ldc); sA, sB, sC are batch strides in elements.  flags bit 0: A is
 * MN-major (element (m, k) at A[k*lda + m]), bit 1: B is MN-major (element (n, k) at
 * B[k*ldb + n]).  K, lda, ldb, sA, sB and an MN-major operand's M (N) must be multiples
 * of 8 and A, B 16-byte aligned (FI_ERR_ARG otherwise). */
int fi_fno_gemm(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, const void* B, int32_t ldb,
                float* C, int32_t ldc, int32_t batch, int64_t sA, int64_t sB, int64_t sC, int32_t flags);

/* The surrogate network: input x [B][6][S][S] FP32 (x fastest; the caller's normalised
 * fields), output y [B][S][S] FP32.  Lift 6 -> 32, four Fourier layers of width 32
 * keeping kx in [0,16) x ky in {0..15, S-16..S-1} (GELU after the first three),
 * projection 32 -> 128 (GELU) -> 1.  S is a multiple of 32 in [32, 256]; batches are
 * 1..max_batch.  All tensors are device pointers; every call returns after its work has
 * finished.  Parameters are one flat FP32 vector in this order: P[32][6], bP[32]; per
 * layer: W[512 modes (kx*32 + kyi)][re, im][ci 32][co 32], Wloc[co][ci], bloc[32];
 * Q1[128][32], b1[128], Q2[128], b2.  seed draws the default initialisation. */
typedef struct fi_fno fi_fno;
int fi_fno_create(int32_t S, int32_t max_batch, int32_t device, uint64_t seed, fi_fno** out);
int64_t fi_fno_num_params(const fi_fno* h);
int fi_fno_get_params(fi_fno* h, float* out, int64_t n);      /* host buffer of n floats */
int fi_fno_set_params(fi_fno* h, const float* in, int64_t n); /* also resets Adam's moments */
int fi_fno_get_grads(fi_fno* h, float* out, int64_t n);
int fi_fno_forward(fi_fno* h, int32_t B, const float* x, float* y);
/* gradients of sum(dy * y) for the last fi_fno_forward (same B), overwriting the previous */
int fi_fno_backward(fi_fno* h, int32_t B, const float* dy);
/* forward, mean-squared-error loss against target [B][S][S], backward, one Adam step */
int fi_fno_train_step(fi_fno* h, int32_t B, const float* x, const float* target, float lr, float* loss);
/* the same with per-sample loss weights w [B] (device): loss = mean over samples and
 * cells of w_b (y - target)^2 */
int fi_fno_train_step_weighted(fi_fno* h, int32_t B, const float* x, const float* target, const float* w,
                               float lr, float* loss);
int fi_fno_adam(fi_fno* h, float lr); /* one Adam step with the current gradients */
/* Data-parallel training: forward, loss and backward without the optimizer step, then
 * the caller reduces the gradient vector (fi_fno_grads_device: num_params floats on the
 * handle's device, valid for its lifetime) across ranks in place, e.g. an NCCL
 * all-reduce averaged over the ranks, and calls fi_fno_adam on every rank.  Ranks that
 * start from the same parameters stay identical. */
int fi_fno_loss_backward(fi_fno* h, int32_t B, const float* x, const float* target, const float* w, float* loss);
void* fi_fno_grads_device(fi_fno* h);
int fi_fno_set_adam(fi_fno* h, float beta1, float beta2, float eps); /* default 0.9, 0.999, 1e-8 */
const char* fi_fno_last_error(const fi_fno* h);
void fi_fno_destroy(fi_fno* h);

/* Diagnostics (no counterpart in the reference): bounds of the library's device
 * waits, process-wide, for the launches that follow.  FI_WAIT_GRID_POLLS: polls of a
 * grid-barrier wait in the persistent step kernel (default 2^24, >= 1 s);
 * FI_WAIT_GRID_EXTRA_ARRIVALS: arrivals a grid barrier expects beyond the launched
 * grid (default 0; a positive value makes every barrier wait run out, which the
 * kernel reports as FI_ERR_TIMEOUT); FI_WAIT_TC_POLLS: polls of a tensor-core commit
 * wait in the surrogate's GEMMs (default 2^26; 0 makes the first wait give up at
 * once: the kernel then lets its issued MMAs finish, frees its tensor memory and
 * reports FI_ERR_TIMEOUT).  value < 0 restores the default.  Tests use this to show
 * that an expired wait returns an error and leaves the context usable. */
enum { FI_WAIT_GRID_POLLS = 0, FI_WAIT_GRID_EXTRA_ARRIVALS = 1, FI_WAIT_TC_POLLS = 2 };
int fi_debug_set_wait_limit(int32_t which, int64_t value);

const char* fi_last_error(const fi_handle* h);
const char* fi_status_string(int32_t status);
void fi_destroy(fi_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* FASTISO_B200_H */
