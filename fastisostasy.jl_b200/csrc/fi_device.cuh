// fi_device.cuh -- device helpers shared by the fused and plain forms:
// step-size controller, sparse-update gate, ice interpolation, block reductions.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "../../include/fastiso_b200.h"
#include "fi_internal.cuh"

namespace fi {

__host__ __device__ inline double ulp_above(double x) {
    x = fabs(x);
    return nextafter(x, INFINITY) - x;
}

__host__ __device__ inline double dtmin_at(double dtmin, double t) {
    const double e = ulp_above(t);
    return dtmin > e ? dtmin : e;
}

// interpolate(x, ::TimeInterpolation0D) with flat_bc = false (src/interpolations.jl:20-40):
// linear inside [xs[0], xs[n-1]], FI_ERR_FORCING_RANGE outside.
__host__ __device__ inline int interp0d(const double* xs, const double* ys, int n, double x, double* y) {
    if (n < 2 || !(x >= xs[0]) || x > xs[n - 1]) return FI_ERR_FORCING_RANGE;
    int lo = 0, hi = n - 1;  // last index with xs[lo] <= x, lo < n - 1
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (xs[mid] <= x) lo = mid; else hi = mid;
    }
    const double w = (x - xs[lo]) / (xs[lo + 1] - xs[lo]);
    *y = ys[lo] + w * (ys[lo + 1] - ys[lo]);
    return FI_OK;
}

// update_bsl!(bsl, -delta_V, t) of each BSL (src/barystatic_sealevel.jl:215-235) on the
// control block's z_bsl / A_bsl; dV = -delta_V.  Tables: the ocean surface A(z) of
// PiecewiseConstantBSL, the history z(t) of ImposedBSL.
__host__ __device__ inline int bsl_update(Ctl* c, int mode, double ref_z, double ref_A, double dV, double t,
                                          const double* oz, const double* oA, int no, const double* ht,
                                          const double* hz, int nh) {
    switch (mode) {
        case FI_BSL_CONSTANT: c->z_bsl = ref_z; return FI_OK;
        case FI_BSL_CONSTANT_OCEAN_SURFACE:
            c->A_bsl = ref_A;
            c->z_bsl += dV / c->A_bsl;
            return FI_OK;
        case FI_BSL_PIECEWISE_CONSTANT: {
            c->z_bsl += dV / c->A_bsl;
            double A;
            const int st = interp0d(oz, oA, no, c->z_bsl, &A);
            if (st == FI_OK) c->A_bsl = A;
            return st;
        }
        case FI_BSL_IMPOSED: {
            double z;
            const int st = interp0d(ht, hz, nh, t, &z);
            if (st == FI_OK) c->z_bsl = z;
            return st;
        }
        default: return FI_ERR_ARG;
    }
}

// Sparse-update gate of update_diagnostics!: (t - t0)/dt_sparse >= count
// (src/simulation.jl:355-356).  When it fires, the elastic displacement of this
// call goes to the other ue buffer while z_b still reads the old one (the
// reference updates z_b before the elastic response, src/simulation.jl:341-362).
__device__ inline int gate_eval(const Member& m, Ctl* c, double t_rhs) {
    const int g = ((t_rhs - c->t0) / m.dt_sparse) >= (double)c->count_sparse;
    c->iue_zb = c->iue;
    if (g) {
        c->count_sparse += 1;
        c->iue ^= 1;
        // internal_update_bsl! of an ImposedBSL: z_bsl(t) (the volume-driven BSLs run in
        // the plain form, which sums the volumes first)
        if (m.bsl_imposed) {
            double z;
            if (interp0d(m.bslh_t, m.bslh_z, m.n_bslh, t_rhs, &z) == FI_OK) c->z_bsl = z;
            else c->status = FI_ERR_FORCING_RANGE;
        }
    }
    c->gate = g;
    return g;
}

// Loop header of the next step attempt (fix_dt_at_bounds!, modify_dt_for_tstops!,
// check_error!) -- OrdinaryDiffEqCore semantics.
__host__ __device__ inline void loopheader_prep(Ctl* c) {
    c->iter += 1;
    if (c->dt > c->dtmax) c->dt = c->dtmax;
    const double dm = dtmin_at(c->dtmin, c->t);
    if (c->dt < dm) c->dt = dm;
    const double rem = c->t_stop - c->t;
    if (rem < c->dt) c->dt = rem;
    if (c->max_steps > 0 && c->iter > c->max_steps) c->status = FI_ERR_MAXITERS;
    if (!(c->dt == c->dt)) c->status = FI_ERR_NONFINITE;
    else if (c->dt <= c->dtmin) c->status = FI_ERR_DT_UNDERFLOW;
}

// PI step-size controller + accept/reject (stepsize_controller!,
// step_accept_controller!, step_reject_controller!, _loopfooter!), given the two
// powers EEst^beta1 and qold^beta2.  Returns 1 if the step was accepted.  tout:
// output times (nout_condition).
__host__ __device__ inline int controller_update_pw(Ctl* c, double EEst, double q11, double qold_b2,
                                                    const double* tout) {
    c->EEst = EEst;
    if (!(EEst == EEst)) {
        c->status = FI_ERR_NONFINITE;
        c->accept_step = 0;
        return 0;
    }
    double q;
    if (EEst == 0.0) {
        q = 1.0 / QMAX;
    } else {
        q = q11 / qold_b2;
        c->q11 = q11;
        q = q / GAMMA;
        if (q > 1.0 / QMIN) q = 1.0 / QMIN;
        if (q < 1.0 / QMAX) q = 1.0 / QMAX;
    }
    const double ttmp = c->t + c->dt;
    // replay: this attempt took replay_dt[replay_i - 1]; its sign is the decision
    const bool replay = c->replay_n > 0 && c->replay_i <= c->replay_n;
    c->accept_step = replay ? (c->replay_dt[c->replay_i - 1] > 0.0) : (EEst <= 1.0);
    if (c->rec_dt && c->rec_n < c->rec_cap) c->rec_dt[c->rec_n] = c->accept_step ? c->dt : -c->dt;
    c->rec_n += 1;
    if (c->accept_step) {
        c->naccept += 1;
        c->qold = EEst > QOLDINIT ? EEst : QOLDINIT;
        const double dtnew = c->dt / q;
        const double ts = c->t_stop;
        const double big = c->t > ts ? c->t : ts;
        c->t = (fabs(ttmp - ts) < 100.0 * ulp_above(big)) ? ts : ttmp;
        double dp = dtnew < c->dtmax ? dtnew : c->dtmax;
        const double dm = dtmin_at(c->dtmin, c->t);
        c->dtpropose = dp > dm ? dp : dm;
        if (replay) {
            // the recorded sequence: the next attempt takes the next recorded dt
            if (c->replay_i < c->replay_n) c->dtpropose = fabs(c->replay_dt[c->replay_i]);
            c->replay_i += 1;
        }
        c->dt = c->dtpropose;  // apply_step!
        c->ibuf ^= 1;
        c->ik ^= 1;
        if (c->kout < c->nout && c->t >= tout[c->kout]) c->pending_output = 1;
    } else {
        c->nreject += 1;
        const double qq = c->q11 / GAMMA;
        c->dt /= (1.0 / QMIN < qq ? 1.0 / QMIN : qq);
        if (replay) {
            if (c->replay_i < c->replay_n) c->dt = fabs(c->replay_dt[c->replay_i]);
            c->replay_i += 1;
        }
    }
    return c->accept_step;
}

// Loop footer of a fixed-step Euler step (no error control): always accepted, t
// snapped to the tstop, the next step back to the fixed dt (clipped again at tstops by
// loopheader_prep).
__host__ __device__ inline void euler_accept(Ctl* c, double dt_fixed, const double* tout) {
    c->EEst = 0.0;
    c->accept_step = 1;
    if (c->rec_dt && c->rec_n < c->rec_cap) c->rec_dt[c->rec_n] = c->dt;
    c->rec_n += 1;
    c->naccept += 1;
    const double ttmp = c->t + c->dt;
    const double ts = c->t_stop;
    const double big = c->t > ts ? c->t : ts;
    c->t = (fabs(ttmp - ts) < 100.0 * ulp_above(big)) ? ts : ttmp;
    c->dtpropose = dt_fixed;
    c->dt = dt_fixed;
    c->ibuf ^= 1;
    c->ik ^= 1;
    if (c->kout < c->nout && c->t >= tout[c->kout]) c->pending_output = 1;
}

__host__ __device__ inline int controller_update(Ctl* c, double EEst, const double* tout) {
    const bool pw = (EEst == EEst) && EEst != 0.0;
    return controller_update_pw(c, EEst, pw ? pow(EEst, PI_BETA1) : 0.0, pw ? pow(c->qold, PI_BETA2) : 1.0, tout);
}

// TimeInterpolation2D lookup (src/interpolations.jl:51-74): snapshot index i and
// weight w such that H = H_i + (H_{i+1} - H_i) * w; w = 0 selects H_i exactly.
// Returns a status code.
__device__ inline int ice_lookup(const double* __restrict__ tt, int K, int flat, double t, int* i_out,
                                 double* w_out) {
    if (t < tt[0]) {
        *i_out = 0; *w_out = 0.0;
        return flat ? FI_OK : FI_ERR_FORCING_RANGE;
    }
    if (t > tt[K - 1]) {
        *i_out = K - 1; *w_out = 0.0;
        return flat ? FI_OK : FI_ERR_FORCING_RANGE;
    }
    int lo = 0, hi = K - 1;  // first index with tt[i] >= t
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (tt[mid] < t) lo = mid + 1; else hi = mid;
    }
    if (tt[lo] == t) { *i_out = lo; *w_out = 0.0; return FI_OK; }
    const int i = lo - 1;
    *i_out = i;
    *w_out = (t - tt[i]) / (tt[i + 1] - tt[i]);
    return FI_OK;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values per thread; result valid in every thread.
template <int NV>
__device__ __forceinline__ void block_sum(double* v, double* scratch /* >= 32*NV */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) scratch[wid * NV + k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double s = 0.0;
        for (int w = 0; w < nw; w++) s += scratch[w * NV + k];
        v[k] = s;
    }
    __syncthreads();
}

// Corner values v(0,y) and v(nx-1,y) of the real row whose half spectrum is A
// (normalisation already folded in): the inverse real DFT evaluated directly.
// Partial sums of this thread over k = tid, tid+nth, ...
template <typename C, typename T>
__device__ __forceinline__ void row_corner_partial(const C* A, int nx, const T* __restrict__ twr,
                                                   double* v0, double* v1) {
    // twr: forward twiddles exp(-2 pi i k / nx) as (re, im) pairs
    const int kmax = (nx - 1) / 2;
    double s0 = 0.0, s1 = 0.0;
    for (int k = threadIdx.x; k <= kmax; k += blockDim.x) {
        const C a = A[k];
        if (k == 0) {
            s0 += (double)a.x;
            s1 += (double)a.x;
        } else {
            const double wr = (double)twr[2 * k], wi = (double)twr[2 * k + 1];
            s0 += 2.0 * (double)a.x;
            s1 += 2.0 * ((double)a.x * wr - (double)a.y * wi);
        }
    }
    if ((nx % 2 == 0) && threadIdx.x == 0) {
        const C a = A[nx / 2];
        s0 += (double)a.x;
        s1 -= (double)a.x;
    }
    *v0 += s0;
    *v1 += s1;
}

}  // namespace fi
