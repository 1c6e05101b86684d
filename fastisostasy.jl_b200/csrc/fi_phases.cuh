// fi_phases.cuh -- the phases of one FP32 right-hand side as device functions.
//
// Both executors run these bodies: the persistent cooperative step kernel
// (fi_persist.cu, one launch per output segment, phases separated by a grid barrier)
// and the per-phase kernels of fi_fused.cu (host-driven calls, the CUDA-graph
// executor and per-phase timing).  A phase never writes the control block: the
// caller owns every control-block update.
//
//   ph_rows_fwd     stage state u = uprev + dt*sum(a_sj k_j) in FP64 -> corner BC
//                   (boundary_conditions.jl:144-148) -> column anomalies
//                   (loads.jl:31-106, topography.jl:30-39) -> flexure operator
//                   rhs = -g sigma_full + dxx Mxx + 2 dxy Mxy + dyy Myy with the CPU
//                   edge rules (deformation.jl:110-131, derivatives.jl:48-191;
//                   u-derivatives in FP64, moment derivatives in FP32) -> times
//                   K/(2 eta) -> real row FFT, two rows per complex FFT.  Stages 3
//                   and 4 first invert the previous stage's spectrum rows (with a
//                   2-row halo) to get k2 / k3.
//   ph_cols         column FFT, multiply by spy/(nx ny R|k|) with DC zeroed, inverse
//                   column FFT (deformation.jl:95-98, solidearth.jl:222); per task,
//                   its columns' share of the field's four corner values.
//   ph_rows_inv     inverse real row FFT -> dudt rows; optional BS3 error-norm terms.
//   ph_conv_*       padded linear convolutions of the elastic and sea-surface loads
//                   (convolutions.jl:94-154), crop window + raw corner values.
//
// Latency: the column and inverse-row phases first issue their global inputs as
// asynchronous copies into shared memory (cp.async), wait once, and then compute from
// shared memory.  The forward-row phase reads its inputs in place by default (measured
// faster: its sub-steps hide the loads), or stages them the same way where the member's
// shared-memory budget allows and staging is selected (FwdLayout offset -1: in place).
//
// The corner values of a dudt field (the dudt corner BC, deformation.jl:101) come from
// the column pass: each column task adds its columns' terms of the inverse real DFT
// at x = 0 and x = nx-1 for rows 0 and ny-1 (cpart); consumers sum the tasks in a fixed
// order.
//
// The half spectrum is double-buffered: stage 3 of a BS3 step uses S[1], every
// other right-hand side S[0], so a fused inverse+forward row phase reads the
// previous stage's rows (with halo) from one buffer while other row tiles of the
// same phase write the next stage into the other.
#pragma once
#include "fi_device.cuh"
#include "fi_kernels.h"

namespace fi {

constexpr int RT = ROW_THREADS, TX = 128, TY = RT / TX;

struct RowRanges {
    int y0, y1, loM, hiM, loU, hiU;
};

__host__ __device__ inline RowRanges row_ranges(int tile, int h, int ny) {
    RowRanges r;
    r.y0 = tile * h;
    r.y1 = r.y0 + h < ny ? r.y0 + h : ny;
    r.loM = (r.y0 == 0) ? 0 : r.y0 - 1;
    r.hiM = (r.y1 == ny) ? ny : r.y1 + 1;
    if (r.y0 == 0) r.hiM = r.hiM > (ny < 3 ? ny : 3) ? r.hiM : (ny < 3 ? ny : 3);
    if (r.y1 == ny) r.loM = r.loM < ny - 3 ? r.loM : ny - 3;
    r.loU = (r.loM == 0) ? 0 : r.loM - 1;
    r.hiU = (r.hiM == ny) ? ny : r.hiM + 1;
    if (r.loM == 0) r.hiU = r.hiU > (ny < 3 ? ny : 3) ? r.hiU : (ny < 3 ? ny : 3);
    if (r.hiM == ny) r.loU = r.loU < ny - 3 ? r.loU : ny - 3;
    return r;
}

__host__ __device__ inline int capU_of(int h) { return h + 4 > 5 ? h + 4 : 5; }
__host__ __device__ inline int capM_of(int h) { return h + 2 > 3 ? h + 2 : 3; }
__host__ __device__ inline size_t al16(size_t b) { return (b + 15) / 16 * 16; }

// ---------------------------------------------------------------------------
// shared-memory layouts (host and device)
// ---------------------------------------------------------------------------
// Forward row phase of tile height h.  budget: bytes available for the workspace;
// mandatory buffers first, then (stage != 0) the inputs in order of use while they
// fit.  stage == 0 reads every input in place from global memory.
__host__ __device__ inline void fwd_layout(int nx, int h, int flags, int ncols, size_t budget, int stage,
                                           FwdLayout* L) {
    const size_t capU = capU_of(h), capM = capM_of(h), NH = nx / 2 + 1;
    size_t off = 0;
    auto take = [&](size_t bytes) -> int {
        const int o = (int)off;
        off += al16(bytes);
        return o;
    };
    L->U = take(capU * nx * 8);
    const size_t mom = 3 * capM * nx * 4, inv_fft = 2 * ((capU + 1) / 2) * nx * 8;
    L->MS = take(mom > inv_fft ? mom : inv_fft);
    L->KB = take(capU * nx * 4);
    L->KC = take(capU * nx * 4);
    L->R = take((size_t)h * nx * 4);
    L->cpart = take((size_t)ncols * 4 * 8);
    L->stage_u = stage ? 1 : 0;
    auto opt = [&](size_t bytes) -> int {
        if (!stage || off + al16(bytes) > budget) return -1;
        return take(bytes);
    };
    const size_t row = (size_t)h * nx * 4;
    L->S_in = opt(capU * NH * 8);
    L->KA = opt(capU * nx * 4);
    L->D = opt(capM * nx * 4);
    L->Ha = opt(row);
    L->Hb = opt(row);
    L->ue = opt(row);
    L->uz = opt(row);
    L->dz = opt(row);
    L->visc = opt(row);
    L->zbss = (flags & FLAG_ZBSS) ? opt(row) : -1;
    L->mask = (flags & FLAG_MASK) ? opt(row) : -1;
    L->hafref = (flags & FLAG_HAFREF) ? opt(row) : -1;
    L->sigref = (flags & FLAG_SIGREF) ? opt(row) : -1;
    L->ueref = (flags & FLAG_UEREF) ? opt(row) : -1;
    L->bytes = (int)off;
}
__host__ __device__ inline size_t ws_rows_fwd_min(int nx, int h, int ncols) {
    FwdLayout L;
    fwd_layout(nx, h, 0, ncols, 0, 0, &L);
    return (size_t)L.bytes;
}
// column phase: FFT buffers, multipliers
__host__ __device__ inline size_t ws_cols(int ny, int B) { return al16((size_t)2 * B * ny * 8) + al16((size_t)B * ny * 4); }
// last-stage inverse rows: [S rows h x NH][FFT 2 x ceil(h/2) x nx][k1 k2 k3 h x nx][up un h x nx f64][cpart]
struct InvLayout {
    int S_in, fft, k1, k2, k3, up, un, cpart, bytes;
};
__host__ __device__ inline void inv_layout(int nx, int h, int ncols, InvLayout* L) {
    const size_t NH = nx / 2 + 1;
    size_t off = 0;
    auto take = [&](size_t bytes) -> int {
        const int o = (int)off;
        off += al16(bytes);
        return o;
    };
    L->S_in = take((size_t)h * NH * 8);
    L->fft = take((size_t)2 * ((h + 1) / 2) * nx * 8);
    L->k1 = take((size_t)h * nx * 4);
    L->k2 = take((size_t)h * nx * 4);
    L->k3 = take((size_t)h * nx * 4);
    L->up = take((size_t)h * nx * 8);
    L->un = take((size_t)h * nx * 8);
    L->cpart = take((size_t)ncols * 4 * 8);
    L->bytes = (int)off;
}
__host__ __device__ inline size_t ws_rows_inv(int nx, int h, int ncols) {
    InvLayout L;
    inv_layout(nx, h, ncols, &L);
    return (size_t)L.bytes;
}
__host__ __device__ inline size_t ws_conv_rows(int Mx, int h) { return al16((size_t)2 * 2 * ((h + 1) / 2) * Mx * 8); }
__host__ __device__ inline size_t ws_conv_cols(int My, int B) { return al16((size_t)2 * 2 * B * My * 8); }

// ---------------------------------------------------------------------------
// asynchronous global -> shared copies (cp.async; 16-byte pieces where both sides
// are aligned).  Every thread waits for its own copies with cpa_wait(); a
// __syncthreads() after it publishes them to the block.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cpa4(void* s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa8(void* s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa16(void* s, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// bytes: a multiple of 4; dst and src 4-byte aligned
__device__ __forceinline__ void cpa_bytes(void* dst, const void* src, int bytes) {
    unsigned char* d = (unsigned char*)dst;
    const unsigned char* g = (const unsigned char*)src;
    const int tid = threadIdx.x, nth = blockDim.x;
    if ((((uintptr_t)d ^ (uintptr_t)g) & 15) == 0) {
        const int head = (int)((16 - ((uintptr_t)d & 15)) & 15) < bytes ? (int)((16 - ((uintptr_t)d & 15)) & 15) : bytes;
        const int nb16 = (bytes - head) / 16;
        const int tail0 = head + nb16 * 16;
        for (int i = tid; i < head / 4; i += nth) cpa4(d + 4 * i, g + 4 * i);
        for (int i = tid; i < nb16; i += nth) cpa16(d + head + 16 * i, g + head + 16 * i);
        for (int i = tid; i < (bytes - tail0) / 4; i += nth) cpa4(d + tail0 + 4 * i, g + tail0 + 4 * i);
    } else if ((((uintptr_t)d ^ (uintptr_t)g) & 7) == 0) {
        const int head = ((uintptr_t)d & 7) ? 4 : 0;
        const int head_n = head < bytes ? head : bytes;
        const int nb8 = (bytes - head_n) / 8;
        const int tail0 = head_n + nb8 * 8;
        for (int i = tid; i < head_n / 4; i += nth) cpa4(d + 4 * i, g + 4 * i);
        for (int i = tid; i < nb8; i += nth) cpa8(d + head_n + 8 * i, g + head_n + 8 * i);
        for (int i = tid; i < (bytes - tail0) / 4; i += nth) cpa4(d + tail0 + 4 * i, g + tail0 + 4 * i);
    } else {
        for (int i = tid; i < bytes / 4; i += nth) cpa4(d + 4 * i, g + 4 * i);
    }
}

// the same, called out of line: the optional input staging of the forward row phase,
// kept out of the phase's instruction stream (with inputs read in place it never runs,
// and its inlined copy loops would only spread the executed code over more cache lines)
static __device__ __noinline__ void cpa_bytes_ool(void* dst, const void* src, int bytes) { cpa_bytes(dst, src, bytes); }

// cooperative copy of a struct (8-byte words) by all threads of the block
__device__ __forceinline__ void copy_words(void* dst, const void* src, int bytes) {
    const unsigned long long* s = (const unsigned long long*)src;
    unsigned long long* d = (unsigned long long*)dst;
    for (int i = threadIdx.x; i < bytes / 8; i += blockDim.x) d[i] = s[i];
}

// rows [r0, r1) of an nx-wide array of T into smem buffer at offset off (if off >= 0);
// returns the row-r0-based view (smem, or global in place)
template <typename T>
__device__ __forceinline__ const T* stage_rows(unsigned char* ws, int off, const T* g, int r0, int r1, int nx) {
    const T* src = g + (size_t)r0 * nx;
    if (off < 0 || !g) return src;
    T* dst = (T*)(ws + off);
    cpa_bytes_ool(dst, src, (r1 - r0) * nx * (int)sizeof(T));
    return dst;
}

// ---------------------------------------------------------------------------
// corner values of a dudt field from the column tasks' partials
// ---------------------------------------------------------------------------
__device__ __forceinline__ double cmean(const double* c, double border) {
    return 0.25 * (c[0] + c[1] + c[2] + c[3]) - border;
}

__device__ __forceinline__ int corner_index(int q, int nx, int ny) {
    return q == 0 ? 0 : q == 1 ? nx - 1 : q == 2 ? (ny - 1) * nx : (ny - 1) * nx + nx - 1;
}

// warps 0..3 sum partial q over the tasks (lane-strided, then a butterfly); out4 in
// shared memory; the caller synchronises before reading it.
__device__ __forceinline__ void corners_from_partials(const double* cp, int ncols, double* out4) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w < 4) {
        double acc = 0.0;
        for (int t = lane; t < ncols; t += 32) acc += cp[4 * t + w];
        acc = warp_sum(acc);
        if (lane == 0) out4[w] = acc;
    }
}

// the same sum read straight from the global partials (L2: other blocks wrote them
// before the last grid barrier), in the same order, so the result is identical
__device__ __forceinline__ void corners_from_partials_g(const double* cp, int ncols, double* out4) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w < 4) {
        double acc = 0.0;
        for (int t = lane; t < ncols; t += 32) acc += __ldcg(cp + 4 * t + w);
        acc = warp_sum(acc);
        if (lane == 0) out4[w] = acc;
    }
}

// this column task's share of corner value qc (0: (0,0), 1: (nx-1,0), 2: (0,ny-1),
// 3: (nx-1,ny-1)): terms kx0..kx0+nb-1 of the inverse real DFT of row 0 or ny-1
// (q: the task's columns, y fastest)
__device__ __forceinline__ double column_corner_term(const float2* q, int ny, int nx, int kx0, int nb,
                                                     const float2* twx, int qc) {
    const int y = qc < 2 ? 0 : ny - 1;
    const bool right = qc & 1;
    double v = 0.0;
    for (int b = 0; b < nb; b++) {
        const int kx = kx0 + b;
        const float2 a = q[b * ny + y];
        if (kx == 0) {
            v += (double)a.x;
        } else if ((nx % 2 == 0) && kx == nx / 2) {
            v += right ? -(double)a.x : (double)a.x;
        } else if (!right) {
            v += 2.0 * (double)a.x;
        } else {
            const double wr = (double)twx[kx].x, wi = (double)twx[kx].y;
            v += 2.0 * ((double)a.x * wr - (double)a.y * wi);
        }
    }
    return v;
}

// ---------------------------------------------------------------------------
// scalars of a forward row phase
// ---------------------------------------------------------------------------
struct FwdScalars {
    double a1, a2, a3, c1, c2, c3, off;  // stage combination and the stage vector's corner offset
    double cue, cuz, cdz;                // corner offsets of ue (current, for z_b) and of dz
    double w;                            // ice interpolation weight
    double dzbsl, zbsl;                  // z_bsl - ReferenceBSL z, and z_bsl
    int gated;                           // this call ran the sparse update
    int pad_g;
    const double* uprev;
    double* unew;                        // where the boundary-corrected stage vector goes (or null)
    int ice_i, iue, iuz, ik;
    int stage;
    int status;
};

// stage 0: uin at t_call; 1: the state at t_call; 2-4: BS3 stages.  tice: ice times
// (shared or global).  Everything except the corner offsets.
__device__ inline void fwd_static(const Member& m, const Ctl& c, int stage, const double* uin, const double* tice,
                                  FwdScalars& s) {
    const double t = c.t, dt = c.dt;
    double a1 = 0, a2 = 0, a3 = 0, tr = 0;
    if (stage <= 1) tr = c.t_call;
    else if (stage == 2) { tr = t + C2 * dt; a1 = dt * A21; }
    else if (stage == 3) { tr = t + C3 * dt; a2 = dt * A32; }
    else { tr = t + dt; a1 = dt * A41; a2 = dt * A42; a3 = dt * A43; }
    s.a1 = a1; s.a2 = a2; s.a3 = a3;
    s.cue = cmean(c.ue_corner[c.iue], m.border_e);
    s.cuz = cmean(c.ue_corner[c.iue_zb], m.border_e);
    s.cdz = cmean(c.dz_corner, m.border_g);
    s.iue = c.iue;
    s.iuz = c.iue_zb;
    s.dzbsl = c.z_bsl - m.bsl_ref_z;
    s.zbsl = c.z_bsl;
    s.gated = c.gate;
    s.stage = stage;
    s.ik = c.ik;
    s.uprev = (stage == 0) ? uin : m.u[c.ibuf];
    s.unew = (stage == 4 || stage <= 1) ? m.u[c.ibuf ^ 1] : nullptr;
    s.status = FI_OK;
    int ii = 0;
    double w = 0.0;
    if (!m.ice_external) s.status = ice_lookup(tice, m.K, m.ice_flat, tr, &ii, &w);
    s.ice_i = ii;
    s.w = w;
}

// corner offsets from the k corners of the control block and uc, the four corner
// values of the vector the stage starts from
__device__ inline void fwd_offsets(const Member& m, const Ctl& c, const double* uc, FwdScalars& s) {
    const double* kc1 = c.kcorner[c.ik];
    const double* kc2 = c.kcorner[2];
    const double* kc3 = c.kcorner[3];
    const double c1 = cmean(kc1, m.border_v), c2 = cmean(kc2, m.border_v), c3 = cmean(kc3, m.border_v);
    double us = 0.0;
    for (int q = 0; q < 4; q++) {
        double v = uc[q];
        if (s.a1 != 0.0) v += s.a1 * (kc1[q] - c1);
        if (s.a2 != 0.0) v += s.a2 * (kc2[q] - c2);
        if (s.a3 != 0.0) v += s.a3 * (kc3[q] - c3);
        us += 0.25 * v;
    }
    s.c1 = c1; s.c2 = c2; s.c3 = c3;
    s.off = us - m.border_v;
}

// ---------------------------------------------------------------------------
// forward rows
// ---------------------------------------------------------------------------
// Views of one forward row tile: row-based pointers into shared memory or global.
struct FwdViews {
    const float2* S;
    const float *k1, *k2g, *D, *Ha, *Hb, *ue, *uz, *dz, *visc, *zbss, *mask, *hafref, *sigref, *ueref;
};

// Issues the tile's asynchronous copies; s (shared) holds the stage's scalars; thread 0
// publishes the views to vsh.  No local copies: every value comes from shared memory.
__device__ inline void fwd_prefetch(const Member& m, const FwdScalars& s, unsigned char* ws, const RowRanges& rr,
                                    int inv_prev, const float2* Sprev, FwdViews* vsh) {
    const FwdLayout& L = m.fl;
    const int nx = m.nx, stage = s.stage;
    const bool t0 = threadIdx.x == 0;
    if (L.stage_u) cpa_bytes_ool(ws + L.U, s.uprev + (size_t)rr.loU * nx, (rr.hiU - rr.loU) * nx * 8);
    if (inv_prev && L.S_in >= 0) {
        // spectrum rows have pitch sp; copy the NH used entries of each row
        for (int r = rr.loU; r < rr.hiU; r++)
            cpa_bytes_ool(ws + L.S_in + (size_t)(r - rr.loU) * m.NH * 8, Sprev + (size_t)r * m.sp, m.NH * 8);
        if (t0) vsh->S = (const float2*)(ws + L.S_in);
    } else if (t0) {
        vsh->S = nullptr;
    }
    const float* p;
    p = (stage == 2 || stage == 4) ? stage_rows(ws, L.KA, (const float*)m.k14[s.ik], rr.loU, rr.hiU, nx) : nullptr;
    if (t0) vsh->k1 = p;
    p = (stage == 4) ? stage_rows(ws, L.stage_u ? L.KB : -1, (const float*)m.k2, rr.loU, rr.hiU, nx) : nullptr;
    if (t0) vsh->k2g = p;
    p = stage_rows(ws, L.D, m.D, rr.loM, rr.hiM, nx);
    if (t0) vsh->D = p;
    const float* pue = stage_rows(ws, L.ue, (const float*)m.ue[s.iue], rr.y0, rr.y1, nx);
    if (t0) vsh->ue = pue;
    p = (s.iuz == s.iue) ? pue : stage_rows(ws, L.uz, (const float*)m.ue[s.iuz], rr.y0, rr.y1, nx);
    if (t0) vsh->uz = p;
    p = stage_rows(ws, L.dz, (const float*)m.dz, rr.y0, rr.y1, nx);
    if (t0) vsh->dz = p;
    p = stage_rows(ws, L.visc, m.visc_fac, rr.y0, rr.y1, nx);
    if (t0) vsh->visc = p;
    const int fl = m.flags;
    p = (fl & FLAG_ZBSS) ? stage_rows(ws, L.zbss, m.zbss_ref, rr.y0, rr.y1, nx) : nullptr;
    if (t0) vsh->zbss = p;
    p = (fl & FLAG_MASK) ? stage_rows(ws, L.mask, m.mask, rr.y0, rr.y1, nx) : nullptr;
    if (t0) vsh->mask = p;
    p = (fl & FLAG_HAFREF) ? stage_rows(ws, L.hafref, m.H_af_ref, rr.y0, rr.y1, nx) : nullptr;
    if (t0) vsh->hafref = p;
    p = (fl & FLAG_SIGREF) ? stage_rows(ws, L.sigref, m.sigma_ref, rr.y0, rr.y1, nx) : nullptr;
    if (t0) vsh->sigref = p;
    p = (fl & FLAG_UEREF) ? stage_rows(ws, L.ueref, m.ue_ref, rr.y0, rr.y1, nx) : nullptr;
    if (t0) vsh->ueref = p;
    const float* Ha = m.ice_external ? m.H_ext : m.H_tab + (size_t)s.ice_i * nx * m.ny;
    const float* pha = stage_rows(ws, L.Ha, Ha, rr.y0, rr.y1, nx);
    if (t0) vsh->Ha = pha;
    p = (s.w != 0.0) ? stage_rows(ws, L.Hb, Ha + (size_t)nx * m.ny, rr.y0, rr.y1, nx) : pha;
    if (t0) vsh->Hb = p;
}

// Sout: the spectrum this stage writes.  inv_prev (stages 3, 4): v.S / Sprev hold the
// previous stage's spectrum after the column pass; its rows [loU, hiU) are inverted
// here (halo recomputed), its own rows stored to kdst (k2 or k3) and used for the
// stage vector.  The prefetched copies have landed and s is final.
// WIDE (the one-block-per-SM build, whose register budget allows it): each thread issues
// the loads of several of its elements before the first use, so a sub-step pays one
// memory round trip per group instead of one per element; the elements and their
// arithmetic are the same, so the results are identical.
template <int SX = 0, int WIDE = 0>
__device__ inline void ph_rows_fwd(const Member& m, const FwdScalars& s, const FwdViews& v, const FftPlan& plan,
                                   unsigned char* ws, const RowRanges& rr, int h, float2* Sout, int inv_prev,
                                   const float2* Sprev, float* kdst) {
    const FwdLayout& L = m.fl;
    const int nx = m.nx, ny = m.ny, NH = m.NH, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int capM = capM_of(h);
    double* sU = (double*)(ws + L.U);
    float* sMxx = (float*)(ws + L.MS);
    float* sMyy = sMxx + capM * nx;
    float* sMxy = sMyy + capM * nx;
    float* sR = (float*)(ws + L.R);
    float* sKinv = (float*)(ws + (s.stage == 3 ? L.KB : L.KC));
    if (inv_prev) {
        // inverse real row transform of the previous stage, rows [loU, hiU), two rows
        // per complex FFT; the FFT scratch aliases the moment buffers
        float2* zb = (float2*)(ws + L.MS);
        const int lo = rr.loU, hi = rr.hiU, npi = (hi - lo + 1) / 2;
        const float2* Sv = v.S ? v.S : Sprev + (size_t)lo * m.sp;
        const int pitch = v.S ? NH : m.sp;
        for (int p = ty; p < npi; p += TY) {
            const bool hasb = lo + 2 * p + 1 < hi;
            const float2* Sa = Sv + (2 * p) * pitch;
            const float2* Sb = Sv + (2 * p + 1) * pitch;
            float2* zr = zb + p * nx;
            for (int k = tx; k < nx; k += TX) {
                const int kk = (k < NH) ? k : nx - k;
                const float2 A = Sa[kk];
                const float2 Bv = hasb ? Sb[kk] : make_float2(0.0f, 0.0f);
                zr[k] = (k < NH) ? make_float2(A.x - Bv.y, A.y + Bv.x) : make_float2(A.x + Bv.y, -A.y + Bv.x);
            }
        }
        __syncthreads();
        const float2* res = fft_run<true, float, SX>(zb, zb + npi * nx, plan, npi, nx);
        for (int rl = ty; rl < hi - lo; rl += TY) {
            const float2* rz = res + (rl >> 1) * nx;
            const int q = rl & 1;
            float* d = sKinv + rl * nx;
            const int r = lo + rl;
            const bool own = r >= rr.y0 && r < rr.y1;
            for (int x = tx; x < nx; x += TX) {
                const float val = q ? rz[x].y : rz[x].x;
                d[x] = val;
                if (own) kdst[r * nx + x] = val;
            }
        }
        __syncthreads();
    }
    // 1: stage vector rows [loU, hiU) in FP64 (in place over the prefetched uprev), corner BC
    {
        const float* k1 = v.k1;
        const float* k2 = (s.stage == 3) ? sKinv : v.k2g;
        const float* k3 = sKinv;
        const double a1 = s.a1, a2 = s.a2, a3 = s.a3, c1 = s.c1, c2 = s.c2, c3 = s.c3, off = s.off;
        const int nU = (rr.hiU - rr.loU) * nx;
        const double* ub = L.stage_u ? sU : s.uprev + (size_t)rr.loU * nx;
        // ub may alias sU: every element is read before it is written
        constexpr int BQ = WIDE ? 4 : 1;
        for (int i0 = tid; i0 < nU; i0 += BQ * RT) {
            double ur[BQ];
            float q1[BQ], q2[BQ], q3[BQ];
#pragma unroll
            for (int q = 0; q < BQ; q++) {
                const int i = i0 + q * RT;
                if (i < nU) {
                    ur[q] = ub[i];
                    q1[q] = a1 != 0.0 ? k1[i] : 0.0f;
                    q2[q] = a2 != 0.0 ? k2[i] : 0.0f;
                    q3[q] = a3 != 0.0 ? k3[i] : 0.0f;
                }
            }
#pragma unroll
            for (int q = 0; q < BQ; q++) {
                const int i = i0 + q * RT;
                if (i < nU) {
                    double u = ur[q];
                    if (a1 != 0.0) u += a1 * ((double)q1[q] - c1);
                    if (a2 != 0.0) u += a2 * ((double)q2[q] - c2);
                    if (a3 != 0.0) u += a3 * ((double)q3[q] - c3);
                    sU[i] = u - off;
                }
            }
        }
    }
    __syncthreads();
    // 2a: bending moments on rows [loM, hiM) (u-derivatives in FP64)
    {
        const double dx = m.dx, dy = m.dy, nu = m.nu;
        const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy), i2dx = 1.0 / (2 * dx), idx = 1.0 / dx;
        const double i2dy = 1.0 / (2 * dy), idy = 1.0 / dy;
        for (int r = rr.loM + ty; r < rr.hiM; r += TY) {
            const double* Ur = sU + (r - rr.loU) * nx;
            const int rc = min(max(r, 1), ny - 2);
            const double* U0 = sU + (rc - rr.loU) * nx;
            const double* Ua;
            const double* Ub;
            double sy;
            if (r == 0) { Ua = sU + (1 - rr.loU) * nx; Ub = sU + (0 - rr.loU) * nx; sy = idy; }
            else if (r == ny - 1) { Ua = sU + (ny - 1 - rr.loU) * nx; Ub = sU + (ny - 2 - rr.loU) * nx; sy = idy; }
            else { Ua = Ur + nx; Ub = Ur - nx; sy = i2dy; }
            const int mo = (r - rr.loM) * nx;
            const float* Dr = v.D + (r - rr.loM) * nx;
            constexpr int BX = WIDE ? 3 : 1;
            for (int x0 = tx; x0 < nx; x0 += BX * TX) {
            float Dq[BX];
#pragma unroll
            for (int q = 0; q < BX; q++)
                if (x0 + q * TX < nx) Dq[q] = Dr[x0 + q * TX];
#pragma unroll
            for (int q = 0; q < BX; q++) {
                const int x = x0 + q * TX;
                if (x >= nx) continue;
                const int xc = min(max(x, 1), nx - 2);
                const double uxx = (Ur[xc + 1] - 2.0 * Ur[xc] + Ur[xc - 1]) * idx2;
                const double uyy = (U0[nx + x] - 2.0 * U0[x] + U0[x - nx]) * idy2;
                double da, db;
                if (x == 0) { da = (Ua[1] - Ua[0]) * idx; db = (Ub[1] - Ub[0]) * idx; }
                else if (x == nx - 1) { da = (Ua[nx - 1] - Ua[nx - 2]) * idx; db = (Ub[nx - 1] - Ub[nx - 2]) * idx; }
                else { da = (Ua[x + 1] - Ua[x - 1]) * i2dx; db = (Ub[x + 1] - Ub[x - 1]) * i2dx; }
                const double uxy = (da - db) * sy;
                const double D = (double)Dq[q];
                sMxx[mo + x] = (float)(-D * (nu * uyy + uxx));
                sMyy[mo + x] = (float)(-D * (nu * uxx + uyy));
                sMxy[mo + x] = (float)(-D * (1.0 - nu) * uxy);
            }
            }
        }
    }
    // 2b: column anomalies on the own rows; -g sigma_full to sR
    {
        const double cue = s.cue, cuz = s.cuz, cdz = s.cdz;
        const float fw = (float)s.w;
        double* unew = s.unew;
        const int flags = m.flags;
        const int n_own = (rr.y1 - rr.y0) * nx;
        const double* Uown = sU + (rr.y0 - rr.loU) * nx;
        constexpr int BI = WIDE ? 3 : 1;
        for (int i0 = tid; i0 < n_own; i0 += BI * RT) {
        float qa[BI], qb[BI], qe[BI], qz[BI], qd[BI];
#pragma unroll
        for (int q = 0; q < BI; q++) {
            const int i = i0 + q * RT;
            if (i < n_own) {
                qa[q] = v.Ha[i];
                qb[q] = fw != 0.0f ? v.Hb[i] : 0.0f;
                qe[q] = v.ue[i];
                qz[q] = v.uz[i];
                qd[q] = v.dz[i];
            }
        }
#pragma unroll
        for (int q = 0; q < BI; q++) {
            const int i = i0 + q * RT;
            if (i >= n_own) continue;
            const int g = rr.y0 * nx + i;
            const double u = Uown[i];
            const float ha = qa[q];
            const double H = (double)(fw != 0.0f ? ha + (qb[q] - ha) * fw : ha);
            const double uev = (double)qe[q] - cue;
            const double dzv = (double)qd[q] - cdz;
            const double zdiff = (double)((flags & FLAG_ZBSS) ? v.zbss[i] : m.zbss_scalar) +
                                 ((double)qz[q] - cuz) + u - dzv - s.dzbsl;
            double haf = H + (zdiff < 0.0 ? zdiff : 0.0) * m.rho_sw_ice;
            haf = haf > 0.0 ? haf : 0.0;
            const double mk = (flags & FLAG_MASK) ? (double)v.mask[i] : 1.0;
            const double hafref = (flags & FLAG_HAFREF) ? (double)v.hafref[i] : 0.0;
            double ssw = 0.0;
            if (s.gated) {
                // update_maskgrounded!, update_maskocean!, watercolumn!, columnanom_water!
                // (src/topography.jl:1-28, src/loads.jl:56-85) after the sparse update
                const bool gr = haf > 0.0;
                const double w = -zdiff;  // z_ss - z_b
                const bool oc = w > 0.0 && !gr;
                const double wc = w > 0.0 ? w : 0.0;
                const double hw = (H <= 1.0 ? wc : 0.0) + ((!gr && H > 1.0) ? wc - H / m.rho_sw_ice : 0.0);
                if (m.sl_interactive && oc) ssw = m.rho_sw * (dzv + s.zbsl) * mk;
                m.sw[g] = (float)ssw;
                m.mgr[g] = gr ? 1.0f : 0.0f;
                m.moc[g] = oc ? 1.0f : 0.0f;
                m.hwater[g] = (float)hw;
            } else if (m.sl_interactive) {
                ssw = (double)m.sw[g];
            }
            const double sload = mk * (m.rho_ice * (haf - hafref) + ssw);
            double sfull = mk * (m.rho_ice * haf + m.rho_litho * uev + m.rho_um * u + ssw);
            if (flags & FLAG_SIGREF) sfull -= (double)v.sigref[i];
            m.sig_load[g] = (float)sload;
            double geo = sfull;
            if (m.column_compressible) {
                // A (sigma_load + m sigma_mantle) = A (sigma_full - m sigma_litho), sealevel.jl:193-197
                const double uer = (flags & FLAG_UEREF) ? (double)v.ueref[i] : 0.0;
                geo = sfull - mk * m.rho_litho * (uev - uer);
            }
            m.sig_geo[g] = (float)(m.A * geo);
            sR[i] = (float)(-m.g * sfull);
            if (unew) unew[g] = u;
        }
        }
    }
    __syncthreads();
    // 3: moment divergence in FP32 -> f = rhs * K/(2 eta), rows packed in pairs
    float2* zb = (float2*)(ws + L.U);  // aliases the stage vector (dead now)
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
            const float* Mx = sMxx + (rv - rr.loM) * nx;
            const int rc = min(max(rv, 1), ny - 2);
            const float* My0 = sMyy + (rc - rr.loM) * nx;
            const float* Ma;
            const float* Mb;
            float sy;
            if (rv == 0) { Ma = sMxy + (1 - rr.loM) * nx; Mb = sMxy + (0 - rr.loM) * nx; sy = idy; }
            else if (rv == ny - 1) { Ma = sMxy + (ny - 1 - rr.loM) * nx; Mb = sMxy + (ny - 2 - rr.loM) * nx; sy = idy; }
            else { Ma = sMxy + (rv + 1 - rr.loM) * nx; Mb = sMxy + (rv - 1 - rr.loM) * nx; sy = i2dy; }
            float* zrow = (float*)(zb + p * nx) + q;
            const float* vf = v.visc + (rv - rr.y0) * nx;
            const float* sr = sR + (rv - rr.y0) * nx;
            constexpr int BV = WIDE ? 3 : 1;
            for (int x0 = tx; x0 < nx; x0 += BV * TX) {
            float vq[BV];
#pragma unroll
            for (int k = 0; k < BV; k++)
                vq[k] = (valid && x0 + k * TX < nx) ? vf[x0 + k * TX] : 0.0f;
#pragma unroll
            for (int k = 0; k < BV; k++) {
                const int x = x0 + k * TX;
                if (x >= nx) continue;
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
                    f = rhs * vq[k];
                }
                zrow[2 * x] = f;
            }
            }
        }
    }
    __syncthreads();
    float2* res = fft_run<false, float, SX>(zb, zb + np * nx, plan, np, nx);
    // split the pair spectra, store the half-spectrum rows
    for (int p = ty; p < np; p += TY) {
        const int ra = rr.y0 + 2 * p;
        const bool hb = ra + 1 < rr.y1;
        float2* Sa = Sout + (size_t)ra * m.sp;
        float2* Sb = Sout + (size_t)(ra + 1) * m.sp;
        const float2* rz = res + p * nx;
        for (int kx = tx; kx < NH; kx += TX) {
            const float2 Z = rz[kx];
            const float2 Zc = rz[kx == 0 ? 0 : nx - kx];
            Sa[kx] = make_float2(0.5f * (Z.x + Zc.x), 0.5f * (Z.y - Zc.y));
            if (hb) Sb[kx] = make_float2(0.5f * (Z.y + Zc.y), -0.5f * (Z.x - Zc.x));
        }
    }
    __syncthreads();  // the workspace is reused by the caller's next phase
}

// ---------------------------------------------------------------------------
// columns (in place on S); cpart_out: this task's 4 corner terms
// ---------------------------------------------------------------------------
template <int SY = 0>
__device__ inline void ph_cols(const Member& m, const FftPlan& plan, const float2* twx, unsigned char* ws, int tile,
                               int B, float2* S, double* cpart_out) {
    const int ny = m.ny, tid = threadIdx.x, nth = blockDim.x;
    const int kx0 = tile * B;
    const int nb = min(B, m.NH - kx0);
    float2* b0 = (float2*)ws;
    float2* b1 = b0 + B * ny;
    float* mu = (float*)(ws + al16((size_t)2 * B * ny * 8));
    // gather the columns and their multipliers asynchronously
    for (int i = tid; i < nb * ny; i += nth) {
        const int b = i / ny, y = i - b * ny;
        cpa8(b0 + i, S + (size_t)y * m.sp + kx0 + b);
    }
    cpa_bytes(mu, m.mult + (size_t)kx0 * ny, nb * ny * 4);
    cpa_wait();
    __syncthreads();
    float2* r = fft_run<false, float, SY>(b0, b1, plan, nb, ny);
    float2* o = (r == b0) ? b1 : b0;
    for (int i = tid; i < nb * ny; i += nth) {
        const float sc = mu[i];
        const float2 v = r[i];
        r[i] = make_float2(v.x * sc, v.y * sc);
    }
    __syncthreads();
    float2* q = fft_run<true, float, SY>(r, o, plan, nb, ny);
    for (int i = tid; i < nb * ny; i += nth) {
        const int b = i / ny, y = i - b * ny;
        S[(size_t)y * m.sp + kx0 + b] = q[i];
    }
    if (tid < 4) cpart_out[tid] = column_corner_term(q, ny, m.nx, kx0, nb, twx, tid);
    __syncthreads();
}

// ---------------------------------------------------------------------------
// inverse rows
// ---------------------------------------------------------------------------
// BS3 embedded-error inputs of the last stage
struct ErrTerms {
    double dt, abstol, reltol, cc1, cc2, cc3;
    const double* up;
    const double* un;
    const float* k1;
};

// Issues the copies of an inverse row tile (spectrum rows and, with e, the error-norm
// inputs); the caller copies the corner partials to the layout's cpart slot.
__device__ inline void inv_prefetch(const Member& m, const float2* S, unsigned char* ws, int tile, int h,
                                    const ErrTerms* e) {
    InvLayout L;
    inv_layout(m.nx, h, m.ncols, &L);
    const int nx = m.nx, ny = m.ny, NH = m.NH;
    const int y0 = tile * h, y1 = min(y0 + h, ny);
    for (int r = y0; r < y1; r++) cpa_bytes(ws + L.S_in + (size_t)(r - y0) * NH * 8, S + (size_t)r * m.sp, NH * 8);
    if (e) {
        const size_t g0 = (size_t)y0 * nx;
        const int n = (y1 - y0) * nx;
        cpa_bytes(ws + L.k1, e->k1 + g0, n * 4);
        cpa_bytes(ws + L.k2, m.k2 + g0, n * 4);
        cpa_bytes(ws + L.k3, m.k3 + g0, n * 4);
        cpa_bytes(ws + L.up, e->up + g0, n * 8);
        cpa_bytes(ws + L.un, e->un + g0, n * 8);
    }
}

// Inverse rows of S (prefetched) into dst; corners4 (shared): the field's corner
// values.  Returns (in every thread) the block's sum of squared scaled errors when
// e != null.
template <int SX = 0>
__device__ inline double ph_rows_inv(const Member& m, const FftPlan& plan, unsigned char* ws, double* red, int tile,
                                     int h, float* dst, const ErrTerms* e, const double* corners4) {
    InvLayout L;
    inv_layout(m.nx, h, m.ncols, &L);
    const int nx = m.nx, ny = m.ny, NH = m.NH, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int y0 = tile * h, y1 = min(y0 + h, ny);
    const int np = (y1 - y0 + 1) / 2;
    const float2* Sv = (const float2*)(ws + L.S_in);
    float2* zb = (float2*)(ws + L.fft);
    for (int p = ty; p < np; p += TY) {
        const bool hasb = y0 + 2 * p + 1 < y1;
        const float2* Sa = Sv + (2 * p) * NH;
        const float2* Sb = Sv + (2 * p + 1) * NH;
        float2* zr = zb + p * nx;
        for (int k = tx; k < nx; k += TX) {
            const int kk = (k < NH) ? k : nx - k;
            const float2 A = Sa[kk];
            const float2 Bv = hasb ? Sb[kk] : make_float2(0.0f, 0.0f);
            zr[k] = (k < NH) ? make_float2(A.x - Bv.y, A.y + Bv.x) : make_float2(A.x + Bv.y, -A.y + Bv.x);
        }
    }
    __syncthreads();
    const float2* res = fft_run<true, float, SX>(zb, zb + np * nx, plan, np, nx);
    const double cs = cmean(corners4, m.border_v);
    const int n = (y1 - y0) * nx;
    const float* k1 = (const float*)(ws + L.k1);
    const float* k2 = (const float*)(ws + L.k2);
    const float* k3 = (const float*)(ws + L.k3);
    const double* up = (const double*)(ws + L.up);
    const double* un = (const double*)(ws + L.un);
    double acc = 0.0;
    for (int i = tid; i < n; i += RT) {
        const int rl = i / nx, x = i - rl * nx;
        const float2 z = res[(rl >> 1) * nx + x];
        const float v = (rl & 1) ? z.y : z.x;
        dst[y0 * nx + i] = v;
        if (e) {
            const double ut = e->dt * (BT1 * ((double)k1[i] - e->cc1) + BT2 * ((double)k2[i] - e->cc2) +
                                       BT3 * ((double)k3[i] - e->cc3) + BT4 * ((double)v - cs));
            const double a = fabs(up[i]), b = fabs(un[i]);
            const double sc = ut / (e->abstol + (a > b ? a : b) * e->reltol);
            acc += sc * sc;
        }
    }
    double sum = 0.0;
    if (e) {
        double vv[1] = {acc};
        block_sum<1>(vv, red);
        sum = vv[0];
    }
    __syncthreads();
    return sum;
}

// Sum of the error-norm partials in a fixed order (lane-strided, then a butterfly) by
// one warp; every lane returns the total.
__device__ __forceinline__ double partials_sum(const double* part, int n) {
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    int i = lane;
    for (; i + 96 < n; i += 128) {
        const double a = __ldcg(part + i), b = __ldcg(part + i + 32), c = __ldcg(part + i + 64),
                     d = __ldcg(part + i + 96);
        acc += a;
        acc += b;
        acc += c;
        acc += d;
    }
    for (; i < n; i += 32) acc += __ldcg(part + i);
    return warp_sum(acc);
}

// ---------------------------------------------------------------------------
// sparse update: padded linear convolutions (elastic = channel A, sea surface = B).
// Row pairs of the same channel share one complex FFT: packing the two channels
// together would mix their FP32 rounding (their inputs differ by the cell area, ~1e9).
// ---------------------------------------------------------------------------
__device__ inline void ph_conv_rows(const Member& m, const FftPlan& plan, unsigned char* ws, int tile, int h) {
    const int nx = m.nx, ny = m.ny, Mx = m.Mx, MH = m.MH, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int y0 = tile * h, y1 = min(y0 + h, ny);
    const int np = (y1 - y0 + 1) / 2;
    const int nch = m.elastic_on + m.geoid_on;
    if (nch == 0) return;
    const float* in[2];
    float2* out[2];
    int cc = 0;
    if (m.elastic_on) { in[cc] = m.sig_load; out[cc] = m.SA; cc++; }  // * K^2, K == 1
    if (m.geoid_on) { in[cc] = m.sig_geo; out[cc] = m.SB; cc++; }
    const int nt = nch * np;
    float2* zb = (float2*)ws;
    for (int tr = ty; tr < nt; tr += TY) {
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        const bool hb = ra + 1 < y1;
        const float* ia = in[ch] + ra * nx;
        const float* ib = in[ch] + (ra + 1) * nx;
        float2* zr = zb + tr * Mx;
        for (int x = tx; x < Mx; x += TX)
            zr[x] = (x < nx) ? make_float2(ia[x], hb ? ib[x] : 0.0f) : make_float2(0.0f, 0.0f);
    }
    __syncthreads();
    float2* res = fft_batch<false, float>(zb, zb + nt * Mx, plan, nt, Mx);
    for (int tr = ty; tr < nt; tr += TY) {
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        const bool hb = ra + 1 < y1;
        float2* oa = out[ch] + (size_t)ra * m.msp;
        float2* ob = out[ch] + (size_t)(ra + 1) * m.msp;
        const float2* rz = res + tr * Mx;
        for (int kx = tx; kx < MH; kx += TX) {
            const float2 Z = rz[kx];
            const float2 Zc = rz[kx == 0 ? 0 : Mx - kx];
            oa[kx] = make_float2(0.5f * (Z.x + Zc.x), 0.5f * (Z.y - Zc.y));
            if (hb) ob[kx] = make_float2(0.5f * (Z.y + Zc.y), -0.5f * (Z.x - Zc.x));
        }
    }
    __syncthreads();
}

__device__ inline void ph_conv_cols(const Member& m, const FftPlan& plan, unsigned char* ws, int tile, int B) {
    const int ny = m.ny, My = m.My, tid = threadIdx.x, nth = blockDim.x;
    const int kx0 = tile * B;
    const int nb = min(B, m.MH - kx0);
    // transform list: [channel][b][y]; channel 0 = A (elastic), 1 = B (sea surface)
    float2* b0 = (float2*)ws;
    float2* b1 = b0 + 2 * B * My;
    const int nt = 2 * nb;
    const int lanes = nb, rows_per = nth / lanes;
    const int bl = tid % lanes, r0 = tid / lanes;
    if (r0 < rows_per)
        for (int y = r0; y < My; y += rows_per) {
            const float2 za = (y < ny) ? m.SA[(size_t)y * m.msp + kx0 + bl] : make_float2(0.0f, 0.0f);
            const float2 zc = (y < ny) ? m.SB[(size_t)y * m.msp + kx0 + bl] : make_float2(0.0f, 0.0f);
            b0[bl * My + y] = za;
            b0[(nb + bl) * My + y] = zc;
        }
    __syncthreads();
    float2* r = fft_batch<false, float>(b0, b1, plan, nt, My);
    float2* o = (r == b0) ? b1 : b0;
    for (int tr = 0; tr < nt; tr++) {
        const int ch = tr / nb, b = tr - ch * nb;
        const float2* G = (ch == 0 ? m.GA : m.GB) + (size_t)(kx0 + b) * My;
        float2* rt = r + tr * My;
        for (int ky = tid; ky < My; ky += nth) rt[ky] = cmul(rt[ky], __ldg(&G[ky]));
    }
    __syncthreads();
    float2* q = fft_batch<true, float>(r, o, plan, nt, My);
    // keep the crop window rows j1..j1+ny-1 and the two corner rows 0, 2ny-2
    const int nrow = ny + 2;
    if (r0 < rows_per)
        for (int ry = r0; ry < nrow; ry += rows_per) {
            const int y = ry < ny ? m.j1 + ry : (ry == ny ? 0 : 2 * ny - 2);
            m.TA[(size_t)ry * m.msp + kx0 + bl] = q[bl * My + y];
            m.TB[(size_t)ry * m.msp + kx0 + bl] = q[(nb + bl) * My + y];
        }
    __syncthreads();
}

// Writes the new ue (buffer iue) / dz crop rows and, from the tile holding the corner
// rows, their raw corner values (ue_corner / dz_corner, each double[4]).
__device__ inline void ph_conv_rows_inv(const Member& m, const FftPlan& plan, unsigned char* ws, int tile, int h, int iue,
                                 double* ue_corner, double* dz_corner) {
    const int nx = m.nx, ny = m.ny, Mx = m.Mx, MH = m.MH, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int nrow = ny + 2;  // crop rows j1..j1+ny-1, then corner rows 0 and 2ny-2
    const int y0 = tile * h, y1 = min(y0 + h, nrow);
    const int np = (y1 - y0 + 1) / 2;
    if (!m.elastic_on) {
        // RigidLithosphere: ue = 0 (src/deformation.jl:186-189)
        for (int ry = y0 + ty; ry < min(y1, ny); ry += TY)
            for (int x = tx; x < nx; x += TX) m.ue[iue][ry * nx + x] = 0.0f;
        if (tid == 0 && y1 > ny)
            for (int q = 0; q < 4; q++) ue_corner[q] = 0.0;
    }
    const int nch = m.elastic_on + m.geoid_on;
    if (nch == 0) return;
    const float2* src[2];
    float* dst[2];
    double* corner[2];
    int cc = 0;
    if (m.elastic_on) { src[cc] = m.TA; dst[cc] = m.ue[iue]; corner[cc] = ue_corner; cc++; }
    if (m.geoid_on) { src[cc] = m.TB; dst[cc] = m.dz; corner[cc] = dz_corner; cc++; }
    const int nt = nch * np;
    float2* zb = (float2*)ws;
    for (int tr = ty; tr < nt; tr += TY) {
        const int ch = tr / np, p = tr - ch * np;
        const int ra = y0 + 2 * p;
        const bool hb = ra + 1 < y1;
        const float2* Sa = src[ch] + (size_t)ra * m.msp;
        const float2* Sb = src[ch] + (size_t)(ra + 1) * m.msp;
        float2* zr = zb + tr * Mx;
        for (int k = tx; k < Mx; k += TX) {
            const int kk = (k < MH) ? k : Mx - k;
            const float2 A = Sa[kk];
            const float2 Bv = hb ? Sb[kk] : make_float2(0.0f, 0.0f);
            zr[k] = (k < MH) ? make_float2(A.x - Bv.y, A.y + Bv.x) : make_float2(A.x + Bv.y, -A.y + Bv.x);
        }
    }
    __syncthreads();
    float2* res = fft_batch<true, float>(zb, zb + nt * Mx, plan, nt, Mx);
    for (int tr = ty; tr < nt; tr += TY) {
        const int ch = tr / np, p = tr - ch * np;
        for (int q = 0; q < 2; q++) {
            const int ry = y0 + 2 * p + q;
            if (ry >= ny || ry >= y1) continue;
            float* d = dst[ch] + ry * nx;
            const float2* z = res + tr * Mx + m.i1;
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
                const float2 za = res[tr * Mx + 0];
                const float2 zc = res[tr * Mx + 2 * nx - 2];
                corner[ch][q0] = (double)(q == 0 ? za.x : za.y);
                corner[ch][q0 + 1] = (double)(q == 0 ? zc.x : zc.y);
            }
        }
    }
    __syncthreads();
}

}  // namespace fi
