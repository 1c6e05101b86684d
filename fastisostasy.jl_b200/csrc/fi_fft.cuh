// fi_fft.cuh -- shared-memory mixed-radix FFT for sm_100a.
//
// Batched 1D complex transforms staged in shared memory: Stockham autosort
// passes (natural order in and out) with radix-2/3/4/5/7/8 butterflies held in
// registers and a generic odd-radix pass for any other prime factor.  These
// replace the FFTW/CUFFT plans of the reference (src/tools.jl:100-108,
// src/convolutions.jl:229-244).  Twiddles come from a per-length FP64 table
// (rounded to FP32 for the single-precision form), so the only rounding is in
// the butterflies themselves.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fi {

template <typename T> struct cplx_of;
template <> struct cplx_of<float> { using type = float2; };
template <> struct cplx_of<double> { using type = double2; };
template <typename T> using cplx = typename cplx_of<T>::type;

template <typename C> __device__ __forceinline__ C cmk(decltype(C::x) a, decltype(C::x) b) { C r; r.x = a; r.y = b; return r; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) { return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C> __device__ __forceinline__ C cconj(C a) { return cmk<C>(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return cmk<C>(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> __device__ __forceinline__ C mul_mi(C a) { return INV ? cmk<C>(-a.y, a.x) : cmk<C>(a.y, -a.x); }

constexpr int FFT_MAX_PASSES = 20;
constexpr int FFT_MAX_LEN = 4096;

// One transform length: radix schedule + twiddle tables tw[m] = exp(-2 pi i m / L).
// mag_nb / mag_ns: multiply-high reciprocals of L/R and of Ns for each pass
// (x / d == __umulhi(x, ceil(2^32 / d)) for x * d < 2^32; d == 1 is special-cased).
struct FftPlan {
    int L;
    int npass;
    int radix[FFT_MAX_PASSES];
    unsigned int mag_nb[FFT_MAX_PASSES];
    unsigned int mag_ns[FFT_MAX_PASSES];
    // per pass: L / R, the twiddle stride L / (Ns R) and Ns (product of the earlier
    // radices), precomputed so that no pass divides by a runtime value
    int nb[FFT_MAX_PASSES];
    int tstride[FFT_MAX_PASSES];
    int ns[FFT_MAX_PASSES];
    const float2* tw32;
    const double2* tw64;
    int seq;  // seq_code of the schedule (0: none), for kernels that dispatch on it
    int pad_seq;
};

__host__ __device__ inline unsigned int fastdiv_magic(unsigned int d) {
    return d <= 1 ? 0u : (unsigned int)((0x100000000ull + d - 1) / d);
}

__device__ __forceinline__ unsigned int fastdiv(unsigned int x, unsigned int d, unsigned int m) {
    return d == 1 ? x : __umulhi(x, m);
}

template <typename T> __device__ __forceinline__ const cplx<T>* plan_tw(const FftPlan& p);
template <> __device__ __forceinline__ const float2* plan_tw<float>(const FftPlan& p) { return p.tw32; }
template <> __device__ __forceinline__ const double2* plan_tw<double>(const FftPlan& p) { return p.tw64; }

// ---------------------------------------------------------------------------
// small DFTs in registers; forward uses exp(-2 pi i qr/R)
// ---------------------------------------------------------------------------
template <int R, bool INV, typename T> struct SmallDft;

template <bool INV, typename T> struct SmallDft<2, INV, T> {
    using C = cplx<T>;
    static __device__ __forceinline__ void run(C* v) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <bool INV, typename T> struct SmallDft<3, INV, T> {
    using C = cplx<T>;
    static __device__ __forceinline__ void run(C* v) {
        const T s = T(0.86602540378443864676372317075294);  // sin(2 pi / 3)
        C s12 = cadd(v[1], v[2]);
        C d12 = csub(v[1], v[2]);
        C y0 = cadd(v[0], s12);
        C t1 = cmk<C>(v[0].x - T(0.5) * s12.x, v[0].y - T(0.5) * s12.y);
        C t2 = mul_mi<INV>(cscale(d12, s));
        v[0] = y0;
        v[1] = cadd(t1, t2);
        v[2] = csub(t1, t2);
    }
};

template <bool INV, typename T> struct SmallDft<4, INV, T> {
    using C = cplx<T>;
    static __device__ __forceinline__ void run(C* v) {
        C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        C c = cadd(v[1], v[3]), d = mul_mi<INV>(csub(v[1], v[3]));
        v[0] = cadd(a, c);
        v[2] = csub(a, c);
        v[1] = cadd(b, d);
        v[3] = csub(b, d);
    }
};

template <bool INV, typename T> struct SmallDft<5, INV, T> {
    using C = cplx<T>;
    static __device__ __forceinline__ void run(C* v) {
        const T c1 = T(0.30901699437494742410229341718282);   // cos(2 pi/5)
        const T c2 = T(-0.80901699437494742410229341718282);  // cos(4 pi/5)
        const T s1 = T(0.95105651629515357211643933337938);   // sin(2 pi/5)
        const T s2 = T(0.58778525229247312916870595463907);   // sin(4 pi/5)
        C p14 = cadd(v[1], v[4]), m14 = csub(v[1], v[4]);
        C p23 = cadd(v[2], v[3]), m23 = csub(v[2], v[3]);
        C a1 = cmk<C>(v[0].x + c1 * p14.x + c2 * p23.x, v[0].y + c1 * p14.y + c2 * p23.y);
        C a2 = cmk<C>(v[0].x + c2 * p14.x + c1 * p23.x, v[0].y + c2 * p14.y + c1 * p23.y);
        C b1 = mul_mi<INV>(cmk<C>(s1 * m14.x + s2 * m23.x, s1 * m14.y + s2 * m23.y));
        C b2 = mul_mi<INV>(cmk<C>(s2 * m14.x - s1 * m23.x, s2 * m14.y - s1 * m23.y));
        v[0] = cadd(v[0], cadd(p14, p23));
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    }
};

template <bool INV, typename T> struct SmallDft<7, INV, T> {
    using C = cplx<T>;
    static __device__ __forceinline__ void run(C* v) {
        const T c[4] = {T(1), T(0.62348980185873353052500488400424), T(-0.22252093395631440428890256449680),
                        T(-0.90096886790241912623610231950745)};
        const T s[4] = {T(0), T(0.78183148246802980870844452667406), T(0.97492791218182360701813168299393),
                        T(0.43388373911755812047576833284836)};
        C p[4], m[4];
#pragma unroll
        for (int r = 1; r <= 3; r++) { p[r] = cadd(v[r], v[7 - r]); m[r] = csub(v[r], v[7 - r]); }
        C y[7];
        y[0] = cadd(v[0], cadd(p[1], cadd(p[2], p[3])));
#pragma unroll
        for (int q = 1; q <= 3; q++) {
            C a = v[0];
            C b = cmk<C>(T(0), T(0));
#pragma unroll
            for (int r = 1; r <= 3; r++) {
                const int qr = (q * r) % 7;
                const T cq = qr <= 3 ? c[qr] : c[7 - qr];
                const T sq = qr <= 3 ? s[qr] : -s[7 - qr];
                a = cmk<C>(a.x + cq * p[r].x, a.y + cq * p[r].y);
                b = cmk<C>(b.x + sq * m[r].x, b.y + sq * m[r].y);
            }
            C ib = mul_mi<INV>(b);
            y[q] = cadd(a, ib);
            y[7 - q] = csub(a, ib);
        }
#pragma unroll
        for (int q = 0; q < 7; q++) v[q] = y[q];
    }
};

template <bool INV, typename T> struct SmallDft<8, INV, T> {
    using C = cplx<T>;
    static __device__ __forceinline__ void run(C* v) {
        const T h = T(0.70710678118654752440084436210485);
        C a[4], b[4];
#pragma unroll
        for (int r = 0; r < 4; r++) { a[r] = cadd(v[r], v[r + 4]); b[r] = csub(v[r], v[r + 4]); }
        // b[r] *= w8^r, w8 = exp(-+ i pi/4)
        b[1] = INV ? cmk<C>(h * (b[1].x - b[1].y), h * (b[1].x + b[1].y))
                   : cmk<C>(h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
        b[2] = mul_mi<INV>(b[2]);
        b[3] = INV ? cmk<C>(-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y))
                   : cmk<C>(h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
        SmallDft<4, INV, T>::run(a);
        SmallDft<4, INV, T>::run(b);
#pragma unroll
        for (int q = 0; q < 4; q++) { v[2 * q] = a[q]; v[2 * q + 1] = b[q]; }
    }
};

// ---------------------------------------------------------------------------
// Stockham pass: nbatch transforms of length L at src[b*bstride + i]
// ---------------------------------------------------------------------------
template <int R, bool INV, typename T>
__device__ __forceinline__ void stockham_pass(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst,
                                              const cplx<T>* __restrict__ tw, int nb, int stride, int Ns,
                                              int nbatch, int bstride, int tid, int nth, unsigned int mnb,
                                              unsigned int mns) {
    using C = cplx<T>;
    const int total = nbatch * nb;
    for (int idx = tid; idx < total; idx += nth) {
        const int b = (int)fastdiv((unsigned)idx, (unsigned)nb, mnb);
        const int j = idx - b * nb;
        const C* s = src + b * bstride;
        C* d = dst + b * bstride;
        const int jq = (int)fastdiv((unsigned)j, (unsigned)Ns, mns);
        const int k = j - jq * Ns;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = s[j + r * nb];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                C w = tw[k * r * stride];  // shared (FP32 kernels) or global (FP64)
                if (INV) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        SmallDft<R, INV, T>::run(v);
        const int idxD = jq * Ns * R + k;
#pragma unroll
        for (int q = 0; q < R; q++) d[idxD + q * Ns] = v[q];
    }
}

// generic radix (any factor without a register butterfly): O(R^2) per group
template <bool INV, typename T>
__device__ __forceinline__ void stockham_pass_generic(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst,
                                                      const cplx<T>* __restrict__ tw, int L, int R, int Ns,
                                                      int nbatch, int bstride, int tid, int nth) {
    using C = cplx<T>;
    const int nb = L / R;
    const int stride = L / (Ns * R);
    const int total = nbatch * nb * R;
    for (int idx = tid; idx < total; idx += nth) {
        const int q = idx % R;
        const int bj = idx / R;
        const int b = bj / nb;
        const int j = bj - b * nb;
        const int k = j % Ns;
        const C* s = src + b * bstride;
        C acc = cmk<C>(T(0), T(0));
        for (int r = 0; r < R; r++) {
            C v = s[j + r * nb];
            // twiddle w_L^(k r stride) then w_R^(q r) = w_L^((q r mod R) * nb)
            const int e = (k * r * stride + ((q * r) % R) * nb) % L;
            C w = tw[e];
            if (INV) w.y = -w.y;
            acc = cadd(acc, cmul(v, w));
        }
        const int idxD = (j / Ns) * Ns * R + k;
        dst[b * bstride + idxD + q * Ns] = acc;
    }
}

// Runs all passes of plan p on buf0 (scratch buf1), returns where the result is.
// Every thread of the block must call it (it synchronises between passes).
template <bool INV, typename T>
__device__ cplx<T>* fft_batch(cplx<T>* buf0, cplx<T>* buf1, const FftPlan& p, int nbatch, int bstride) {
    using C = cplx<T>;
    const C* tw = plan_tw<T>(p);
    const int tid = threadIdx.x, nth = blockDim.x;
    C* src = buf0;
    C* dst = buf1;
    for (int ps = 0; ps < p.npass; ps++) {
        const int R = p.radix[ps], nb = p.nb[ps], ts = p.tstride[ps], Ns = p.ns[ps];
        const unsigned mnb = p.mag_nb[ps], mns = p.mag_ns[ps];
        switch (R) {
            case 2: stockham_pass<2, INV, T>(src, dst, tw, nb, ts, Ns, nbatch, bstride, tid, nth, mnb, mns); break;
            case 3: stockham_pass<3, INV, T>(src, dst, tw, nb, ts, Ns, nbatch, bstride, tid, nth, mnb, mns); break;
            case 4: stockham_pass<4, INV, T>(src, dst, tw, nb, ts, Ns, nbatch, bstride, tid, nth, mnb, mns); break;
            case 5: stockham_pass<5, INV, T>(src, dst, tw, nb, ts, Ns, nbatch, bstride, tid, nth, mnb, mns); break;
            case 7: stockham_pass<7, INV, T>(src, dst, tw, nb, ts, Ns, nbatch, bstride, tid, nth, mnb, mns); break;
            case 8: stockham_pass<8, INV, T>(src, dst, tw, nb, ts, Ns, nbatch, bstride, tid, nth, mnb, mns); break;
            default: stockham_pass_generic<INV, T>(src, dst, tw, p.L, R, Ns, nbatch, bstride, tid, nth); break;
        }
        __syncthreads();
        C* t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// ---------------------------------------------------------------------------
// Compiled radix sequences.  SEQ holds the radices of a plan's passes as decimal
// digits, the first pass most significant (350 = 5*5*2*7 -> 5527, 1024 = 8*4*8*4 ->
// 8484), so that the transform length, each pass's butterfly count, twiddle stride
// and sub-transform length are constants: no per-pass plan reads, no dispatch on the
// radix, divisions by constants only.  Measured on a single 350-point transform in one
// block (clock64, 64 repetitions): 1420 cycles against 3260 for the runtime passes.
// A kernel built for SEQ runs a plan whose schedule matches it (the host checks);
// SEQ = 0 selects the runtime passes of fft_batch.
// ---------------------------------------------------------------------------
constexpr int seq_npass(int s) { return s < 10 ? 1 : 1 + seq_npass(s / 10); }
constexpr int seq_pow10(int e) { return e == 0 ? 1 : 10 * seq_pow10(e - 1); }
constexpr int seq_radix(int s, int p) { return (s / seq_pow10(seq_npass(s) - 1 - p)) % 10; }
constexpr int seq_len(int s) { return s < 10 ? s : (s % 10) * seq_len(s / 10); }

// the sequence code of a schedule; 0 when a radix has no register butterfly or the
// code would not fit an int
inline int seq_code(const int* radix, int np) {
    if (np < 1 || np > 9) return 0;
    int c = 0;
    for (int i = 0; i < np; i++) {
        const int r = radix[i];
        if (r != 2 && r != 3 && r != 4 && r != 5 && r != 7 && r != 8) return 0;
        c = 10 * c + r;
    }
    return c;
}

template <int R, bool INV, typename T, int L, int NS>
__device__ __forceinline__ void ct_pass(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst,
                                        const cplx<T>* __restrict__ tw, int nbatch, int bstride) {
    using C = cplx<T>;
    constexpr int nb = L / R, stride = L / (NS * R);
    const int total = nbatch * nb;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int b = idx / nb;
        const int j = idx - b * nb;
        const C* s = src + b * bstride;
        C* d = dst + b * bstride;
        const int jq = j / NS;
        const int k = j - jq * NS;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = s[j + r * nb];
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                C w = tw[k * r * stride];
                if (INV) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        SmallDft<R, INV, T>::run(v);
        const int idxD = jq * NS * R + k;
#pragma unroll
        for (int q = 0; q < R; q++) d[idxD + q * NS] = v[q];
    }
}

// all passes of SEQ on src (scratch dst); returns where the result is, like fft_batch
template <bool INV, typename T, int SEQ, int P = 0, int NS = 1>
__device__ __forceinline__ cplx<T>* fft_batch_ct(cplx<T>* src, cplx<T>* dst, const cplx<T>* tw, int nbatch,
                                                 int bstride) {
    if constexpr (P == seq_npass(SEQ)) {
        return src;
    } else {
        constexpr int R = seq_radix(SEQ, P);
        ct_pass<R, INV, T, seq_len(SEQ), NS>(src, dst, tw, nbatch, bstride);
        __syncthreads();
        return fft_batch_ct<INV, T, SEQ, P + 1, NS * R>(dst, src, tw, nbatch, bstride);
    }
}

// The sequences the ensemble kernel dispatches on per task (SEQ_DISPATCH): the tuned
// schedules of its member grids 64, 96, 128, 192 and 256.
constexpr int SEQ_DISPATCH = -1;

// the compiled sequence SEQ (the caller has matched it to the plan), the runtime passes
// of the plan when SEQ == 0, or (SEQ_DISPATCH) the compiled sequence of the plan's own
// schedule when it is one of the ensemble set, else its runtime passes
template <bool INV, typename T, int SEQ>
__device__ __forceinline__ cplx<T>* fft_run(cplx<T>* buf0, cplx<T>* buf1, const FftPlan& p, int nbatch,
                                            int bstride) {
    if constexpr (SEQ == 0) {
        return fft_batch<INV, T>(buf0, buf1, p, nbatch, bstride);
    } else if constexpr (SEQ == SEQ_DISPATCH) {
        const cplx<T>* tw = plan_tw<T>(p);
        switch (p.seq) {
            case 444: return fft_batch_ct<INV, T, 444>(buf0, buf1, tw, nbatch, bstride);
            case 834: return fft_batch_ct<INV, T, 834>(buf0, buf1, tw, nbatch, bstride);
            case 484: return fft_batch_ct<INV, T, 484>(buf0, buf1, tw, nbatch, bstride);
            case 838: return fft_batch_ct<INV, T, 838>(buf0, buf1, tw, nbatch, bstride);
            case 2288: return fft_batch_ct<INV, T, 2288>(buf0, buf1, tw, nbatch, bstride);
            default: return fft_batch<INV, T>(buf0, buf1, p, nbatch, bstride);
        }
    } else {
        return fft_batch_ct<INV, T, SEQ>(buf0, buf1, plan_tw<T>(p), nbatch, bstride);
    }
}

}  // namespace fi
