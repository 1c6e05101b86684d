// fi_api.cu -- the C ABI (include/fastiso_b200.h): handle lifecycle, FP64 set-up,
// the fused FP32 step loop as a CUDA graph (conditional WHILE over BS3 steps,
// conditional IF per sparse update), and the plain FP64 form with a host-side
// step controller.  Integrator semantics: OrdinaryDiffEq BS3 as driven by
// run!/init_integrator/step! (src/simulation.jl:236-322).
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <complex>
#include <map>
#include <string>
#include <vector>

#include "../../include/fastiso_b200.h"
#include "fi_device.cuh"
#include "fi_kernels.h"
#include "fi_noalloc.cuh"
#include "fi_phases.cuh"
#include "fi_plain.h"

using namespace fi;

namespace {

constexpr int NT = 256;
enum { EXEC_PERSIST = FI_EXEC_PERSIST, EXEC_GRAPH = FI_EXEC_GRAPH, EXEC_LOOP = FI_EXEC_LOOP };

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }
inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

struct Plan {
    int L;
    int npass;
    int radix[FFT_MAX_PASSES];
    unsigned mag_nb[FFT_MAX_PASSES], mag_ns[FFT_MAX_PASSES];
    int nb[FFT_MAX_PASSES], tstride[FFT_MAX_PASSES], ns[FFT_MAX_PASSES];
    float2* tw32;
    double2* tw64;
};

struct PlainBufs {
    double *u[2], *k14[2], *k2, *k3, *tmp, *uin, *fscratch;
    double *now_u, *ue, *dz, *H, *H_af, *z_b, *z_ss, *s_i, *s_l, *s_m, *s_load, *s_full, *dudt;
    double *rhs, *bxx, *byy, *bx, *bxy, *Mxx, *Myy, *Mxy, *buf, *cropped, *off, *partial;
    double2 *fftrhs, *P;
    double *D, *eta, *mask, *u_ref, *ue_ref, *z_b_ref, *z_ss_ref, *H_af_ref, *H_tab;
    double *s_sw, *mgr, *moc, *hwater;  // seawater anomaly, masks, water column
    double *tau, *u_eq;                 // ELRA relaxation time and equilibrium displacement
    double2 *Gv_hat, *fftU;             // ELRA kernel spectrum; spectrum of u (laterally-constant Maxwell)
    double2 *Ge_hat, *Gg_hat;
};

}  // namespace

struct fi_handle {
    fi_config cfg;
    std::string err;
    cudaStream_t stream = nullptr;
    int nx, ny, NH, sp, Mx, My, MH, msp, mx, my, i1, j1;
    double dx, dy;
    std::vector<void*> allocs;
    // FFT plans
    std::map<int, int> plan_of_len;
    size_t n_plans_dev = 0;
    std::vector<Plan> plans;
    FftPlan* d_plans = nullptr;
    int plan_x, plan_y, plan_Mx, plan_My;
    // host-side inputs
    std::vector<double> D, eta, R, mask, u_ref, ue_ref, dz_ss_ref, z_b_ref, u_init, tau;
    bool R_given = false, u_set = false;
    std::vector<double> ice_t, ice_H;
    std::vector<double> rm, GE;
    std::vector<double> ch_ratio, ch_thick;
    // FP64 set-up products
    double *d_pd = nullptr, *d_R = nullptr, *d_spinv = nullptr, *d_Ge = nullptr, *d_Gg = nullptr;
    double2 *d_P64 = nullptr;
    std::vector<double> H_ice_ref, H_af_ref, z_ss_ref;
    // fused form
    Member mem{};
    Member* d_mem = nullptr;
    Ctl* d_ctl = nullptr;
    Task *t_rows = nullptr, *t_cols = nullptr, *t_crow = nullptr, *t_ccol = nullptr, *t_crowi = nullptr;
    int n_rows, n_cols, n_crow, n_ccol, n_crowi;
    int h_rows = 2, B_cols = 2, h_conv = 2, B_conv = 1;
    int stage_inputs = 0;  // forward row inputs: 1 = async copies into shared memory, 0 = in place
    double* d_uin = nullptr;
    float* d_vscr = nullptr;
    double* d_cscr = nullptr;
    double* d_red = nullptr;
    int red_blocks = 0;
    double* d_tout = nullptr;
    cudaGraphExec_t seg_exec = nullptr;
    cudaGraph_t seg_graph = nullptr;
    bool graph_ok = true;
    // step executor of the fused form: persistent cooperative kernel, CUDA graph, or
    // host-driven loop of per-phase launches (FI_EXECUTOR=persist|graph|loop)
    int executor = EXEC_PERSIST;
    unsigned int* d_bar = nullptr;
    PersistArgs pargs{};
    int persist_grid = 0;
    int persist_minb = 2;  // which k_persist build runs (blocks per SM of its register budget)
    size_t persist_smem = 0;
    unsigned long long* d_trace = nullptr;  // phase timeline of the persistent executor
    // plain form
    PlainBufs p{};
    // integrator (host mirror for the plain form; snapshot for the fused form)
    Ctl ctl{};
    std::vector<double> tstops, tout;
    bool initialized = false, integ_started = false;
    int last_call = 0;  // 0: step loop, 1: fi_rhs
    bool fsal_pending = false;  // FSAL re-evaluation owed by the last output callback
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double gpu_ms = 0.0, last_gpu_ms = 0.0;
    long long segments = 0;
    size_t smem_cap = 0;    // dynamic shared memory every per-phase kernel accepts
    size_t smem_optin = 0;  // the device's opt-in shared memory per block
    double last_rhs_t = 0.0;
    long long nf_plain = 0;
    // asynchronous output pipeline of fi_run: two staging slots (device FP64 copies of
    // u, ue, dudt, dz_ss), read back on a copy stream into pinned host slots
    cudaStream_t cstream = nullptr;
    cudaEvent_t ev_staged[2] = {nullptr, nullptr}, ev_copied[2] = {nullptr, nullptr};
    double* d_out_slot[2] = {nullptr, nullptr};
    double* h_out_slot[2] = {nullptr, nullptr};
    struct PendingOut {
        bool busy = false;
        int k = 0;
        double* dst[4] = {nullptr, nullptr, nullptr, nullptr};
    } pend[2];
    // sea level: tables of PiecewiseConstantBSL (z -> A) and ImposedBSL (t -> z)
    std::vector<double> osurf_z, osurf_A, bslh_t, bslh_z;
    // step-sequence record / replay buffers (FP32 form: device, plain form: host)
    double* d_rec = nullptr;
    double* d_replay = nullptr;
    std::vector<double> h_rec, h_replay;
};

static int set_err(fi_handle* h, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    h->err = buf;
    return code;
}

#define CK(x)                                                                                         \
    do {                                                                                              \
        cudaError_t e__ = (x);                                                                        \
        if (e__ != cudaSuccess)                                                                       \
            return set_err(h, FI_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #x, cudaGetErrorString(e__)); \
    } while (0)

#define CKL()                                                                                         \
    do {                                                                                              \
        cudaError_t e__ = cudaGetLastError();                                                         \
        if (e__ != cudaSuccess)                                                                       \
            return set_err(h, FI_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e__)); \
    } while (0)

#define RET(x)                 \
    do {                       \
        int r__ = (x);         \
        if (r__) return r__;   \
    } while (0)

template <typename T>
static int dalloc(fi_handle* h, T** p, size_t n) {
    void* q = nullptr;
    CK(cudaMalloc(&q, (n ? n : 1) * sizeof(T)));
    CK(cudaMemsetAsync(q, 0, (n ? n : 1) * sizeof(T), h->stream));
    h->allocs.push_back(q);
    *p = (T*)q;
    return FI_OK;
}

// radix schedule of a plan (passes in order) and the fast-division constants of each pass
static void plan_schedule(Plan& p, const int* radix, int np) {
    p.npass = np;
    for (int i = 0, Ns = 1; i < np; i++) {
        p.radix[i] = radix[i];
        p.mag_nb[i] = fastdiv_magic((unsigned)(p.L / radix[i]));
        p.mag_ns[i] = fastdiv_magic((unsigned)Ns);
        p.nb[i] = p.L / radix[i];
        p.tstride[i] = p.L / (Ns * radix[i]);
        p.ns[i] = Ns;
        Ns *= radix[i];
    }
}

// default schedule: radix 8 while possible, then 4, 2, 7, 5, 3, larger odd factors
static int default_schedule(int L, int* radix) {
    int m = L, np = 0;
    while (m % 8 == 0) { radix[np++] = 8; m /= 8; }
    while (m % 4 == 0) { radix[np++] = 4; m /= 4; }
    while (m % 2 == 0) { radix[np++] = 2; m /= 2; }
    const int small[3] = {7, 5, 3};
    for (int q : small) while (m % q == 0) { radix[np++] = q; m /= q; }
    for (int f = 11; f * f <= m; f += 2) while (m % f == 0) { radix[np++] = f; m /= f; }
    if (m > 1) radix[np++] = m;
    return np;
}

static int get_plan(fi_handle* h, int L, int* out) {
    auto it = h->plan_of_len.find(L);
    if (it != h->plan_of_len.end()) { *out = it->second; return FI_OK; }
    if (L < 1 || L > FFT_MAX_LEN) return set_err(h, FI_ERR_ARG, "transform length %d outside [1, %d]", L, FFT_MAX_LEN);
    Plan p{};
    p.L = L;
    int radix[FFT_MAX_PASSES];
    plan_schedule(p, radix, default_schedule(L, radix));
    std::vector<double2> t64(L);
    std::vector<float2> t32(L);
    for (int k = 0; k < L; k++) {
        const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)L;
        t64[k] = make_double2((double)cosl(a), (double)sinl(a));
        t32[k] = make_float2((float)t64[k].x, (float)t64[k].y);
    }
    RET(dalloc(h, &p.tw64, L));
    RET(dalloc(h, &p.tw32, L));
    CK(cudaMemcpyAsync(p.tw64, t64.data(), L * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(p.tw32, t32.data(), L * sizeof(float2), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *out = (int)h->plans.size();
    h->plan_of_len[L] = *out;
    h->plans.push_back(p);
    return FI_OK;
}

static void copy_plan(const Plan& q, FftPlan& dst) {
    dst.L = q.L;
    dst.npass = q.npass;
    memcpy(dst.radix, q.radix, sizeof(dst.radix));
    memcpy(dst.mag_nb, q.mag_nb, sizeof(dst.mag_nb));
    memcpy(dst.mag_ns, q.mag_ns, sizeof(dst.mag_ns));
    memcpy(dst.nb, q.nb, sizeof(dst.nb));
    memcpy(dst.tstride, q.tstride, sizeof(dst.tstride));
    memcpy(dst.ns, q.ns, sizeof(dst.ns));
    dst.tw32 = q.tw32;
    dst.tw64 = q.tw64;
    dst.seq = seq_code(q.radix, q.npass);
}

// The FP32 kernels read the plans from the member descriptor (staged in shared memory);
// refreshed whenever a schedule changes before fi_init uploads the descriptor.
static void copy_member_plans(fi_handle* h) {
    Member& m = h->mem;
    copy_plan(h->plans[h->plan_x], m.px);
    copy_plan(h->plans[h->plan_y], m.py);
    copy_plan(h->plans[h->plan_Mx], m.pMx);
    copy_plan(h->plans[h->plan_My], m.pMy);
}

static int upload_plans(fi_handle* h) {
    std::vector<FftPlan> v(h->plans.size());
    for (size_t i = 0; i < v.size(); i++) {
        v[i].L = h->plans[i].L;
        v[i].npass = h->plans[i].npass;
        memcpy(v[i].radix, h->plans[i].radix, sizeof(v[i].radix));
        memcpy(v[i].mag_nb, h->plans[i].mag_nb, sizeof(v[i].mag_nb));
        memcpy(v[i].mag_ns, h->plans[i].mag_ns, sizeof(v[i].mag_ns));
        memcpy(v[i].nb, h->plans[i].nb, sizeof(v[i].nb));
        memcpy(v[i].tstride, h->plans[i].tstride, sizeof(v[i].tstride));
        memcpy(v[i].ns, h->plans[i].ns, sizeof(v[i].ns));
        v[i].tw32 = h->plans[i].tw32;
        v[i].tw64 = h->plans[i].tw64;
        v[i].seq = seq_code(h->plans[i].radix, h->plans[i].npass);
    }
    if (!h->d_plans || h->n_plans_dev != v.size()) {
        RET(dalloc(h, &h->d_plans, v.size()));
        h->n_plans_dev = v.size();
    }
    CK(cudaMemcpyAsync(h->d_plans, v.data(), v.size() * sizeof(FftPlan), cudaMemcpyHostToDevice, h->stream));
    return FI_OK;
}

static int nextfastfft(int n) {
    for (int m = std::max(n, 1);; m++) {
        int r = m;
        for (int p : {2, 3, 5, 7}) while (r % p == 0) r /= p;
        if (r == 1) return m;
    }
}

static inline size_t N2(const fi_handle* h) { return (size_t)h->nx * h->ny; }

extern "C" {

void fi_config_default(fi_config* c, int32_t nx, int32_t ny, double Wx, double Wy) {
    memset(c, 0, sizeof(*c));
    c->nx = nx; c->ny = ny; c->Wx = Wx; c->Wy = Wy;
    c->mE = 5.972e24;
    c->r_pole = 6357e3;
    c->g = 9.8;
    c->seconds_per_year = 60.0 * 60.0 * 24 * 365.25;
    c->rho_ice = 0.910e3;
    c->rho_water = 1e3;
    c->rho_seawater = 1.023e3;
    c->rho_litho = 3.2e3;
    c->rho_uppermantle = 3.4e3;
    c->litho_poissonratio = 0.28;
    c->lithosphere = FI_LITHO_LATERALLY_VARIABLE;
    c->lithosphere_column = FI_COLUMN_INCOMPRESSIBLE;
    c->sea_surface = FI_SEA_SURFACE_LATERALLY_CONSTANT;
    c->ice_mode = FI_ICE_TIME_INTERPOLATED;
    c->t0 = 0.0;
    c->t1 = 1.0;
    c->reltol = (double)1e-5f;
    c->abstol = 1e-6;
    c->dt_sparse_diagnostics = 10.0;
    c->max_steps = 1000000;
    c->form = FI_FORM_FP32;
    c->sealevel_load = FI_SEALEVEL_LOAD_NONE;
    c->bsl_mode = FI_BSL_CONSTANT;
    c->bsl_update = FI_BSL_UPDATE_INTERNAL;
    c->volume_contribution = FI_CONTRIB_GOELZER;
    c->density_contribution = FI_CONTRIB_GOELZER;
    c->adjustment_contribution = FI_CONTRIB_NONE;
    c->bsl_ref_A = 3.625e14;  // A_OCEAN_PD, src/barystatic_sealevel.jl:1
}

const char* fi_status_string(int32_t s) {
    switch (s) {
        case FI_OK: return "ok";
        case FI_ERR_ARG: return "invalid argument";
        case FI_ERR_CUDA: return "CUDA error";
        case FI_ERR_NONFINITE: return "non-finite value in the state or error norm";
        case FI_ERR_DT_UNDERFLOW: return "dt below dtmin";
        case FI_ERR_FORCING_RANGE: return "TimeInterpolation2D out of range.";
        case FI_ERR_TIMEOUT: return "device wait timed out";
        case FI_ERR_STATE: return "call out of lifecycle order";
        case FI_ERR_UNSUPPORTED: return "option outside the LV-ELVA path";
        case FI_ERR_MAXITERS: return "maximum number of steps reached";
        default: return "unknown";
    }
}

const char* fi_last_error(const fi_handle* h) { return h ? h->err.c_str() : "null handle"; }

static int create_buffers(fi_handle* h);

int fi_create(const fi_config* cfg, fi_handle** out) {
    if (!cfg || !out) return FI_ERR_ARG;
    *out = nullptr;
    if (cfg->nx < 4 || cfg->ny < 4 || cfg->nx > 2048 || cfg->ny > 2048) return FI_ERR_ARG;
    if (!(cfg->Wx > 0) || !(cfg->Wy > 0) || !(cfg->t1 >= cfg->t0)) return FI_ERR_ARG;
    if (cfg->form != FI_FORM_FP32 && cfg->form != FI_FORM_FP64) return FI_ERR_ARG;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return FI_ERR_CUDA;
    fi_handle* h = new fi_handle();
    h->cfg = *cfg;
    h->nx = cfg->nx; h->ny = cfg->ny;
    h->mx = h->nx / 2; h->my = h->ny / 2;
    h->NH = h->nx / 2 + 1;
    h->sp = round_up(h->NH, 16);
    h->Mx = nextfastfft(2 * h->nx - 1);
    h->My = nextfastfft(2 * h->ny - 1);
    h->MH = h->Mx / 2 + 1;
    h->msp = round_up(h->MH, 16);
    h->i1 = (h->nx % 2 == 0) ? h->mx - 1 : h->mx;  // samesize_conv_indices, 0-based
    h->j1 = (h->ny % 2 == 0) ? h->my - 1 : h->my;
    h->dx = 2 * cfg->Wx / h->nx;
    h->dy = 2 * cfg->Wy / h->ny;
    const size_t n = N2(h);
    h->D.assign(n, 0.0);
    h->eta.assign(n, 0.0);
    h->R.assign(n, 1.0);
    h->mask.assign(n, 1.0);
    h->u_ref.assign(n, 0.0);
    h->ue_ref.assign(n, 0.0);
    h->dz_ss_ref.assign(n, 0.0);
    h->z_b_ref.assign(n, 1e6);
    h->u_init.assign(n, 0.0);
    h->tau.assign(n, 855.0);  // DEFAULT_MANTLE_TAU, src/solidearth.jl:121
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return FI_ERR_CUDA;
    }
    const char* ex = getenv("FI_EXECUTOR");
    if (ex && !strcmp(ex, "graph")) h->executor = EXEC_GRAPH;
    if (ex && !strcmp(ex, "loop")) h->executor = EXEC_LOOP;
    const char* ng = getenv("FI_NO_GRAPH");
    if (ng && ng[0] == '1') h->executor = EXEC_LOOP;
    if (h->executor == EXEC_LOOP) h->graph_ok = false;
    int rc = create_buffers(h);
    if (!rc && (cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess)) rc = FI_ERR_CUDA;
    if (rc) {
        fprintf(stderr, "fi_create: %s\n", h->err.c_str());
        fi_destroy(h);
        return rc;
    }
    *out = h;
    return FI_OK;
}

void fi_destroy(fi_handle* h) {
    if (!h) return;
    cudaSetDevice(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->seg_exec) cudaGraphExecDestroy(h->seg_exec);
    if (h->seg_graph) cudaGraphDestroy(h->seg_graph);
    for (void* p : h->allocs) cudaFree(p);
    if (h->d_rec) cudaFree(h->d_rec);
    if (h->d_replay) cudaFree(h->d_replay);
    for (int q = 0; q < 2; q++) {
        if (h->ev_staged[q]) cudaEventDestroy(h->ev_staged[q]);
        if (h->ev_copied[q]) cudaEventDestroy(h->ev_copied[q]);
        if (h->d_out_slot[q]) cudaFree(h->d_out_slot[q]);
        if (h->h_out_slot[q]) cudaFreeHost(h->h_out_slot[q]);
    }
    if (h->cstream) {
        cudaStreamSynchronize(h->cstream);
        cudaStreamDestroy(h->cstream);
    }
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------
static void set_task_counts(fi_handle* h) {
    h->n_rows = cdiv(h->ny, h->h_rows);
    h->n_cols = cdiv(h->NH, h->B_cols);
    h->n_crow = cdiv(h->ny, h->h_conv);
    h->n_ccol = cdiv(h->MH, h->B_conv);
    h->n_crowi = cdiv(h->ny + 2, h->h_conv);
}

static int create_buffers(fi_handle* h) {
    const size_t n = N2(h);
    RET(get_plan(h, h->nx, &h->plan_x));
    RET(get_plan(h, h->ny, &h->plan_y));
    RET(get_plan(h, h->Mx, &h->plan_Mx));
    RET(get_plan(h, h->My, &h->plan_My));
    RET(upload_plans(h));
    RET(dalloc(h, &h->d_pd, n));
    RET(dalloc(h, &h->d_R, n));
    RET(dalloc(h, &h->d_spinv, n));
    RET(dalloc(h, &h->d_Ge, n));
    RET(dalloc(h, &h->d_Gg, n));
    RET(dalloc(h, &h->d_P64, (size_t)h->Mx * h->My));
    h->red_blocks = std::min(1024, cdiv((long long)n, NT));
    RET(dalloc(h, &h->d_red, 2 * (size_t)h->red_blocks));
    RET(dalloc(h, &h->d_tout, MAX_TSTOPS));
    if (h->cfg.form == FI_FORM_FP32) {
        Member& m = h->mem;
        m.nx = h->nx; m.ny = h->ny; m.NH = h->NH; m.sp = h->sp;
        m.Mx = h->Mx; m.My = h->My; m.MH = h->MH; m.msp = h->msp;
        m.i1 = h->i1; m.j1 = h->j1;
        m.plan_x = h->plan_x; m.plan_y = h->plan_y; m.plan_Mx = h->plan_Mx; m.plan_My = h->plan_My;
        copy_member_plans(h);
        for (int b = 0; b < 2; b++) {
            RET(dalloc(h, &m.u[b], n));
            RET(dalloc(h, &m.k14[b], n));
            RET(dalloc(h, &m.ue[b], n));
        }
        RET(dalloc(h, &m.k2, n));
        RET(dalloc(h, &m.k3, n));
        float *D, *vf, *mult, *mask, *hafref, *sigref, *zbss, *ueref, *Hext;
        RET(dalloc(h, &D, n)); m.D = D;
        RET(dalloc(h, &vf, n)); m.visc_fac = vf;
        RET(dalloc(h, &mult, (size_t)h->NH * h->ny)); m.mult = mult;
        RET(dalloc(h, &mask, n)); m.mask = mask;
        RET(dalloc(h, &hafref, n)); m.H_af_ref = hafref;
        RET(dalloc(h, &sigref, n)); m.sigma_ref = sigref;
        RET(dalloc(h, &zbss, n)); m.zbss_ref = zbss;
        RET(dalloc(h, &ueref, n)); m.ue_ref = ueref;
        RET(dalloc(h, &Hext, n)); m.H_ext = Hext;
        RET(dalloc(h, &m.dz, n));
        RET(dalloc(h, &m.sw, n));
        RET(dalloc(h, &m.mgr, n));
        RET(dalloc(h, &m.moc, n));
        RET(dalloc(h, &m.hwater, n));
        RET(dalloc(h, &m.sig_load, n));
        RET(dalloc(h, &m.sig_geo, n));
        RET(dalloc(h, &m.S[0], (size_t)h->ny * h->sp));
        RET(dalloc(h, &m.S[1], (size_t)h->ny * h->sp));
        RET(dalloc(h, &m.SA, (size_t)h->ny * h->msp));
        RET(dalloc(h, &m.SB, (size_t)h->ny * h->msp));
        RET(dalloc(h, &m.TA, (size_t)(h->ny + 2) * h->msp));
        RET(dalloc(h, &m.TB, (size_t)(h->ny + 2) * h->msp));
        float2 *GA, *GB;
        RET(dalloc(h, &GA, (size_t)h->MH * h->My)); m.GA = GA;
        RET(dalloc(h, &GB, (size_t)h->MH * h->My)); m.GB = GB;
        RET(dalloc(h, &m.partial, (size_t)h->ny + 16));
        RET(dalloc(h, &m.cpart, (size_t)4 * (h->NH + 16)));
        RET(dalloc(h, &h->d_ctl, 1));
        RET(dalloc(h, &h->d_bar, 4));
        RET(dalloc(h, &h->d_trace, 2 * PH_COUNT));
        m.ctl = h->d_ctl;
        m.tout = h->d_tout;
        RET(dalloc(h, &h->d_uin, n));
        RET(dalloc(h, &h->d_vscr, n));
        RET(dalloc(h, &h->d_cscr, 8));
        RET(dalloc(h, &h->d_mem, 1));
        // tunables
        h->h_rows = 2;
        h->B_cols = h->ny >= 768 ? 1 : 2;
        if (const char* e = getenv("FI_H_ROWS")) h->h_rows = std::max(1, std::min(8, atoi(e)));
        if (const char* e = getenv("FI_B_COLS")) h->B_cols = std::max(1, std::min(8, atoi(e)));
        if (const char* e = getenv("FI_STAGE_INPUTS")) h->stage_inputs = atoi(e) ? 1 : 0;
        h->h_conv = h->Mx >= 1024 ? 1 : 2;
        h->B_conv = 1;
        set_task_counts(h);
        // task lists (0, i) sized for the smallest tiles, so fi_set_tiles only changes counts
        auto mk = [&](Task** dst, int count) -> int {
            std::vector<Task> t(count);
            for (int i = 0; i < count; i++) t[i] = Task{0, i};
            RET(dalloc(h, dst, count));
            CK(cudaMemcpyAsync(*dst, t.data(), count * sizeof(Task), cudaMemcpyHostToDevice, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            return FI_OK;
        };
        RET(mk(&h->t_rows, h->ny));
        RET(mk(&h->t_cols, h->NH));
        RET(mk(&h->t_crow, h->ny));
        RET(mk(&h->t_ccol, h->MH));
        RET(mk(&h->t_crowi, h->ny + 2));
        // opt in to the full shared memory per block less each kernel's static shared
        // memory (member descriptor, control block, plans); the actual need (which
        // depends on the ice-table length) is checked in fi_init
        int smax = 0;
        CK(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->cfg.device));
        h->smem_optin = (size_t)smax;
        const void* fk[] = {(const void*)k_rows_fwd, (const void*)k_cols, (const void*)k_rows_inv,
                            (const void*)k_conv_rows, (const void*)k_conv_cols, (const void*)k_conv_rows_inv};
        size_t cap = (size_t)smax;
        for (const void* f : fk) {
            cudaFuncAttributes fa{};
            CK(cudaFuncGetAttributes(&fa, f));
            if (fa.sharedSizeBytes >= (size_t)smax) return set_err(h, FI_ERR_CUDA, "static shared memory too large");
            const size_t dyn = (size_t)smax - fa.sharedSizeBytes;
            CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
            cap = std::min(cap, dyn);
        }
        h->smem_cap = cap;
    } else {
        PlainBufs& p = h->p;
        const size_t M = (size_t)h->Mx * h->My;
        double** bufs[] = {&p.u[0], &p.u[1], &p.k14[0], &p.k14[1], &p.k2, &p.k3, &p.tmp, &p.uin, &p.fscratch,
                           &p.now_u, &p.ue, &p.dz, &p.H, &p.H_af, &p.z_b, &p.z_ss, &p.s_i, &p.s_l, &p.s_m,
                           &p.s_load, &p.s_full, &p.dudt, &p.rhs, &p.bxx, &p.byy, &p.bx, &p.bxy, &p.Mxx,
                           &p.Myy, &p.Mxy, &p.buf, &p.D, &p.eta, &p.mask, &p.u_ref, &p.ue_ref, &p.z_b_ref,
                           &p.z_ss_ref, &p.H_af_ref, &p.s_sw, &p.mgr, &p.moc, &p.hwater, &p.tau, &p.u_eq};
        for (double** b : bufs) RET(dalloc(h, b, n));
        RET(dalloc(h, &p.cropped, (size_t)(2 * h->nx - 1) * (2 * h->ny - 1)));
        RET(dalloc(h, &p.off, 4));
        RET(dalloc(h, &p.partial, 3 * (size_t)h->red_blocks));
        RET(dalloc(h, &p.fftrhs, n));
        RET(dalloc(h, &p.fftU, n));
        RET(dalloc(h, &p.P, M));
        RET(dalloc(h, &p.Ge_hat, M));
        RET(dalloc(h, &p.Gg_hat, M));
        const size_t s1 = fft64_rows_smem(std::max(h->nx, h->Mx), 1), s2 = fft64_cols_smem(std::max(h->ny, h->My), 1);
        CK(cudaFuncSetAttribute(k_fft64_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1));
        CK(cudaFuncSetAttribute(k_fft64_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2));
    }
    if (h->cfg.form == FI_FORM_FP32) {
        // FP64 transforms of the set-up are needed by both forms
        const size_t s1 = fft64_rows_smem(h->Mx, 1), s2 = fft64_cols_smem(h->My, 1);
        CK(cudaFuncSetAttribute(k_fft64_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s1));
        CK(cudaFuncSetAttribute(k_fft64_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2));
    }
    CK(cudaStreamSynchronize(h->stream));
    return FI_OK;
}

// FP64 2D transform of an nx-by-ny complex plane with row pitch nx (1 line per block)
static int fft2_64(fi_handle* h, double2* a, int nx, int ny, int inverse) {
    int px, py;
    RET(get_plan(h, nx, &px));
    RET(get_plan(h, ny, &py));
    const double scale = inverse ? 1.0 / ((double)nx * ny) : 1.0;
    if (!inverse) {
        k_fft64_rows<<<ny, NT, fft64_rows_smem(nx, 1), h->stream>>>(a, nx, ny, nx, h->d_plans, px, 0, 1);
        CKL();
        k_fft64_cols<<<nx, NT, fft64_cols_smem(ny, 1), h->stream>>>(a, nx, ny, nx, h->d_plans, py, 0, 1, 1.0);
        CKL();
    } else {
        k_fft64_cols<<<nx, NT, fft64_cols_smem(ny, 1), h->stream>>>(a, nx, ny, nx, h->d_plans, py, 1, 1, scale);
        CKL();
        k_fft64_rows<<<ny, NT, fft64_rows_smem(nx, 1), h->stream>>>(a, nx, ny, nx, h->d_plans, px, 1, 1);
        CKL();
    }
    return FI_OK;
}

// ---------------------------------------------------------------------------
// field access
// ---------------------------------------------------------------------------
template <typename T>
static int upload(fi_handle* h, T* dst, const std::vector<double>& src) {
    std::vector<T> tmp(src.begin(), src.end());
    CK(cudaMemcpyAsync(dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FI_OK;
}

template <typename T>
static int download(fi_handle* h, std::vector<double>& dst, const T* src, size_t n) {
    std::vector<T> tmp(n);
    CK(cudaMemcpyAsync(tmp.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    dst.assign(tmp.begin(), tmp.end());
    return FI_OK;
}

static int read_ctl(fi_handle* h) {
    if (h->cfg.form != FI_FORM_FP32) return FI_OK;
    CK(cudaMemcpyAsync(&h->ctl, h->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FI_OK;
}

static int write_ctl(fi_handle* h) {
    if (h->cfg.form != FI_FORM_FP32) return FI_OK;
    CK(cudaMemcpyAsync(h->d_ctl, &h->ctl, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FI_OK;
}

static double corner_mean(const double* c) { return 0.25 * (c[0] + c[1] + c[2] + c[3]); }

static void interp_ice_host(const fi_handle* h, double t, std::vector<double>& H, int* status) {
    const size_t n = N2(h);
    H.assign(n, 0.0);
    *status = FI_OK;
    if (h->cfg.ice_mode != FI_ICE_TIME_INTERPOLATED || h->ice_t.empty()) return;
    const std::vector<double>& tt = h->ice_t;
    const int K = (int)tt.size();
    int i;
    if (t < tt[0] || t > tt[K - 1]) {
        if (!h->cfg.ice_flat_bc) { *status = FI_ERR_FORCING_RANGE; return; }
        i = t < tt[0] ? 0 : K - 1;
        std::copy(h->ice_H.begin() + (size_t)i * n, h->ice_H.begin() + (size_t)(i + 1) * n, H.begin());
        return;
    }
    i = (int)(std::lower_bound(tt.begin(), tt.end(), t) - tt.begin());
    if (tt[i] == t) {
        std::copy(h->ice_H.begin() + (size_t)i * n, h->ice_H.begin() + (size_t)(i + 1) * n, H.begin());
        return;
    }
    i -= 1;
    const double* a = &h->ice_H[(size_t)i * n];
    const double* b = &h->ice_H[(size_t)(i + 1) * n];
    const double dti = tt[i + 1] - tt[i], ts = t - tt[i];
    for (size_t k = 0; k < n; k++) H[k] = a[k] + (b[k] - a[k]) / dti * ts;
}

static double haf_host(double rho_sw_ice, double H, double zb, double zss) {
    double m = zb - zss;
    if (m > 0) m = 0;
    const double v = H + m * rho_sw_ice;
    return v > 0 ? v : 0.0;
}

extern "C" int fi_set_field(fi_handle* h, int32_t field, const double* host, size_t n) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !host) return FI_ERR_ARG;
    if (n != N2(h)) return set_err(h, FI_ERR_ARG, "field size %zu != nx*ny", n);
    if (field == FI_FIELD_U && h->initialized) {
        // integrator.u .= host, as a coupling callback does: copied straight from the
        // caller's buffer (pinned memory makes it one DMA); the next step re-evaluates
        // the FSAL derivative at the new state (u_modified!)
        if (h->cfg.form == FI_FORM_FP32) {
            RET(read_ctl(h));
            CK(cudaMemcpyAsync(h->mem.u[h->ctl.ibuf], host, n * 8, cudaMemcpyHostToDevice, h->stream));
        } else {
            CK(cudaMemcpyAsync(h->p.u[h->ctl.ibuf], host, n * 8, cudaMemcpyHostToDevice, h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
        if (h->integ_started) h->fsal_pending = true;
        return FI_OK;
    }
    std::vector<double> v(host, host + n);
    switch (field) {
        case FI_FIELD_LITHO_RIGIDITY: h->D = v; return FI_OK;
        case FI_FIELD_EFFECTIVE_VISCOSITY: h->eta = v; return FI_OK;
        case FI_FIELD_PSEUDODIFF_SCALING: h->R = v; h->R_given = true; return FI_OK;
        case FI_FIELD_MASKACTIVE: h->mask = v; return FI_OK;
        case FI_FIELD_U_REF: h->u_ref = v; return FI_OK;
        case FI_FIELD_UE_REF: h->ue_ref = v; return FI_OK;
        case FI_FIELD_DZ_SS_REF: h->dz_ss_ref = v; return FI_OK;
        case FI_FIELD_Z_B_REF: h->z_b_ref = v; return FI_OK;
        case FI_FIELD_TAU:
            for (double x : v)
                if (!(x > 0)) return set_err(h, FI_ERR_ARG, "tau must be positive");
            h->tau = v;
            return FI_OK;
        case FI_FIELD_U: h->u_init = v; h->u_set = true; return FI_OK;
        case FI_FIELD_H_ICE:
            if (h->cfg.ice_mode != FI_ICE_EXTERNAL)
                return set_err(h, FI_ERR_ARG, "H_ice is set externally only with FI_ICE_EXTERNAL");
            if (h->cfg.form == FI_FORM_FP32) return upload(h, h->mem.H_ext, v);
            return upload(h, h->p.H, v);
        default: return set_err(h, FI_ERR_ARG, "field %d is not settable", field);
    }
}

extern "C" int fi_set_ice_history(fi_handle* h, int32_t K, const double* t, const double* H) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || K < 1 || !t || !H) return FI_ERR_ARG;
    for (int k = 1; k < K; k++)
        if (!(t[k] > t[k - 1])) return set_err(h, FI_ERR_ARG, "ice times must increase");
    h->ice_t.assign(t, t + K);
    h->ice_H.assign(H, H + (size_t)K * N2(h));
    return FI_OK;
}

static int set_table(fi_handle* h, int32_t n, const double* x, const double* y, std::vector<double>& xo,
                     std::vector<double>& yo) {
    if (n < 2 || !x || !y) return set_err(h, FI_ERR_ARG, "a table needs >= 2 points");
    for (int k = 1; k < n; k++)
        if (!(x[k] > x[k - 1])) return set_err(h, FI_ERR_ARG, "table abscissae must increase");
    if (h->initialized) return set_err(h, FI_ERR_STATE, "tables are set before fi_init");
    xo.assign(x, x + n);
    yo.assign(y, y + n);
    return FI_OK;
}

extern "C" int fi_set_ocean_surface_table(fi_handle* h, int32_t n, const double* z, const double* A) {
    if (!h) return FI_ERR_ARG;
    return set_table(h, n, z, A, h->osurf_z, h->osurf_A);
}

extern "C" int fi_set_bsl_history(fi_handle* h, int32_t n, const double* t, const double* z) {
    if (!h) return FI_ERR_ARG;
    return set_table(h, n, t, z, h->bslh_t, h->bslh_z);
}

extern "C" int fi_set_elastic_table(fi_handle* h, int32_t n, const double* rm, const double* GE) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || n < 2 || !rm || !GE) return FI_ERR_ARG;
    h->rm.assign(rm, rm + n);
    h->GE.assign(GE, GE + n);
    return FI_OK;
}

extern "C" int fi_set_channel_scaling(fi_handle* h, int32_t n, const double* ratio, const double* thick) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || n < 0 || (n > 0 && (!ratio || !thick))) return FI_ERR_ARG;
    h->ch_ratio.assign(ratio, ratio + n);
    h->ch_thick.assign(thick, thick + n);
    return FI_OK;
}

extern "C" int fi_set_tiles(fi_handle* h, int32_t h_rows, int32_t B_cols) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h) return FI_ERR_ARG;
    if (h->initialized) return set_err(h, FI_ERR_STATE, "fi_set_tiles must precede fi_init");
    if (h->cfg.form != FI_FORM_FP32) return set_err(h, FI_ERR_UNSUPPORTED, "tiles apply to the FP32 form");
    if (h_rows < 1 || h_rows > 16 || B_cols < 1 || B_cols > 16)
        return set_err(h, FI_ERR_ARG, "tile height %d / column block %d outside [1, 16]", h_rows, B_cols);
    h->h_rows = h_rows;
    h->B_cols = B_cols;
    set_task_counts(h);
    return FI_OK;
}

extern "C" int fi_set_fft_schedule(fi_handle* h, int32_t L, int32_t n, const int32_t* radices) {
    if (!h) return FI_ERR_ARG;
    cudaSetDevice(h->cfg.device);
    if (h->initialized) return set_err(h, FI_ERR_STATE, "fi_set_fft_schedule must precede fi_init");
    auto it = h->plan_of_len.find(L);
    if (it == h->plan_of_len.end()) return set_err(h, FI_ERR_ARG, "%d is not a transform length of this grid", L);
    if (n < 1 || n > FFT_MAX_PASSES || !radices) return set_err(h, FI_ERR_ARG, "schedule of %d passes", n);
    long long prod = 1;
    int radix[FFT_MAX_PASSES];
    for (int i = 0; i < n; i++) {
        if (radices[i] < 2) return set_err(h, FI_ERR_ARG, "radix %d < 2", radices[i]);
        radix[i] = radices[i];
        prod *= radices[i];
        if (prod > L) break;
    }
    if (prod != L) return set_err(h, FI_ERR_ARG, "radices do not multiply to %d", L);
    plan_schedule(h->plans[it->second], radix, n);
    RET(upload_plans(h));
    if (h->cfg.form == FI_FORM_FP32) copy_member_plans(h);
    CK(cudaStreamSynchronize(h->stream));
    return FI_OK;
}

extern "C" int fi_get_fft_schedule(fi_handle* h, int32_t L, int32_t* n, int32_t* radices) {
    if (!h || !n || !radices) return FI_ERR_ARG;
    auto it = h->plan_of_len.find(L);
    if (it == h->plan_of_len.end()) return set_err(h, FI_ERR_ARG, "%d is not a transform length of this grid", L);
    const Plan& p = h->plans[it->second];
    *n = p.npass;
    for (int i = 0; i < p.npass; i++) radices[i] = p.radix[i];
    return FI_OK;
}

// ---------------------------------------------------------------------------
// set-up (Simulation constructor tail)
// ---------------------------------------------------------------------------
static int build_kernel_spectrum(fi_handle* h, const double* G, float2* half32, double2* full64) {
    const size_t M = (size_t)h->Mx * h->My;
    k_pad_real<<<cdiv(M, NT), NT, 0, h->stream>>>(G, h->nx, h->ny, h->d_P64, h->Mx, h->My);
    CKL();
    RET(fft2_64(h, h->d_P64, h->Mx, h->My, 0));
    if (half32) {
        k_half_spectrum32<<<cdiv((size_t)h->MH * h->My, NT), NT, 0, h->stream>>>(
            h->d_P64, h->Mx, h->My, h->MH, 1.0 / ((double)h->Mx * h->My), half32);
        CKL();
    }
    if (full64) CK(cudaMemcpyAsync(full64, h->d_P64, M * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    return FI_OK;
}

// K_0(z) of a complex argument with Re z > 0: K_0(z) = int_0^inf exp(-z cosh t) dt
// (Abramowitz & Stegun 9.6.24), trapezoidal rule with step 1/20 -- the integrand is
// entire and decays doubly exponentially, so the rule converges geometrically (about
// 1e-15 relative on the ray arg z = pi/4 that the Kelvin function uses).
static std::complex<double> bessel_k0(std::complex<double> z) {
    const double step = 0.05;
    std::complex<double> acc = 0.5 * std::exp(-z);
    for (int k = 1; k < 4000; k++) {
        const std::complex<double> v = std::exp(-z * std::cosh(k * step));
        acc += v;
        if (k * step > 1.0 && std::abs(v) < 1e-18 * std::abs(acc)) break;
    }
    return step * acc;
}

// The ELRA Green's function green_viscous(domain, rho_uppermantle, mean(D))
// (src/material.jl:370-399, src/tools.jl:53-58): -(L^2 / (2 pi D)) kei(max(R, 1) / L) dx dy,
// kei(x) = Im K_0(x e^{i pi/4}), L = (D / (rho_m 9.81))^(1/4), on the grid x_i = -W + i dx.
static std::vector<double> viscous_green(const fi_handle* h) {
    const size_t n = N2(h);
    double D = 0.0;
    for (double d : h->D) D += d;
    D /= (double)n;
    const double L = pow(D / (h->cfg.rho_uppermantle * 9.81), 0.25);
    const std::complex<double> rot = std::polar(1.0, M_PI / 4.0);
    std::vector<double> G(n);
    for (int j = 0; j < h->ny; j++)
        for (int i = 0; i < h->nx; i++) {
            const double x = -h->cfg.Wx + (i + 1) * h->dx, y = -h->cfg.Wy + (j + 1) * h->dy;
            const double R = std::max(sqrt(x * x + y * y), 1.0);
            const double kei = bessel_k0(R / L * rot).imag();
            G[i + (size_t)j * h->nx] = -(L * L / (2.0 * M_PI * D) * kei) * (h->dx * h->dy);
        }
    return G;
}

static int rhs_fused(fi_handle* h, int stage, const double* uin, float* vout, double* cout);
static int setup_persist(fi_handle* h, int K);
static int plan_layouts(fi_handle* h, int K);
static int rhs_plain(fi_handle* h, double t, double* u, double* dudt);

extern "C" int fi_init(fi_handle* h) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h) return FI_ERR_ARG;
    if (h->initialized) return set_err(h, FI_ERR_STATE, "fi_init called twice");
    const fi_config& c = h->cfg;
    const size_t n = N2(h);
    for (size_t k = 0; k < n; k++)
        if (!(h->eta[k] > 0) || !(h->D[k] >= 0))
            return set_err(h, FI_ERR_ARG, "litho_rigidity / effective_viscosity not set (or non-positive)");
    if (c.ice_mode == FI_ICE_TIME_INTERPOLATED && h->ice_t.empty())
        return set_err(h, FI_ERR_STATE, "ice history not set");
    const bool elastic = c.lithosphere != FI_LITHO_RIGID, geoid = c.sea_surface == FI_SEA_SURFACE_LATERALLY_VARIABLE;
    if (elastic && h->rm.size() < 2) return set_err(h, FI_ERR_STATE, "elastic Green table not set");
    if (c.mantle < FI_MANTLE_MAXWELL || c.mantle > FI_MANTLE_RIGID || c.alg < FI_ALG_BS3 || c.alg > FI_ALG_EULER ||
        c.lithosphere < FI_LITHO_LATERALLY_VARIABLE || c.lithosphere > FI_LITHO_LATERALLY_CONSTANT)
        return set_err(h, FI_ERR_ARG, "unknown mantle, lithosphere or integrator");
    if (c.mantle == FI_MANTLE_RELAXED && c.lithosphere == FI_LITHO_LATERALLY_VARIABLE)
        return set_err(h, FI_ERR_UNSUPPORTED, "Relaxed rheology is not implemented for laterally variable lithosphere.");
    if ((c.alg == FI_ALG_EULER) != (c.dt_min > 0))
        return set_err(h, FI_ERR_ARG, "The `dt_min` option is only compatible with the Euler algorithm.");
    if (c.form == FI_FORM_FP32 &&
        (c.mantle != FI_MANTLE_MAXWELL || c.lithosphere == FI_LITHO_LATERALLY_CONSTANT || c.alg != FI_ALG_BS3))
        return set_err(h, FI_ERR_UNSUPPORTED, "the FP32 form runs the LV-ELVA path (MaxwellMantle, laterally variable "
                                              "or rigid lithosphere, BS3); other rheologies run in the plain form");
    if (c.sealevel_load != FI_SEALEVEL_LOAD_NONE && c.sealevel_load != FI_SEALEVEL_LOAD_INTERACTIVE)
        return set_err(h, FI_ERR_ARG, "unknown sea-level load %d", c.sealevel_load);
    if (c.bsl_mode < FI_BSL_CONSTANT || c.bsl_mode > FI_BSL_IMPOSED)
        return set_err(h, FI_ERR_ARG, "unknown BSL %d", c.bsl_mode);
    const bool bsl_internal = c.bsl_update == FI_BSL_UPDATE_INTERNAL;
    if (bsl_internal && c.bsl_mode == FI_BSL_PIECEWISE_CONSTANT && h->osurf_z.size() < 2)
        return set_err(h, FI_ERR_STATE, "PiecewiseConstantBSL needs fi_set_ocean_surface_table");
    if (bsl_internal && c.bsl_mode == FI_BSL_IMPOSED && h->bslh_t.size() < 2)
        return set_err(h, FI_ERR_STATE, "ImposedBSL needs fi_set_bsl_history");
    if (c.form == FI_FORM_FP32 && bsl_internal &&
        (c.bsl_mode == FI_BSL_CONSTANT_OCEAN_SURFACE || c.bsl_mode == FI_BSL_PIECEWISE_CONSTANT))
        return set_err(h, FI_ERR_UNSUPPORTED,
                       "a BSL driven by the ice volume runs in the plain FP64 form (the FP32 form's sparse update "
                       "does not sum the volumes)");
    if (c.sealevel_load == FI_SEALEVEL_LOAD_INTERACTIVE) {
        size_t active = 0;
        for (size_t k = 0; k < n; k++) active += h->mask[k] != 0.0;
        if ((double)active > 0.6 * (double)n)
            return set_err(h, FI_ERR_ARG, "Mask defining regions of active load must not cover more than 60%% of "
                                          "the cells when using an interactive sea level.");
    }
    // spectral factors and Green's functions, FP64 on the device
    double *d_ratio = nullptr, *d_thick = nullptr, *d_Rg = nullptr;
    const int nch = (int)h->ch_ratio.size();
    RET(dalloc(h, &d_ratio, std::max(nch, 1)));
    RET(dalloc(h, &d_thick, std::max(nch, 1)));
    if (nch) {
        RET(upload(h, d_ratio, h->ch_ratio));
        RET(upload(h, d_thick, h->ch_thick));
    }
    if (h->R_given) {
        RET(dalloc(h, &d_Rg, n));
        RET(upload(h, d_Rg, h->R));
    }
    float* mult = (c.form == FI_FORM_FP32) ? (float*)h->mem.mult : nullptr;
    float* mult_tmp = nullptr;
    if (!mult) RET(dalloc(h, &mult_tmp, (size_t)h->NH * h->ny));
    k_spectral_factors<<<cdiv(n, NT), NT, 0, h->stream>>>(h->nx, h->ny, c.Wx, c.Wy, nch, d_ratio, d_thick, d_Rg,
                                                           c.seconds_per_year, h->d_pd, h->d_R, h->d_spinv,
                                                           mult ? mult : mult_tmp, h->NH);
    CKL();
    double *d_rm = nullptr, *d_GE = nullptr;
    if (elastic) {
        RET(dalloc(h, &d_rm, h->rm.size()));
        RET(dalloc(h, &d_GE, h->GE.size()));
        RET(upload(h, d_rm, h->rm));
        RET(upload(h, d_GE, h->GE));
        k_elastic_green<<<cdiv(n, NT), NT, 0, h->stream>>>(h->d_Ge, h->nx, h->ny, h->mx, h->my, h->dx, h->dy, d_rm,
                                                            d_GE, (int)h->rm.size());
        CKL();
    }
    k_geoid_green<<<cdiv(n, NT), NT, 0, h->stream>>>(h->d_Gg, h->nx, h->ny, c.Wx, c.Wy, h->dx, h->dy, c.r_pole, c.mE);
    CKL();
    // reference state (src/simulation.jl:132-151) in FP64 on the host
    int st;
    interp_ice_host(h, c.t0, h->H_ice_ref, &st);
    if (st) return set_err(h, st, "TimeInterpolation2D out of range.");
    h->z_ss_ref.resize(n);
    h->H_af_ref.resize(n);
    const double rsi = c.rho_seawater / c.rho_ice;
    // ReferenceState masks and water column (CurrentState copies them) and the volumes
    // of init_problem! (src/simulation.jl:132-151, 305-312)
    std::vector<double> mgr0(n), moc0(n), hw0(n);
    double saf = 0.0, sden = 0.0, spov = 0.0;
    for (size_t k = 0; k < n; k++) {
        h->z_ss_ref[k] = c.z_bsl + h->dz_ss_ref[k];
        h->H_af_ref[k] = haf_host(rsi, h->H_ice_ref[k], h->z_b_ref[k], h->z_ss_ref[k]);
        const bool gr = h->H_af_ref[k] > 0;
        const double w = h->z_ss_ref[k] - h->z_b_ref[k];
        const bool oc = w > 0 && !gr;
        const double wc = w > 0 ? w : 0.0, H = h->H_ice_ref[k];
        mgr0[k] = gr;
        moc0[k] = oc;
        hw0[k] = (H <= 1 ? wc : 0.0) + ((!gr && H > 1) ? wc - H * (c.rho_ice / c.rho_seawater) : 0.0);
        saf += h->H_af_ref[k] * h->dx * h->dy;
        sden += H * h->dx * h->dy;
        spov += wc * h->dx * h->dy;
    }
    std::vector<double> u0 = h->u_set ? h->u_init : h->u_ref;
    Ctl& ct = h->ctl;
    memset(&ct, 0, sizeof(Ctl));
    ct.t = c.t0; ct.t0 = c.t0; ct.t1 = c.t1;
    ct.dtmax = c.t1 - c.t0;
    ct.dtmin = ulp_above(fabs(c.t0) > fabs(c.t1) ? c.t0 : c.t1);
    ct.reltol = c.reltol; ct.abstol = c.abstol;
    ct.qold = QOLDINIT; ct.q11 = 1.0; ct.EEst = 1.0;
    ct.max_steps = c.max_steps;
    ct.active = 1;
    ct.t_stop = c.t1;
    ct.z_bsl = c.z_bsl;
    ct.A_bsl = c.bsl_ref_A;
    ct.V_af = c.volume_contribution == FI_CONTRIB_GOELZER ? saf * c.rho_ice / c.rho_seawater : 0.0;
    ct.V_den = c.density_contribution == FI_CONTRIB_GOELZER
                   ? sden * (c.rho_ice / c.rho_water - c.rho_ice / c.rho_seawater) : 0.0;
    ct.V_pov = c.adjustment_contribution == FI_CONTRIB_GOELZER ? spov : 0.0;
    if (c.form == FI_FORM_FP32) {
        const int K = (int)h->ice_t.size();
        Member& m = h->mem;
        m.dx = h->dx; m.dy = h->dy; m.A = h->dx * h->dy;
        m.g = c.g; m.rho_ice = c.rho_ice; m.rho_litho = c.rho_litho; m.rho_um = c.rho_uppermantle;
        m.nu = c.litho_poissonratio; m.rho_sw_ice = rsi; m.spy = c.seconds_per_year;
        m.border_v = c.bc_viscous_border; m.border_e = c.bc_elastic_border; m.border_g = c.bc_sea_surface_border;
        m.dt_sparse = c.dt_sparse_diagnostics;
        m.elastic_on = elastic; m.geoid_on = geoid;
        m.column_compressible = c.lithosphere_column == FI_COLUMN_COMPRESSIBLE;
        m.ice_external = c.ice_mode == FI_ICE_EXTERNAL;
        m.ice_flat = c.ice_flat_bc;
        m.sl_interactive = c.sealevel_load == FI_SEALEVEL_LOAD_INTERACTIVE;
        m.bsl_imposed = bsl_internal && c.bsl_mode == FI_BSL_IMPOSED;
        m.bsl_ref_z = c.z_bsl;
        m.rho_sw = c.rho_seawater;
        if (m.bsl_imposed) {
            double *bt, *bz;
            RET(dalloc(h, &bt, h->bslh_t.size()));
            RET(dalloc(h, &bz, h->bslh_z.size()));
            RET(upload(h, bt, h->bslh_t));
            RET(upload(h, bz, h->bslh_z));
            m.bslh_t = bt;
            m.bslh_z = bz;
            m.n_bslh = (int)h->bslh_t.size();
        }
        RET(upload(h, m.mgr, mgr0));
        RET(upload(h, m.moc, moc0));
        RET(upload(h, m.hwater, hw0));
        // FP32 parameter maps
        std::vector<double> vf(n), sigref(n), zbss(n);
        bool any_mask = false, any_haf = false, any_sig = false, any_ueref = false, zb_uniform = true;
        for (size_t k = 0; k < n; k++) {
            vf[k] = 1.0 / (2.0 * h->eta[k]);  // K / (2 eta), K == 1
            sigref[k] = h->mask[k] * (c.rho_ice * h->H_af_ref[k] + c.rho_litho * h->ue_ref[k] +
                                      c.rho_uppermantle * h->u_ref[k]);
            zbss[k] = h->z_b_ref[k] - h->z_ss_ref[k] - c.z_bsl;
            any_mask |= h->mask[k] != 1.0;
            any_haf |= h->H_af_ref[k] != 0.0;
            any_sig |= sigref[k] != 0.0;
            any_ueref |= h->ue_ref[k] != 0.0;
            zb_uniform &= zbss[k] == zbss[0];
        }
        m.flags = (any_mask ? FLAG_MASK : 0) | (any_haf ? FLAG_HAFREF : 0) | (any_sig ? FLAG_SIGREF : 0) |
                  (zb_uniform ? 0 : FLAG_ZBSS) | (any_ueref ? FLAG_UEREF : 0);
        m.zbss_scalar = (float)zbss[0];
        m.ncols = h->n_cols;
        m.h_rows = h->h_rows; m.B_cols = h->B_cols; m.h_conv = h->h_conv; m.B_conv = h->B_conv;
        m.n_rows = h->n_rows; m.n_crow = h->n_crow; m.n_ccol = h->n_ccol; m.n_crowi = h->n_crowi;
        RET(plan_layouts(h, K));
        RET(upload(h, (float*)m.D, h->D));
        RET(upload(h, (float*)m.visc_fac, vf));
        RET(upload(h, (float*)m.mask, h->mask));
        RET(upload(h, (float*)m.H_af_ref, h->H_af_ref));
        RET(upload(h, (float*)m.sigma_ref, sigref));
        RET(upload(h, (float*)m.zbss_ref, zbss));
        RET(upload(h, (float*)m.ue_ref, h->ue_ref));
        RET(upload(h, m.ue[0], h->ue_ref));
        if (!m.ice_external) {
            m.K = (int)h->ice_t.size();
            double* tt;
            float* Ht;
            RET(dalloc(h, &tt, m.K));
            RET(dalloc(h, &Ht, (size_t)m.K * n));
            RET(upload(h, tt, h->ice_t));
            RET(upload(h, Ht, h->ice_H));
            m.t_ice = tt;
            m.H_tab = Ht;
        }
        RET(upload(h, m.u[0], u0));
        if (elastic) RET(build_kernel_spectrum(h, h->d_Ge, (float2*)m.GA, nullptr));
        if (geoid) RET(build_kernel_spectrum(h, h->d_Gg, (float2*)m.GB, nullptr));
        for (int q = 0; q < 4; q++) {
            ct.ue_corner[0][q] = ct.ue_corner[1][q] = c.bc_elastic_border;
            ct.dz_corner[q] = c.bc_sea_surface_border;
        }
        CK(cudaMemcpyAsync(h->d_mem, &m, sizeof(Member), cudaMemcpyHostToDevice, h->stream));
        RET(write_ctl(h));
        // init_problem!: first update_diagnostics! at t0 (forces the sparse update), u <- BC(u)
        ct.t_call = c.t0;
        RET(write_ctl(h));
        RET(rhs_fused(h, 1, nullptr, nullptr, nullptr));
        CK(cudaMemcpyAsync(m.u[0], m.u[1], n * 8, cudaMemcpyDeviceToDevice, h->stream));
        RET(read_ctl(h));
        if (h->ctl.status) return set_err(h, h->ctl.status, "init_problem!: %s", fi_status_string(h->ctl.status));
    } else {
        PlainBufs& p = h->p;
        RET(upload(h, p.D, h->D));
        RET(upload(h, p.eta, h->eta));
        RET(upload(h, p.mask, h->mask));
        RET(upload(h, p.u_ref, h->u_ref));
        RET(upload(h, p.ue_ref, h->ue_ref));
        RET(upload(h, p.z_b_ref, h->z_b_ref));
        RET(upload(h, p.z_ss_ref, h->z_ss_ref));
        RET(upload(h, p.H_af_ref, h->H_af_ref));
        if (c.ice_mode == FI_ICE_TIME_INTERPOLATED) {
            RET(dalloc(h, &p.H_tab, h->ice_H.size()));
            RET(upload(h, p.H_tab, h->ice_H));
        }
        // CurrentState(domain, ref, z_bsl)
        RET(upload(h, p.u[0], u0));
        RET(upload(h, p.ue, h->ue_ref));
        RET(upload(h, p.H, h->H_ice_ref));
        RET(upload(h, p.H_af, h->H_af_ref));
        RET(upload(h, p.z_b, h->z_b_ref));
        RET(upload(h, p.z_ss, h->z_ss_ref));
        RET(upload(h, p.mgr, mgr0));
        RET(upload(h, p.moc, moc0));
        RET(upload(h, p.hwater, hw0));
        RET(upload(h, p.tau, h->tau));
        if (c.mantle == FI_MANTLE_RELAXED) {
            double* d_Gv = nullptr;
            RET(dalloc(h, &d_Gv, n));
            RET(dalloc(h, &p.Gv_hat, (size_t)h->Mx * h->My));
            RET(upload(h, d_Gv, viscous_green(h)));
            RET(build_kernel_spectrum(h, d_Gv, nullptr, p.Gv_hat));
        }
        if (elastic) RET(build_kernel_spectrum(h, h->d_Ge, nullptr, p.Ge_hat));
        if (geoid) RET(build_kernel_spectrum(h, h->d_Gg, nullptr, p.Gg_hat));
        RET(rhs_plain(h, c.t0, p.u[0], p.fscratch));
    }
    CK(cudaStreamSynchronize(h->stream));
    h->initialized = true;
    h->last_call = 0;
    return FI_OK;
}

// ---------------------------------------------------------------------------
// fused form: one host-driven right-hand side (stage 0: uin -> vout/cout;
// stage 1: state -> k1 slot), t taken from ctl.t_call
// ---------------------------------------------------------------------------
static int launch_sparse(fi_handle* h) {
    k_conv_rows<<<h->n_crow, ROW_THREADS, conv_rows_smem(h->Mx, h->h_conv), h->stream>>>(h->d_mem, h->t_crow,
                                                                                       h->h_conv);
    CKL();
    k_conv_cols<<<h->n_ccol, ROW_THREADS, conv_cols_smem(h->My, h->B_conv), h->stream>>>(h->d_mem, h->t_ccol,
                                                                                       h->B_conv);
    CKL();
    k_conv_rows_inv<<<h->n_crowi, ROW_THREADS, conv_rows_smem(h->Mx, h->h_conv), h->stream>>>(
        h->d_mem, h->t_crowi, h->h_conv);
    CKL();
    return FI_OK;
}

// One host-driven right-hand side body (stage 0/1) or one graph-free BS3 stage
// (stages 2-4, fallback loop): forward rows, columns, and for stages 0/1/4 the
// inverse rows.
static int launch_rhs_body(fi_handle* h, int stage, const double* uin, float* vout, double* cout,
                           cudaGraphConditionalHandle hg, cudaGraphConditionalHandle hw) {
    const int inv = (stage == 3 || stage == 4) ? 1 : 0;
    k_rows_fwd<<<h->n_rows, ROW_THREADS, rows_fwd_smem(h->mem.fl.bytes, h->nx, (int)h->ice_t.size()), h->stream>>>(
        h->d_mem, h->t_rows, stage, h->h_rows, uin, inv);
    CKL();
    const int next = (stage == 2 || stage == 3) ? stage + 1 : 0;
    k_cols<<<h->n_cols, ROW_THREADS, cols_smem(h->ny, h->B_cols), h->stream>>>(h->d_mem, h->t_cols, h->B_cols, next, 0);
    CKL();
    if (stage <= 1 || stage == 4) {
        k_rows_inv<<<h->n_rows, ROW_THREADS, rows_inv_smem(h->nx, h->h_rows, h->n_cols), h->stream>>>(
            h->d_mem, h->t_rows, stage, h->h_rows, vout, cout, hg, hw);
        CKL();
    }
    return FI_OK;
}

static int rhs_fused(fi_handle* h, int stage, const double* uin, float* vout, double* cout) {
    k_gate<<<1, 32, 0, h->stream>>>(h->d_mem, 1, h->ctl.t_call, 0);
    CKL();
    RET(launch_sparse(h));
    RET(launch_rhs_body(h, stage, uin, vout, cout, 0, 0));
    return FI_OK;
}

extern "C" int fi_rhs(fi_handle* h, double t, double* u_inout, double* dudt_out) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !u_inout || !dudt_out) return FI_ERR_ARG;
    if (!h->initialized) return set_err(h, FI_ERR_STATE, "fi_init not called");
    const size_t n = N2(h);
    if (h->cfg.form == FI_FORM_FP32) {
        RET(read_ctl(h));
        h->ctl.t_call = t;
        h->ctl.status = FI_OK;
        RET(write_ctl(h));
        CK(cudaMemcpyAsync(h->d_uin, u_inout, n * 8, cudaMemcpyHostToDevice, h->stream));
        RET(rhs_fused(h, 0, h->d_uin, h->d_vscr, h->d_cscr));
        RET(read_ctl(h));
        if (h->ctl.status) return set_err(h, h->ctl.status, "%s", fi_status_string(h->ctl.status));
        std::vector<float> v(n);
        double cc[4];
        CK(cudaMemcpyAsync(u_inout, h->mem.u[h->ctl.ibuf ^ 1], n * 8, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(v.data(), h->d_vscr, n * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(cc, h->d_cscr, 32, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        const double off = corner_mean(cc) - h->cfg.bc_viscous_border;
        for (size_t k = 0; k < n; k++) dudt_out[k] = (double)v[k] - off;
    } else {
        CK(cudaMemcpyAsync(h->p.uin, u_inout, n * 8, cudaMemcpyHostToDevice, h->stream));
        RET(rhs_plain(h, t, h->p.uin, h->p.fscratch));
        CK(cudaMemcpyAsync(u_inout, h->p.uin, n * 8, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(dudt_out, h->p.fscratch, n * 8, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    h->last_call = 1;
    h->last_rhs_t = t;
    return FI_OK;
}

static_assert((size_t)FI_NOALLOC_MAX_CELLS == NOALLOC_MAX_CELLS, "scratch limit mismatch");

// fi_rhs on device buffers with the result scratch in a static device array
// (fi_noalloc.cu): no device or host allocation on the success path.
extern "C" int fi_rhs_noalloc(fi_handle* h, double t, double* u_dev, double* dudt_dev) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !u_dev || !dudt_dev) return FI_ERR_ARG;
    const size_t n = N2(h);
    if (n > NOALLOC_MAX_CELLS)
        return set_err(h, FI_ERR_ARG, "fi_rhs_noalloc: grid of %zu cells exceeds the static scratch limit of %zu cells",
                       n, NOALLOC_MAX_CELLS);
    if (h->cfg.form != FI_FORM_FP32) return set_err(h, FI_ERR_ARG, "fi_rhs_noalloc serves the FP32 form only");
    if (!h->initialized) return set_err(h, FI_ERR_STATE, "fi_init not called");
    void* scr = nullptr;
    CK(noalloc_scratch(&scr));
    RET(read_ctl(h));
    h->ctl.t_call = t;
    h->ctl.status = FI_OK;
    RET(write_ctl(h));
    RET(rhs_fused(h, 0, u_dev, (float*)scr, (double*)((unsigned char*)scr + NOALLOC_CORNER_OFFSET)));
    RET(read_ctl(h));
    if (h->ctl.status) return set_err(h, h->ctl.status, "%s", fi_status_string(h->ctl.status));
    CK(cudaMemcpyAsync(u_dev, h->mem.u[h->ctl.ibuf ^ 1], n * 8, cudaMemcpyDeviceToDevice, h->stream));
    CK(noalloc_finish(scr, h->cfg.bc_viscous_border, n, dudt_dev, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->last_call = 1;
    h->last_rhs_t = t;
    return FI_OK;
}

// ---------------------------------------------------------------------------
// plain FP64 form
// ---------------------------------------------------------------------------
static inline int gs(size_t n) { return std::max(1, std::min(4096, cdiv((long long)n, NT))); }

static int corner_bc_plain(fi_handle* h, double* X, int nx, int ny, double border) {
    kp_corner_off<<<1, 32, 0, h->stream>>>(X, nx, ny, border, h->p.off);
    CKL();
    kp_sub_off<<<gs((size_t)nx * ny), NT, 0, h->stream>>>(X, (size_t)nx * ny, h->p.off);
    CKL();
    return FI_OK;
}

static int conv_plain(fi_handle* h, const double* input, const double2* Ghat, double border, double* output,
                      bool regular = false) {
    const size_t M = (size_t)h->Mx * h->My;
    const int cx = 2 * h->nx - 1, cy = 2 * h->ny - 1;
    PlainBufs& p = h->p;
    k_pad_real<<<cdiv(M, NT), NT, 0, h->stream>>>(input, h->nx, h->ny, p.P, h->Mx, h->My);
    CKL();
    RET(fft2_64(h, p.P, h->Mx, h->My, 0));
    kp_cmul<<<gs(M), NT, 0, h->stream>>>(p.P, Ghat, M);
    CKL();
    RET(fft2_64(h, p.P, h->Mx, h->My, 1));
    kp_crop<<<gs((size_t)cx * cy), NT, 0, h->stream>>>(p.P, h->Mx, cx, cy, p.cropped);
    CKL();
    // samesize_conv! (src/convolutions.jl:134-154): the extended BC space corrects the
    // (2nx-1) x (2ny-1) result before the crop, the regular one the cropped field
    if (!regular) RET(corner_bc_plain(h, p.cropped, cx, cy, border));
    kp_window<<<gs(N2(h)), NT, 0, h->stream>>>(p.cropped, cx, h->i1, h->j1, h->nx, h->ny, output);
    CKL();
    if (regular) RET(corner_bc_plain(h, output, h->nx, h->ny, border));
    return FI_OK;
}

// update_diagnostics!(dudt, u, sim, t), one kernel per broadcast of the reference
static int reduce_host(fi_handle* h, const double* d_partial, int nblk, int stride, double* out);

static int rhs_plain(fi_handle* h, double t, double* u, double* dudt) {
    const fi_config& c = h->cfg;
    PlainBufs& p = h->p;
    const size_t n = N2(h);
    const int nx = h->nx, ny = h->ny;
    const int g = gs(n);
    h->nf_plain += 1;
    RET(corner_bc_plain(h, u, nx, ny, c.bc_viscous_border));
    kp_bedrock<<<g, NT, 0, h->stream>>>(u, p.ue, p.z_b_ref, p.u_ref, p.now_u, p.z_b, p.s_m, c.rho_uppermantle, n);
    CKL();
    if (c.ice_mode == FI_ICE_TIME_INTERPOLATED) {
        const std::vector<double>& tt = h->ice_t;
        const int K = (int)tt.size();
        int i = 0, exact = 1;
        double dti = 1.0, ts = 0.0;
        if (t < tt[0] || t > tt[K - 1]) {
            if (!c.ice_flat_bc) return set_err(h, FI_ERR_FORCING_RANGE, "TimeInterpolation2D out of range.");
            i = t < tt[0] ? 0 : K - 1;
        } else {
            i = (int)(std::lower_bound(tt.begin(), tt.end(), t) - tt.begin());
            if (tt[i] != t) {
                i -= 1;
                exact = 0;
                dti = tt[i + 1] - tt[i];
                ts = t - tt[i];
            }
        }
        const double* Ha = p.H_tab + (size_t)i * n;
        const double* Hb = exact ? Ha : Ha + n;
        kp_ice<<<g, NT, 0, h->stream>>>(Ha, Hb, dti, ts, exact, p.H, n);
        CKL();
    }
    const double rsi = c.rho_seawater / c.rho_ice;
    kp_haf_ice<<<g, NT, 0, h->stream>>>(p.H, p.z_b, p.z_ss, p.H_af_ref, p.H_af, p.s_i, rsi, c.rho_ice, n);
    CKL();
    if (((t - c.t0) / c.dt_sparse_diagnostics) >= (double)h->ctl.count_sparse) {
        if (c.lithosphere == FI_LITHO_RIGID) {
            kp_zero<<<g, NT, 0, h->stream>>>(p.ue, n);
            CKL();
        } else {
            kp_copy<<<g, NT, 0, h->stream>>>(p.buf, p.s_load, n);  // columnanoms.load * K^2
            CKL();
            RET(conv_plain(h, p.buf, p.Ge_hat, c.bc_elastic_border, p.ue));
        }
        kp_litho<<<g, NT, 0, h->stream>>>(p.ue, p.ue_ref, p.s_l, c.rho_litho, n);
        CKL();
        {
            // internal_update_bsl! (src/sealevel.jl:242-262): the volumes on the first
            // H_af of this call, the old z_ss and the current z_b, then update_bsl!
            Ctl& ct = h->ctl;
            kp_volumes<<<h->red_blocks, NT, 0, h->stream>>>(p.H_af, p.H, p.z_ss, p.z_b, h->dx * h->dy, p.partial, n);
            CKL();
            double v3[3] = {0.0, 0.0, 0.0};
            RET(reduce_host(h, p.partial, h->red_blocks, 3, v3));
            const double Vold = ct.V_af + ct.V_den + ct.V_pov;
            ct.V_af = c.volume_contribution == FI_CONTRIB_GOELZER ? v3[0] * c.rho_ice / c.rho_seawater : 0.0;
            ct.V_den = c.density_contribution == FI_CONTRIB_GOELZER
                           ? v3[1] * (c.rho_ice / c.rho_water - c.rho_ice / c.rho_seawater) : 0.0;
            ct.V_pov = c.adjustment_contribution == FI_CONTRIB_GOELZER ? v3[2] : 0.0;
            ct.delta_V = (ct.V_af + ct.V_den + ct.V_pov) - Vold;
            if (c.bsl_update == FI_BSL_UPDATE_INTERNAL) {
                const int st = bsl_update(&ct, c.bsl_mode, c.z_bsl, c.bsl_ref_A, -ct.delta_V, t, h->osurf_z.data(),
                                          h->osurf_A.data(), (int)h->osurf_z.size(), h->bslh_t.data(),
                                          h->bslh_z.data(), (int)h->bslh_t.size());
                if (st) return set_err(h, st, "update_bsl!: BSL %.6g or t = %.6g outside its table", ct.z_bsl, t);
            }
        }
        if (c.sea_surface == FI_SEA_SURFACE_LATERALLY_VARIABLE) {
            kp_geo_in<<<g, NT, 0, h->stream>>>(p.s_load, p.s_full, p.s_m, p.mask,
                                              c.lithosphere_column == FI_COLUMN_COMPRESSIBLE, h->dx * h->dy, p.buf, n);
            CKL();
            RET(conv_plain(h, p.buf, p.Gg_hat, c.bc_sea_surface_border, p.dz));
        }
        kp_zss<<<g, NT, 0, h->stream>>>(p.z_ss_ref, p.dz, h->ctl.z_bsl, p.z_ss, n);
        CKL();
        kp_haf_ice<<<g, NT, 0, h->stream>>>(p.H, p.z_b, p.z_ss, p.H_af_ref, p.H_af, p.s_i, rsi, c.rho_ice, n);
        CKL();
        kp_sealevel<<<g, NT, 0, h->stream>>>(p.H, p.H_af, p.z_ss, p.z_b, p.z_ss_ref, p.mask,
                                             c.sealevel_load == FI_SEALEVEL_LOAD_INTERACTIVE, c.rho_seawater,
                                             c.rho_ice / c.rho_seawater, p.mgr, p.moc, p.hwater, p.s_sw, n);
        CKL();
        h->ctl.count_sparse += 1;
    }
    kp_load_full<<<g, NT, 0, h->stream>>>(p.s_i, p.s_sw, p.s_l, p.s_m, p.mask, p.s_load, p.s_full, n);
    CKL();
    // update_dudt!(dudt, u, sim, t, mantle, lithosphere), src/deformation.jl:21-103
    if (c.mantle == FI_MANTLE_RIGID) {
        kp_zero<<<g, NT, 0, h->stream>>>(dudt, n);
        kp_copy<<<g, NT, 0, h->stream>>>(p.dudt, dudt, n);
        CKL();
        return FI_OK;
    }
    if (c.mantle == FI_MANTLE_RELAXED) {
        kp_elra_in<<<g, NT, 0, h->stream>>>(p.s_load, p.s_l, c.g, p.buf, n);
        CKL();
        RET(conv_plain(h, p.buf, p.Gv_hat, c.bc_viscous_border, p.u_eq, true));
        kp_elra_dudt<<<g, NT, 0, h->stream>>>(p.u_eq, p.now_u, p.tau, dudt, n);
        kp_copy<<<g, NT, 0, h->stream>>>(p.dudt, dudt, n);
        CKL();
        return FI_OK;
    }
    if (c.lithosphere == FI_LITHO_LATERALLY_CONSTANT) {
        // one step of dt_min written into u in place; dudt is left as it is
        kp_lc_in<<<g, NT, 0, h->stream>>>(p.s_load, p.s_l, c.g, u, p.fftrhs, p.fftU, n);
        CKL();
        RET(fft2_64(h, p.fftrhs, nx, ny, 0));
        RET(fft2_64(h, p.fftU, nx, ny, 0));
        kp_lc_step<<<g, NT, 0, h->stream>>>(p.fftU, p.fftrhs, p.eta, h->d_pd, h->d_R, p.D,
                                            c.rho_uppermantle * c.g, c.dt_min * c.seconds_per_year, n);
        CKL();
        RET(fft2_64(h, p.fftU, nx, ny, 1));
        kp_real<<<g, NT, 0, h->stream>>>(p.fftU, u, n);
        CKL();
        RET(corner_bc_plain(h, u, nx, ny, c.bc_viscous_border));
        kp_copy<<<g, NT, 0, h->stream>>>(p.now_u, u, n);
        kp_copy<<<g, NT, 0, h->stream>>>(p.dudt, dudt, n);
        CKL();
        return FI_OK;
    }
    kp_rhs_init<<<g, NT, 0, h->stream>>>(p.s_full, c.g, p.rhs, n);
    CKL();
    kp_dxx<<<g, NT, 0, h->stream>>>(p.bxx, u, nx, ny, h->dx);
    kp_dyy<<<g, NT, 0, h->stream>>>(p.byy, u, nx, ny, h->dy);
    kp_dx<<<g, NT, 0, h->stream>>>(p.bx, u, nx, ny, h->dx);
    kp_dy<<<g, NT, 0, h->stream>>>(p.bxy, p.bx, nx, ny, h->dy);
    CKL();
    kp_moments<<<g, NT, 0, h->stream>>>(p.bxx, p.byy, p.bxy, p.D, c.litho_poissonratio, p.Mxx, p.Myy, p.Mxy, n);
    CKL();
    kp_dxx<<<g, NT, 0, h->stream>>>(p.bxx, p.Mxx, nx, ny, h->dx);
    kp_dyy<<<g, NT, 0, h->stream>>>(p.byy, p.Myy, nx, ny, h->dy);
    kp_dx<<<g, NT, 0, h->stream>>>(p.bx, p.Mxy, nx, ny, h->dx);
    kp_dy<<<g, NT, 0, h->stream>>>(p.bxy, p.bx, nx, ny, h->dy);
    CKL();
    kp_rhs_acc<<<g, NT, 0, h->stream>>>(p.rhs, p.bxx, p.byy, p.bxy, n);
    kp_fftin<<<g, NT, 0, h->stream>>>(p.rhs, p.eta, p.fftrhs, n);
    CKL();
    RET(fft2_64(h, p.fftrhs, nx, ny, 0));
    kp_spec<<<g, NT, 0, h->stream>>>(p.fftrhs, h->d_spinv, n);
    CKL();
    RET(fft2_64(h, p.fftrhs, nx, ny, 1));
    kp_real_spy<<<g, NT, 0, h->stream>>>(p.fftrhs, c.seconds_per_year, dudt, n);
    CKL();
    RET(corner_bc_plain(h, dudt, nx, ny, c.bc_viscous_border));
    kp_copy<<<g, NT, 0, h->stream>>>(p.dudt, dudt, n);
    CKL();
    return FI_OK;
}

static int reduce_host(fi_handle* h, const double* d_partial, int nblk, int stride, double* out) {
    std::vector<double> v((size_t)nblk * stride);
    CK(cudaMemcpyAsync(v.data(), d_partial, v.size() * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int s = 0; s < stride; s++) {
        double acc = 0.0;
        for (int b = 0; b < nblk; b++) acc += v[(size_t)b * stride + s];
        out[s] = acc;
    }
    return FI_OK;
}

// ---------------------------------------------------------------------------
// integrator start (OrdinaryDiffEq __init: FSAL preamble, ode_determine_initdt)
// ---------------------------------------------------------------------------
static int integ_start(fi_handle* h) {
    const fi_config& c = h->cfg;
    const size_t n = N2(h);
    const double nd = (double)n;
    Ctl& ct = h->ctl;
    double d0, d1, d2 = 0.0, eqsum = 0.0;
    double dt0;
    const int nb = h->red_blocks;
    if (c.form == FI_FORM_FP32) {
        RET(read_ctl(h));
        ct.t_call = ct.t;
        RET(write_ctl(h));
        // initialize!: fsalfirst = f(uprev, t)
        RET(rhs_fused(h, 1, nullptr, nullptr, nullptr));
        // f0 = f(u0, t) into the k4 slot
        RET(read_ctl(h));
        const int ik = h->ctl.ik;
        float* f0 = h->mem.k14[ik ^ 1];
        double* c0 = &h->d_ctl->kcorner[ik ^ 1][0];
        RET(rhs_fused(h, 0, h->mem.u[h->ctl.ibuf], f0, c0));
        kf_initdt_norms<<<nb, NT, 0, h->stream>>>(h->mem.u[h->ctl.ibuf], f0, c0, c.bc_viscous_border, c.abstol,
                                                  c.reltol, h->d_red, n);
        CKL();
        double s[2] = {0.0, 0.0};
        RET(reduce_host(h, h->d_red, nb, 2, s));
        d0 = sqrt(s[0] / nd);
        d1 = sqrt(s[1] / nd);
        dt0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : (d0 / d1) / 100;
        if (dt0 > ct.dtmax) dt0 = ct.dtmax;
        if (!(dt0 < 10 * 2.220446049250313e-16)) {
            kf_initdt_u1<<<gs(n), NT, 0, h->stream>>>(h->d_uin, h->mem.u[h->ctl.ibuf], f0, c0, c.bc_viscous_border,
                                                      dt0, n);
            CKL();
            RET(read_ctl(h));
            h->ctl.t_call = ct.t + dt0;
            RET(write_ctl(h));
            RET(rhs_fused(h, 0, h->d_uin, h->d_vscr, h->d_cscr));
            kf_initdt_d2<<<nb, NT, 0, h->stream>>>(h->mem.u[h->ctl.ibuf], f0, c0, h->d_vscr, h->d_cscr,
                                                   c.bc_viscous_border, c.abstol, c.reltol, h->d_red, n);
            CKL();
            RET(reduce_host(h, h->d_red, nb, 2, s));
            d2 = sqrt(s[0] / nd) / dt0;
            eqsum = s[1];
        }
        RET(read_ctl(h));
        if (h->ctl.status) return set_err(h, h->ctl.status, "%s", fi_status_string(h->ctl.status));
    } else if (c.alg == FI_ALG_EULER) {
        // solve(prob, Euler(); dt = dt_min, ...): fsalfirst = f(uprev, t), no initial-dt search
        RET(rhs_plain(h, ct.t, h->p.u[ct.ibuf], h->p.k14[ct.ik]));
        h->ctl.dt = c.dt_min;
        h->ctl.dtpropose = c.dt_min;
        h->ctl.iter = 0;
        h->ctl.kout = 0;
        h->fsal_pending = false;
        h->integ_started = true;
        return FI_OK;
    } else {
        PlainBufs& p = h->p;
        RET(rhs_plain(h, ct.t, p.u[ct.ibuf], p.k14[ct.ik]));  // fsalfirst = f(uprev, t)
        // f0 = f(u, t): the integrator's u is a separate copy of u0; sk uses u0 (already
        // boundary-corrected, so uprev holds the same values)
        CK(cudaMemcpyAsync(p.tmp, p.u[ct.ibuf], n * 8, cudaMemcpyDeviceToDevice, h->stream));
        RET(rhs_plain(h, ct.t, p.tmp, p.k14[ct.ik ^ 1]));
        kp_norms2<<<nb, NT, 0, h->stream>>>(p.tmp, p.k14[ct.ik ^ 1], p.u[ct.ibuf], c.abstol, c.reltol, p.partial, n);
        CKL();
        double s[2] = {0.0, 0.0};
        RET(reduce_host(h, p.partial, nb, 2, s));
        d0 = sqrt(s[0] / nd);
        d1 = sqrt(s[1] / nd);
        dt0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : (d0 / d1) / 100;
        if (dt0 > ct.dtmax) dt0 = ct.dtmax;
        if (!(dt0 < 10 * 2.220446049250313e-16)) {
            kp_stage<<<gs(n), NT, 0, h->stream>>>(p.uin, p.tmp, dt0, p.k14[ct.ik ^ 1], n);
            CKL();
            RET(rhs_plain(h, ct.t + dt0, p.uin, p.fscratch));
            kp_initdt_terms<<<nb, NT, 0, h->stream>>>(p.k14[ct.ik ^ 1], p.fscratch, p.u[ct.ibuf], c.abstol,
                                                      c.reltol, p.partial, n);
            CKL();
            RET(reduce_host(h, p.partial, nb, 2, s));
            d2 = sqrt(s[0] / nd) / dt0;
            eqsum = s[1];
        }
    }
    double dt;
    if (dt0 < 10 * 2.220446049250313e-16) {
        dt = std::max(1e-6, ct.dtmin);
    } else if (eqsum == (double)nb * NT) {
        dt = std::max(ct.dtmin, 100 * dt0);
    } else {
        const double mx = std::max(d1, d2);
        const double dt1 = (mx <= 1e-15) ? std::max(1e-6, dt0 * 1e-3) : pow(10.0, -(2 + log10(mx)) / 3.0);
        dt = std::max(ct.dtmin, std::min(std::min(100 * dt0, dt1), ct.dtmax));
    }
    if (c.form == FI_FORM_FP32) RET(read_ctl(h));
    h->ctl.dt = dt;
    h->ctl.dtpropose = dt;
    h->ctl.iter = 0;
    h->ctl.kout = 0;
    h->fsal_pending = false;
    if (c.form == FI_FORM_FP32) RET(write_ctl(h));
    h->integ_started = true;
    return FI_OK;
}

// ---------------------------------------------------------------------------
// fused form: segment runner (CUDA graph, fallback host loop)
// ---------------------------------------------------------------------------
static int add_kernel(fi_handle* h, cudaGraph_t g, cudaGraphNode_t* prev, void* func, int grid, size_t smem,
                      void** args) {
    cudaKernelNodeParams kp{};
    kp.func = func;
    kp.gridDim = dim3(grid);
    kp.blockDim = dim3(ROW_THREADS);
    kp.sharedMemBytes = (unsigned)smem;
    kp.kernelParams = args;
    cudaGraphNode_t node;
    CK(cudaGraphAddKernelNode(&node, g, *prev ? prev : nullptr, *prev ? 1 : 0, &kp));
    *prev = node;
    return FI_OK;
}

static int add_cond(fi_handle* h, cudaGraph_t g, cudaGraphNode_t* prev, cudaGraphConditionalHandle hc,
                    cudaGraphConditionalNodeType type, cudaGraph_t* body) {
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hc;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, *prev ? prev : nullptr, *prev ? 1 : 0, &cp));
    *body = cp.conditional.phGraph_out[0];
    *prev = node;
    return FI_OK;
}

static int add_sparse(fi_handle* h, cudaGraph_t g) {
    cudaGraphNode_t prev = nullptr;
    const Member* mp = h->d_mem;
    const Task *t1 = h->t_crow, *t2 = h->t_ccol, *t3 = h->t_crowi;
    int hc = h->h_conv, bc = h->B_conv;
    void* a1[] = {(void*)&mp, (void*)&t1, (void*)&hc};
    RET(add_kernel(h, g, &prev, (void*)k_conv_rows, h->n_crow, conv_rows_smem(h->Mx, hc), a1));
    void* a2[] = {(void*)&mp, (void*)&t2, (void*)&bc};
    RET(add_kernel(h, g, &prev, (void*)k_conv_cols, h->n_ccol, conv_cols_smem(h->My, bc), a2));
    void* a3[] = {(void*)&mp, (void*)&t3, (void*)&hc};
    RET(add_kernel(h, g, &prev, (void*)k_conv_rows_inv, h->n_crowi, conv_rows_smem(h->Mx, hc), a3));
    return FI_OK;
}

static int build_segment_graph(fi_handle* h) {
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    h->seg_graph = g;
    cudaGraphConditionalHandle hw, hg[3];
    CK(cudaGraphConditionalHandleCreate(&hw, g, 0, cudaGraphCondAssignDefault));
    for (int i = 0; i < 3; i++) CK(cudaGraphConditionalHandleCreate(&hg[i], g, 0, cudaGraphCondAssignDefault));
    const Member* mp = h->d_mem;
    int one = 1;
    cudaGraphNode_t prev = nullptr;
    {
        void* a[] = {(void*)&mp, (void*)&one, (void*)&hg[0], (void*)&hw};
        cudaKernelNodeParams kp{};
        kp.func = (void*)k_segment_start;
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(32);
        kp.kernelParams = a;
        CK(cudaGraphAddKernelNode(&prev, g, nullptr, 0, &kp));
    }
    cudaGraph_t body;
    RET(add_cond(h, g, &prev, hw, cudaGraphCondTypeWhile, &body));
    cudaGraphNode_t bp = nullptr;
    for (int s = 2; s <= 4; s++) {
        cudaGraph_t sb;
        RET(add_cond(h, body, &bp, hg[s - 2], cudaGraphCondTypeIf, &sb));
        RET(add_sparse(h, sb));
        const Task* tr = h->t_rows;
        const Task* tc = h->t_cols;
        int stage = s, hr = h->h_rows, bcol = h->B_cols, inv = (s > 2) ? 1 : 0;
        int next = (s < 4) ? s + 1 : 0;
        const double* uin = nullptr;
        float* vout = nullptr;
        double* cout = nullptr;
        cudaGraphConditionalHandle hnext = (s < 4) ? hg[s - 1] : 0;
        void* a1[] = {(void*)&mp, (void*)&tr, (void*)&stage, (void*)&hr, (void*)&uin, (void*)&inv};
        RET(add_kernel(h, body, &bp, (void*)k_rows_fwd, h->n_rows, rows_fwd_smem(h->mem.fl.bytes, h->nx, (int)h->ice_t.size()), a1));
        void* a2[] = {(void*)&mp, (void*)&tc, (void*)&bcol, (void*)&next, (void*)&hnext};
        RET(add_kernel(h, body, &bp, (void*)k_cols, h->n_cols, cols_smem(h->ny, bcol), a2));
        if (s == 4) {
            cudaGraphConditionalHandle hgate = hg[0], hloop = hw;
            void* a3[] = {(void*)&mp, (void*)&tr, (void*)&stage, (void*)&hr,
                          (void*)&vout, (void*)&cout, (void*)&hgate, (void*)&hloop};
            RET(add_kernel(h, body, &bp, (void*)k_rows_inv, h->n_rows, rows_inv_smem(h->nx, hr, h->n_cols), a3));
        }
    }
    CK(cudaGraphInstantiate(&h->seg_exec, g, 0));
    return FI_OK;
}

// Shared-memory budget of the row phases: the forward row staging layout is sized so
// that two persistent blocks fit on an SM (one if two cannot), then checked against the
// per-block limit of the per-phase kernels.
static int plan_layouts(fi_handle* h, int K) {
    Member& m = h->mem;
    int smem_sm = 0;
    CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, h->cfg.device));
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, persist_kernel(0, 0, 2)));
    const long long extra = (long long)(h->nx + h->ny) * (long long)sizeof(float2) + (K <= TICE_MAX ? 8LL * K : 0);
    const size_t others[] = {ws_cols(h->ny, h->B_cols), ws_rows_inv(h->nx, h->h_rows, h->n_cols),
                             ws_conv_rows(h->Mx, h->h_conv), ws_conv_cols(h->My, h->B_conv)};
    long long other_max = 0;
    for (size_t q : others) other_max = std::max(other_max, (long long)q);
    bool fits = false;
    for (int target = 2; target >= 1 && !fits; target--) {
        const long long budget = (long long)smem_sm / target - (long long)fa.sharedSizeBytes - 1024 - extra;
        if (budget <= 0) continue;
        fwd_layout(h->nx, h->h_rows, m.flags, h->n_cols, (size_t)budget, h->stage_inputs, &m.fl);
        fits = m.fl.bytes <= budget && other_max <= budget;
    }
    if (!fits) {
        fwd_layout(h->nx, h->h_rows, m.flags, h->n_cols, 0, 0, &m.fl);
        if (h->executor == EXEC_PERSIST) h->executor = EXEC_GRAPH;
    }
    const size_t need[] = {rows_fwd_smem(m.fl.bytes, h->nx, K), cols_smem(h->ny, h->B_cols),
                           rows_inv_smem(h->nx, h->h_rows, h->n_cols), conv_rows_smem(h->Mx, h->h_conv),
                           conv_cols_smem(h->My, h->B_conv)};
    for (size_t q : need)
        if (q + 1024 > h->smem_cap)
            return set_err(h, FI_ERR_ARG, "shared memory need %zu B exceeds the per-block limit", q);
    return setup_persist(h, K);
}

// Persistent executor set-up: shared-memory layout, grid = resident blocks (at most
// two per SM), cooperative launch support.  Falls back to the graph executor.
static int setup_persist(fi_handle* h, int K) {
    if (h->executor != EXEC_PERSIST) return FI_OK;
    PersistArgs& a = h->pargs;
    unsigned long long* trace = a.trace;
    a = PersistArgs{};
    a.trace = trace;
    a.mem = h->d_mem;
    a.bar = h->d_bar;
    a.h_rows = h->h_rows; a.B_cols = h->B_cols; a.h_conv = h->h_conv; a.B_conv = h->B_conv;
    a.n_rows = h->n_rows; a.n_cols = h->n_cols; a.n_crow = h->n_crow; a.n_ccol = h->n_ccol; a.n_crowi = h->n_crowi;
    const size_t smem = persist_layout(h->nx, h->ny, h->Mx, h->My, K, h->mem.fl.bytes, h->h_rows, h->n_cols, h->B_cols,
                                       h->h_conv, h->B_conv, &a);
    int coop = 0, nsm = 0, occ = 0;
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->cfg.device));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->cfg.device));
    const void* k2 = persist_kernel(0, 0, 2);
    const void* k1 = persist_kernel(0, 0, 1);
    cudaFuncAttributes fp{}, fp1{};
    CK(cudaFuncGetAttributes(&fp, k2));
    CK(cudaFuncGetAttributes(&fp1, k1));
    if (!coop || smem + std::max(fp.sharedSizeBytes, fp1.sharedSizeBytes) + 1024 > h->smem_optin) {
        h->executor = EXEC_GRAPH;
        return FI_OK;
    }
    // the 2-blocks-per-SM build where shared memory fits two blocks and the row or
    // column tasks outnumber the SMs, else the one sized for a single block (more
    // registers, no spills: with at most one task per SM a second block only adds barrier
    // arrivals); FI_PERSIST_MINB=1|2 forces one
    CK(cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k2, ROW_THREADS, smem));
    h->persist_minb = (occ >= 2 && std::max(h->n_rows, h->n_cols) > nsm) ? 2 : 1;
    const char* mb = getenv("FI_PERSIST_MINB");
    if (mb && (mb[0] == '1' || mb[0] == '2')) h->persist_minb = mb[0] - '0';
    if (h->persist_minb == 1) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k1, ROW_THREADS, smem));
        occ = std::min(occ, 1);
    }
    if (occ < 1) {
        h->executor = EXEC_GRAPH;
        return FI_OK;
    }
    h->persist_grid = nsm * std::min(occ, 2);
    h->persist_smem = smem;
    return FI_OK;
}

// Wait bounds of the device waits (fi_debug_set_wait_limit): negative = the default.
static std::atomic<long long> g_grid_polls{-1};
static std::atomic<long long> g_grid_extra{0};

// The persistent kernel for the member's current row and column plans: the build with
// their radix sequences compiled in where there is one (the schedules can change after
// set-up, so this is chosen at every launch); FI_PERSIST_SEQ=0 forces the runtime passes.
static int persist_fn(fi_handle* h, const void** out) {
    int sx = 0, sy = 0;
    const char* e = getenv("FI_PERSIST_SEQ");
    if (!(e && e[0] == '0')) {
        const Plan& px = h->plans[h->plan_x];
        const Plan& py = h->plans[h->plan_y];
        sx = seq_code(px.radix, px.npass);
        sy = seq_code(py.radix, py.npass);
    }
    const void* f = persist_kernel(sx, sy, h->persist_minb);
    if (f != persist_kernel(0, 0, h->persist_minb))
        CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->persist_smem));
    *out = f;
    return FI_OK;
}

static int run_segment_persist(fi_handle* h) {
    const void* kfn = nullptr;
    RET(persist_fn(h, &kfn));
    CK(cudaMemsetAsync(h->d_bar, 0, 4 * sizeof(unsigned int), h->stream));
    const long long gp = g_grid_polls.load();
    h->pargs.polls = gp >= 0 ? gp : PERSIST_SPIN_LIMIT;
    h->pargs.bar_extra = (unsigned)g_grid_extra.load();
    void* args[] = {(void*)&h->pargs};
    CK(cudaLaunchCooperativeKernel(kfn, dim3(h->persist_grid), dim3(ROW_THREADS), args,
                                   h->persist_smem, h->stream));
    unsigned int bar[4];
    CK(cudaMemcpyAsync(bar, h->d_bar, sizeof(bar), cudaMemcpyDeviceToHost, h->stream));
    RET(read_ctl(h));
    if (bar[2]) return set_err(h, FI_ERR_TIMEOUT, "persistent step kernel: a grid barrier wait gave up");
    return FI_OK;
}

// Launches one segment of the graph executor without waiting (the ensemble driver
// overlaps the members' segments on their streams).
static int launch_segment_graph_async(fi_handle* h) {
    if (!h->seg_exec) RET(build_segment_graph(h));
    CK(cudaGraphLaunch(h->seg_exec, h->stream));
    return FI_OK;
}

static int run_segment_fused(fi_handle* h) {
    if (h->executor == EXEC_PERSIST) return run_segment_persist(h);
    if (h->graph_ok && !h->seg_exec) {
        if (build_segment_graph(h) != FI_OK) {
            // conditional graph nodes unavailable: use the host loop
            cudaGetLastError();
            if (h->seg_graph) { cudaGraphDestroy(h->seg_graph); h->seg_graph = nullptr; }
            h->graph_ok = false;
        }
    }
    if (h->seg_exec) {
        CK(cudaGraphLaunch(h->seg_exec, h->stream));
        RET(read_ctl(h));
        return FI_OK;
    }
    k_segment_start<<<1, 32, 0, h->stream>>>(h->d_mem, 1, 0, 0);
    CKL();
    const int batch = 32;
    for (;;) {
        for (int b = 0; b < batch; b++) {
            for (int s = 2; s <= 4; s++) {
                RET(launch_sparse(h));
                RET(launch_rhs_body(h, s, nullptr, nullptr, nullptr, 0, 0));
            }
        }
        RET(read_ctl(h));
        if (!h->ctl.active) break;
    }
    return FI_OK;
}

// ---------------------------------------------------------------------------
// plain form: one step attempt + host controller
// ---------------------------------------------------------------------------
static int attempt_plain(fi_handle* h) {
    const fi_config& c = h->cfg;
    PlainBufs& p = h->p;
    Ctl& ct = h->ctl;
    const size_t n = N2(h);
    const double t = ct.t, dt = ct.dt;
    double* up = p.u[ct.ibuf];
    double* un = p.u[ct.ibuf ^ 1];
    double* k1 = p.k14[ct.ik];
    double* k4 = p.k14[ct.ik ^ 1];
    if (c.alg == FI_ALG_EULER) {
        // perform_step!(integrator, ::EulerCache): u = uprev + dt k1, k4 = f(u, t + dt)
        kp_stage<<<gs(n), NT, 0, h->stream>>>(un, up, dt, k1, n);
        CKL();
        RET(rhs_plain(h, t + dt, un, k4));
        euler_accept(&ct, c.dt_min, h->tout.data());
        ct.nsteps_seg += 1;
        return FI_OK;
    }
    kp_stage<<<gs(n), NT, 0, h->stream>>>(p.tmp, up, dt * A21, k1, n);
    CKL();
    RET(rhs_plain(h, t + C2 * dt, p.tmp, p.k2));
    kp_stage<<<gs(n), NT, 0, h->stream>>>(p.tmp, up, dt * A32, p.k2, n);
    CKL();
    RET(rhs_plain(h, t + C3 * dt, p.tmp, p.k3));
    kp_stage4<<<gs(n), NT, 0, h->stream>>>(un, up, dt, k1, p.k2, p.k3, n);
    CKL();
    RET(rhs_plain(h, t + dt, un, k4));
    kp_err<<<h->red_blocks, NT, 0, h->stream>>>(up, un, k1, p.k2, p.k3, k4, dt, c.abstol, c.reltol, p.partial, n);
    CKL();
    double s = 0.0;
    RET(reduce_host(h, p.partial, h->red_blocks, 1, &s));
    const double EEst = sqrt(s / (double)n);
    controller_update(&ct, EEst, h->tout.data());
    ct.nsteps_seg += 1;
    return FI_OK;
}

static int run_segment_plain(fi_handle* h) {
    Ctl& ct = h->ctl;
    ct.pending_output = 0;
    ct.nsteps_seg = 0;
    if (!(ct.t < ct.t_stop)) return FI_OK;
    loopheader_prep(&ct);
    while (ct.status == FI_OK) {
        RET(attempt_plain(h));
        if (ct.status != FI_OK) break;
        if (ct.accept_step && (ct.pending_output || !(ct.t < ct.t_stop))) break;
        loopheader_prep(&ct);
    }
    return FI_OK;
}

// FSAL re-evaluation after a modifying callback: k1 = f(u, t)
static int reeval_fsal(fi_handle* h) {
    if (h->cfg.form == FI_FORM_FP32) {
        RET(read_ctl(h));
        h->ctl.t_call = h->ctl.t;
        RET(write_ctl(h));
        RET(rhs_fused(h, 1, nullptr, nullptr, nullptr));
        RET(read_ctl(h));
    } else {
        // apply_step!: uprev <- u, then f(fsalfirst, u, p, t) on the integrator's u, whose
        // in-place changes (the laterally constant Maxwell step writes u) the next
        // perform_step! overwrites from uprev: evaluate on a copy so that uprev stays
        const size_t n = N2(h);
        CK(cudaMemcpyAsync(h->p.tmp, h->p.u[h->ctl.ibuf], n * 8, cudaMemcpyDeviceToDevice, h->stream));
        RET(rhs_plain(h, h->ctl.t, h->p.tmp, h->p.k14[h->ctl.ik]));
    }
    return FI_OK;
}

struct OutBufs {
    double *t, *u, *ue, *dudt, *dz;
};

// nout_affect! / write_out! (src/simulation.jl:214-225, src/io.jl:349-353) as an
// asynchronous pipeline: the output fields are copied on the device into a staging slot
// (FP32 form: with the corner offsets applied, in FP64) behind the segment that reached
// the output time; a copy stream reads the slot back into pinned host memory while the
// next segment runs; the host moves it into the caller's arrays when the slot is reused
// or when the call ends.  Two slots: at most one output waits while the next is staged.
static int out_finish(fi_handle* h, int slot) {
    fi_handle::PendingOut& pd = h->pend[slot];
    if (!pd.busy) return FI_OK;
    CK(cudaEventSynchronize(h->ev_copied[slot]));
    const size_t n = N2(h);
    for (int f = 0; f < 4; f++)
        if (pd.dst[f]) memcpy(pd.dst[f] + (size_t)pd.k * n, h->h_out_slot[slot] + (size_t)f * n, n * sizeof(double));
    pd.busy = false;
    return FI_OK;
}

static int out_finish_all(fi_handle* h) {
    // oldest first: slot of the lower output index
    int a = 0, b = 1;
    if (h->pend[1].busy && (!h->pend[0].busy || h->pend[1].k < h->pend[0].k)) { a = 1; b = 0; }
    RET(out_finish(h, a));
    RET(out_finish(h, b));
    return FI_OK;
}

static int out_setup(fi_handle* h) {
    if (h->cstream) return FI_OK;
    const size_t bytes = 4 * N2(h) * sizeof(double);
    CK(cudaStreamCreateWithFlags(&h->cstream, cudaStreamNonBlocking));
    for (int q = 0; q < 2; q++) {
        CK(cudaEventCreateWithFlags(&h->ev_staged[q], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->ev_copied[q], cudaEventDisableTiming));
        CK(cudaMalloc(&h->d_out_slot[q], bytes));
        CK(cudaMallocHost(&h->h_out_slot[q], bytes));
    }
    return FI_OK;
}

static int record_output(fi_handle* h, int k, const OutBufs& o) {
    const size_t n = N2(h);
    const fi_config& c = h->cfg;
    if (o.t) o.t[k] = h->ctl.t;
    if (!o.u && !o.ue && !o.dudt && !o.dz) return FI_OK;
    RET(out_setup(h));
    const int slot = k & 1;
    RET(out_finish(h, slot));
    double* d = h->d_out_slot[slot];
    if (c.form == FI_FORM_FP32) {
        Member& m = h->mem;
        const Ctl& ct = h->ctl;
        const double cue = corner_mean(ct.ue_corner[ct.iue]) - c.bc_elastic_border;
        const double cdu = corner_mean(ct.kcorner[ct.ik]) - c.bc_viscous_border;
        const double cdz = corner_mean(ct.dz_corner) - c.bc_sea_surface_border;
        k_out_stage<<<gs(n), NT, 0, h->stream>>>(o.u ? m.u[ct.ibuf] : nullptr, o.ue ? m.ue[ct.iue] : nullptr, cue,
                                                 o.dudt ? m.k14[ct.ik] : nullptr, cdu, o.dz ? m.dz : nullptr, cdz,
                                                 d, n);
        CKL();
    } else {
        PlainBufs& p = h->p;
        const double* src[4] = {p.now_u, p.ue, p.dudt, p.dz};
        const bool want[4] = {o.u != nullptr, o.ue != nullptr, o.dudt != nullptr, o.dz != nullptr};
        for (int f = 0; f < 4; f++)
            if (want[f]) CK(cudaMemcpyAsync(d + (size_t)f * n, src[f], n * 8, cudaMemcpyDeviceToDevice, h->stream));
    }
    CK(cudaEventRecord(h->ev_staged[slot], h->stream));
    CK(cudaStreamWaitEvent(h->cstream, h->ev_staged[slot], 0));
    CK(cudaMemcpyAsync(h->h_out_slot[slot], d, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, h->cstream));
    CK(cudaEventRecord(h->ev_copied[slot], h->cstream));
    fi_handle::PendingOut& pd = h->pend[slot];
    pd.busy = true;
    pd.k = k;
    pd.dst[0] = o.u; pd.dst[1] = o.ue; pd.dst[2] = o.dudt; pd.dst[3] = o.dz;
    return FI_OK;
}

// solve!(integrator): segments between tstops; outputs by nout_condition
static int solve_until_(fi_handle* h, const OutBufs* o);

// device time of one integration call, CUDA events on the handle's stream
static int solve_until(fi_handle* h, const OutBufs* o) {
    CK(cudaEventRecord(h->ev0, h->stream));
    const int rc = solve_until_(h, o);
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->last_gpu_ms = ms;
    h->gpu_ms += ms;
    return rc;
}

static int solve_until_(fi_handle* h, const OutBufs* o) {
    const bool fused = h->cfg.form == FI_FORM_FP32;
    while (!h->tstops.empty()) {
        if (h->fsal_pending) {
            // apply_step! of the next attempt: reset_fsal! after a modifying callback
            RET(reeval_fsal(h));
            h->fsal_pending = false;
            if (h->ctl.status != FI_OK) return set_err(h, h->ctl.status, "%s", fi_status_string(h->ctl.status));
        }
        if (fused) RET(read_ctl(h));
        h->ctl.t_stop = h->tstops.front();
        if (fused) RET(write_ctl(h));
        if (fused) RET(run_segment_fused(h)); else RET(run_segment_plain(h));
        h->segments += 1;
        Ctl& ct = h->ctl;
        if (ct.status != FI_OK)
            return set_err(h, ct.status, "integration stopped at t=%.6g: %s", ct.t, fi_status_string(ct.status));
        if (ct.pending_output) {
            if (o) RET(record_output(h, ct.kout, *o));
            ct.kout += 1;
            ct.pending_output = 0;
            if (fused) RET(write_ctl(h));
            h->fsal_pending = true;
        }
        while (!h->tstops.empty() && h->ctl.t == h->tstops.front()) h->tstops.erase(h->tstops.begin());
        if (!h->tstops.empty() && h->ctl.t > h->tstops.front())
            return set_err(h, FI_ERR_STATE, "integrator stepped past a tstop");
    }
    return FI_OK;
}

static int set_tstops(fi_handle* h, int n, const double* ts, bool outputs) {
    const double t0 = h->cfg.t0, t1 = h->cfg.t1;
    std::vector<double> v;
    for (int i = 0; i < n; i++)
        if (ts[i] > t0 && ts[i] <= t1) v.push_back(ts[i]);
    v.push_back(t1);
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    h->tstops = v;
    h->tout.assign(ts, ts + n);
    if (n > MAX_TSTOPS) return set_err(h, FI_ERR_ARG, "too many output times");
    h->ctl.nout = outputs ? n : 0;
    h->ctl.kout = 0;
    if (n) CK(cudaMemcpyAsync(h->d_tout, ts, n * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FI_OK;
}

extern "C" int fi_run(fi_handle* h, int32_t n_out, const double* t_out, double* out_t, double* out_u,
                      double* out_ue, double* out_dudt, double* out_dz_ss) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || n_out < 0 || (n_out > 0 && !t_out)) return FI_ERR_ARG;
    if (!h->initialized) return set_err(h, FI_ERR_STATE, "fi_init not called");
    for (int k = 1; k < n_out; k++)
        if (t_out[k] < t_out[k - 1]) return set_err(h, FI_ERR_ARG, "t_out must be sorted");
    RET(integ_start(h));
    if (h->cfg.form == FI_FORM_FP32) RET(read_ctl(h));
    RET(set_tstops(h, n_out, t_out, true));
    if (h->cfg.form == FI_FORM_FP32) RET(write_ctl(h));
    OutBufs o{out_t, out_u, out_ue, out_dudt, out_dz_ss};
    const int rc = solve_until(h, &o);
    const int rc2 = out_finish_all(h);  // the caller's arrays are complete when fi_run returns
    h->last_call = 0;
    return rc ? rc : rc2;
}

extern "C" int fi_init_integrator(fi_handle* h, int32_t n_tstops, const double* tstops) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || n_tstops < 0) return FI_ERR_ARG;
    if (!h->initialized) return set_err(h, FI_ERR_STATE, "fi_init not called");
    RET(integ_start(h));
    if (h->cfg.form == FI_FORM_FP32) RET(read_ctl(h));
    // init(prob; tstops = nout.t, callback = nout_callback): the output callback still
    // fires (and forces the FSAL re-evaluation) although nothing is recorded here
    RET(set_tstops(h, n_tstops, tstops, true));
    if (h->cfg.form == FI_FORM_FP32) RET(write_ctl(h));
    return FI_OK;
}

extern "C" int fi_step(fi_handle* h, double dt) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !(dt > 0)) return FI_ERR_ARG;
    if (!h->integ_started) return set_err(h, FI_ERR_STATE, "fi_init_integrator not called");
    if (h->cfg.form == FI_FORM_FP32) RET(read_ctl(h));
    const double next_t = h->ctl.t + dt;
    if (next_t > h->cfg.t1) return set_err(h, FI_ERR_ARG, "step beyond t_span");
    // add_tstop!(integrator, t + dt); advance until t >= next_t
    std::vector<double>& v = h->tstops;
    v.insert(std::lower_bound(v.begin(), v.end(), next_t), next_t);
    v.erase(std::unique(v.begin(), v.end()), v.end());
    std::vector<double> rest;
    while (!v.empty() && v.back() > next_t) { rest.insert(rest.begin(), v.back()); v.pop_back(); }
    int rc = solve_until(h, nullptr);
    v.insert(v.end(), rest.begin(), rest.end());
    h->last_call = 0;
    return rc;
}

// ---------------------------------------------------------------------------
// step-sequence record and replay: the controller (fi_device.cuh) appends every
// accepted dt to ctl.rec_dt and, while a replay is installed, accepts every attempt
// and takes the next dt from ctl.replay_dt.  FP32 form: device arrays (the control
// block lives on the device); plain form: host arrays (host controller).
// ---------------------------------------------------------------------------
extern "C" int fi_record_steps(fi_handle* h, int64_t cap) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || cap < 0) return FI_ERR_ARG;
    if (!h->integ_started) return set_err(h, FI_ERR_STATE, "fi_init_integrator not called");
    const bool fused = h->cfg.form == FI_FORM_FP32;
    if (fused) RET(read_ctl(h));
    if (h->d_rec) {
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaFree(h->d_rec));
        h->d_rec = nullptr;
    }
    h->h_rec.clear();
    h->h_rec.shrink_to_fit();
    double* p = nullptr;
    if (cap > 0) {
        if (fused) {
            CK(cudaMalloc(&h->d_rec, (size_t)cap * sizeof(double)));
            p = h->d_rec;
        } else {
            h->h_rec.assign((size_t)cap, 0.0);
            p = h->h_rec.data();
        }
    }
    h->ctl.rec_dt = p;
    h->ctl.rec_cap = cap;
    h->ctl.rec_n = 0;
    if (fused) RET(write_ctl(h));
    return FI_OK;
}

extern "C" int fi_get_step_record(fi_handle* h, double* dts, int64_t cap, int64_t* n) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !n || cap < 0 || (cap > 0 && !dts)) return FI_ERR_ARG;
    if (!h->integ_started) return set_err(h, FI_ERR_STATE, "fi_init_integrator not called");
    if (h->cfg.form == FI_FORM_FP32) RET(read_ctl(h));
    const long long stored = std::min(h->ctl.rec_n, h->ctl.rec_cap);
    const long long k = std::min<long long>(stored, cap);
    if (k > 0) {
        if (h->cfg.form == FI_FORM_FP32) {
            CK(cudaMemcpyAsync(dts, h->d_rec, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        } else {
            memcpy(dts, h->h_rec.data(), (size_t)k * sizeof(double));
        }
    }
    *n = h->ctl.rec_n;
    return FI_OK;
}

extern "C" int fi_set_step_replay(fi_handle* h, int64_t n, const double* dts) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || n < 0 || (n > 0 && !dts)) return FI_ERR_ARG;
    if (!h->integ_started) return set_err(h, FI_ERR_STATE, "fi_init_integrator not called");
    for (int64_t i = 0; i < n; i++)
        if (!(fabs(dts[i]) > 0 && fabs(dts[i]) < INFINITY))
            return set_err(h, FI_ERR_ARG, "replayed dt[%lld] is zero or not finite", (long long)i);
    const bool fused = h->cfg.form == FI_FORM_FP32;
    if (fused) RET(read_ctl(h));
    if (h->d_replay) {
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaFree(h->d_replay));
        h->d_replay = nullptr;
    }
    h->h_replay.assign(dts, dts + n);
    const double* p = nullptr;
    if (n > 0) {
        if (fused) {
            CK(cudaMalloc(&h->d_replay, (size_t)n * sizeof(double)));
            CK(cudaMemcpyAsync(h->d_replay, dts, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            p = h->d_replay;
        } else {
            p = h->h_replay.data();
        }
        h->ctl.dt = fabs(dts[0]);
        h->ctl.dtpropose = fabs(dts[0]);
    }
    h->ctl.replay_dt = p;
    h->ctl.replay_n = n;
    h->ctl.replay_i = n > 0 ? 1 : 0;
    if (fused) RET(write_ctl(h));
    return FI_OK;
}

// ---------------------------------------------------------------------------
// batched ensembles: the members' step loops run concurrently on their own streams
// ---------------------------------------------------------------------------
struct fi_ensemble {
    std::vector<fi_handle*> mem;
    std::vector<cudaEvent_t> ev_start, ev_end;
    double last_gpu_ms = 0.0;
    std::string err;
    // persistent executor (one cooperative launch per segment for all members)
    bool persist = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Member* d_mems = nullptr;
    Ctl** d_ctls = nullptr;
    unsigned int* d_bar = nullptr;
    unsigned long long* d_counter = nullptr;
    unsigned long long* d_trace = nullptr;
    EnsArgs args{};
    const void* kfn = nullptr;  // the ensemble kernel build (ens_kernel)
    int grid = 0;
    size_t smem = 0;
    long long launches = 0;
};

static void ensemble_free(fi_ensemble* e) {
    if (e->d_mems) cudaFree(e->d_mems);
    if (e->d_ctls) cudaFree(e->d_ctls);
    if (e->d_bar) cudaFree(e->d_bar);
    if (e->d_counter) cudaFree(e->d_counter);
    if (e->d_trace) cudaFree(e->d_trace);
    if (e->e0) cudaEventDestroy(e->e0);
    if (e->e1) cudaEventDestroy(e->e1);
    if (e->stream) cudaStreamDestroy(e->stream);
    e->d_mems = nullptr; e->d_ctls = nullptr; e->d_bar = nullptr; e->d_counter = nullptr; e->d_trace = nullptr;
    e->e0 = e->e1 = nullptr;
    e->stream = nullptr;
}

// Persistent ensemble executor set-up; false leaves the stream executor in charge.
static bool ensemble_setup_persist(fi_ensemble* e) {
    const char* ex = getenv("FI_ENS_EXECUTOR");
    if (ex && !strcmp(ex, "streams")) return false;
    const int n = (int)e->mem.size();
    if (n > ENS_MAX_MEMBERS) return false;
    const int dev = e->mem[0]->cfg.device;
    int coop = 0, nsm = 0, occ = 0, smax = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return false;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    std::vector<Member> hm(n);
    std::vector<Ctl*> hc(n);
    for (int i = 0; i < n; i++) {
        hm[i] = e->mem[i]->mem;
        hc[i] = e->mem[i]->d_ctl;
    }
    EnsArgs& a = e->args;
    a = EnsArgs{};
    const size_t smem = ens_layout(hm.data(), n, &a);
    cudaFuncAttributes fa{};
    const char* es = getenv("FI_ENS_SEQ");
    e->kfn = ens_kernel(!(es && es[0] == '0'));
    if (cudaFuncGetAttributes(&fa, e->kfn) != cudaSuccess) return false;
    if (smem + fa.sharedSizeBytes + 1024 > (size_t)smax) return false;
    if (cudaFuncSetAttribute(e->kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, e->kfn, ROW_THREADS, smem) != cudaSuccess || occ < 1)
        return false;
    const bool okk = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess &&
                     cudaEventCreate(&e->e0) == cudaSuccess && cudaEventCreate(&e->e1) == cudaSuccess &&
                     cudaMalloc(&e->d_mems, n * sizeof(Member)) == cudaSuccess &&
                     cudaMalloc(&e->d_ctls, n * sizeof(Ctl*)) == cudaSuccess &&
                     cudaMalloc(&e->d_bar, 4 * sizeof(unsigned int)) == cudaSuccess &&
                     cudaMalloc(&e->d_counter, sizeof(unsigned long long)) == cudaSuccess &&
                     cudaMalloc(&e->d_trace, 2 * PH_COUNT * sizeof(unsigned long long)) == cudaSuccess &&
                     cudaMemcpy(e->d_mems, hm.data(), n * sizeof(Member), cudaMemcpyHostToDevice) == cudaSuccess &&
                     cudaMemcpy(e->d_ctls, hc.data(), n * sizeof(Ctl*), cudaMemcpyHostToDevice) == cudaSuccess &&
                     cudaMemset(e->d_trace, 0, 2 * PH_COUNT * sizeof(unsigned long long)) == cudaSuccess;
    if (!okk) return false;
    a.mems = e->d_mems;
    a.ctls = e->d_ctls;
    a.nmem = n;
    a.bar = e->d_bar;
    a.counter = e->d_counter;
    a.trace = nullptr;
    e->grid = nsm * std::min(occ, 2);
    e->smem = smem;
    return true;
}

extern "C" int fi_ensemble_create(fi_handle* const* members, int32_t n, fi_ensemble** out) {
    if (!members || n < 1 || !out) return FI_ERR_ARG;
    *out = nullptr;
    const int dev = members[0]->cfg.device;
    for (int i = 0; i < n; i++) {
        fi_handle* h = members[i];
        if (!h || h->cfg.form != FI_FORM_FP32 || h->cfg.device != dev) return FI_ERR_ARG;
        if (!h->integ_started) return FI_ERR_STATE;
        for (int j = 0; j < i; j++)
            if (members[j] == h) return FI_ERR_ARG;
    }
    cudaSetDevice(dev);
    fi_ensemble* e = new fi_ensemble();
    e->mem.assign(members, members + n);
    e->ev_start.resize(n);
    e->ev_end.resize(n);
    e->persist = ensemble_setup_persist(e);
    if (!e->persist) {
        ensemble_free(e);
        cudaGetLastError();
    }
    for (int i = 0; i < n; i++) {
        // each member's step loop is a CUDA graph (the persistent executor assumes the
        // whole GPU); the members' graphs overlap on their streams
        fi_handle* h = e->mem[i];
        if (h->executor == EXEC_PERSIST) h->executor = EXEC_GRAPH;
        if (cudaEventCreate(&e->ev_start[i]) != cudaSuccess || cudaEventCreate(&e->ev_end[i]) != cudaSuccess) {
            fi_ensemble_destroy(e);
            return FI_ERR_CUDA;
        }
    }
    *out = e;
    return FI_OK;
}

void fi_ensemble_destroy(fi_ensemble* e) {
    if (!e) return;
    if (!e->mem.empty()) cudaSetDevice(e->mem[0]->cfg.device);
    for (cudaEvent_t ev : e->ev_start)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : e->ev_end)
        if (ev) cudaEventDestroy(ev);
    ensemble_free(e);
    delete e;
}

// One member's completion of a launched segment (the tail of solve_until_).
static int ensemble_finish_segment(fi_handle* h) {
    RET(read_ctl(h));
    h->segments += 1;
    Ctl& ct = h->ctl;
    if (ct.status != FI_OK)
        return set_err(h, ct.status, "integration stopped at t=%.6g: %s", ct.t, fi_status_string(ct.status));
    if (ct.pending_output) {
        ct.kout += 1;
        ct.pending_output = 0;
        RET(write_ctl(h));
        h->fsal_pending = true;
    }
    while (!h->tstops.empty() && h->ctl.t == h->tstops.front()) h->tstops.erase(h->tstops.begin());
    if (!h->tstops.empty() && h->ctl.t > h->tstops.front())
        return set_err(h, FI_ERR_STATE, "integrator stepped past a tstop");
    return FI_OK;
}

static int ensemble_launch_segment(fi_handle* h) {
    if (h->fsal_pending) {
        RET(reeval_fsal(h));
        h->fsal_pending = false;
        if (h->ctl.status != FI_OK) return set_err(h, h->ctl.status, "%s", fi_status_string(h->ctl.status));
    }
    RET(read_ctl(h));
    h->ctl.t_stop = h->tstops.front();
    RET(write_ctl(h));
    return launch_segment_graph_async(h);
}

// Persistent path of fi_ensemble_step: each launch runs one segment of every member
// that has one left; members are prepared (FSAL, t_stop) and finished on the host.
static int ensemble_step_persist(fi_ensemble* e, std::vector<std::vector<double>>& rest, std::vector<int>& st,
                                 std::vector<int>& state, int32_t* status) {
    const int n = (int)e->mem.size();
    double ms_total = 0.0;
    for (;;) {
        bool any = false;
        for (int i = 0; i < n; i++) {
            if (state[i] != 0) continue;
            fi_handle* h = e->mem[i];
            if (h->tstops.empty()) { state[i] = 2; continue; }
            int rc = FI_OK;
            if (h->fsal_pending) {
                rc = reeval_fsal(h);
                h->fsal_pending = false;
                if (!rc && h->ctl.status != FI_OK) rc = set_err(h, h->ctl.status, "%s", fi_status_string(h->ctl.status));
            }
            if (!rc) rc = read_ctl(h);
            if (!rc) {
                h->ctl.t_stop = h->tstops.front();
                rc = write_ctl(h);
            }
            if (rc) { st[i] = rc; state[i] = 2; continue; }
            state[i] = 1;
            any = true;
        }
        // members without a segment in this ensemble step must not step: their t_stop is their t
        for (int i = 0; i < n; i++) {
            if (state[i] == 1) continue;
            fi_handle* h = e->mem[i];
            if (read_ctl(h) == FI_OK) {
                h->ctl.t_stop = h->ctl.t;
                write_ctl(h);
            }
        }
        if (!any) break;
        if (cudaMemsetAsync(e->d_bar, 0, 4 * sizeof(unsigned int), e->stream) != cudaSuccess ||
            cudaMemsetAsync(e->d_counter, 0, sizeof(unsigned long long), e->stream) != cudaSuccess)
            return FI_ERR_CUDA;
        void* args[] = {(void*)&e->args};
        cudaEventRecord(e->e0, e->stream);
        cudaError_t ce = cudaLaunchCooperativeKernel(e->kfn, dim3(e->grid), dim3(ROW_THREADS), args,
                                                     e->smem, e->stream);
        cudaEventRecord(e->e1, e->stream);
        unsigned int bar[4] = {0, 0, 0, 0};
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(bar, e->d_bar, sizeof(bar), cudaMemcpyDeviceToHost, e->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
        if (ce != cudaSuccess) {
            for (int i = 0; i < n; i++)
                if (state[i] == 1) {
                    st[i] = set_err(e->mem[i], FI_ERR_CUDA, "ensemble kernel: %s", cudaGetErrorString(ce));
                    state[i] = 2;
                }
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e->e0, e->e1);
        ms_total += ms;
        e->launches += 1;
        for (int i = 0; i < n; i++) {
            if (state[i] != 1) continue;
            fi_handle* h = e->mem[i];
            const int rc = bar[2] ? set_err(h, FI_ERR_TIMEOUT, "ensemble kernel: a grid barrier wait gave up")
                                  : ensemble_finish_segment(h);
            state[i] = rc ? 2 : 0;
            if (rc) st[i] = rc;
        }
    }
    for (int i = 0; i < n; i++) {
        fi_handle* h = e->mem[i];
        h->tstops.insert(h->tstops.end(), rest[i].begin(), rest[i].end());
        h->last_call = 0;
    }
    e->last_gpu_ms = ms_total;
    if (status)
        for (int i = 0; i < n; i++) status[i] = st[i];
    return FI_OK;
}

extern "C" int fi_ensemble_step(fi_ensemble* e, double dt, int32_t* status) {
    if (!e || !(dt > 0)) return FI_ERR_ARG;
    const int n = (int)e->mem.size();
    cudaSetDevice(e->mem[0]->cfg.device);
    std::vector<std::vector<double>> rest(n);
    std::vector<int> st(n, FI_OK), state(n, 0);  // state: 0 idle, 1 launched, 2 done
    for (int i = 0; i < n; i++) {
        fi_handle* h = e->mem[i];
        int rc = read_ctl(h);
        const double next_t = h->ctl.t + dt;
        if (!rc && next_t > h->cfg.t1) rc = set_err(h, FI_ERR_ARG, "step beyond t_span");
        if (rc) { st[i] = rc; state[i] = 2; continue; }
        std::vector<double>& v = h->tstops;
        v.insert(std::lower_bound(v.begin(), v.end(), next_t), next_t);
        v.erase(std::unique(v.begin(), v.end()), v.end());
        while (!v.empty() && v.back() > next_t) { rest[i].insert(rest[i].begin(), v.back()); v.pop_back(); }
        if (cudaEventRecord(e->ev_start[i], h->stream) != cudaSuccess) { st[i] = FI_ERR_CUDA; state[i] = 2; }
    }
    if (e->persist) return ensemble_step_persist(e, rest, st, state, status);
    for (;;) {
        bool any = false;
        for (int i = 0; i < n; i++) {
            if (state[i] != 0) continue;
            fi_handle* h = e->mem[i];
            if (h->tstops.empty()) { state[i] = 2; continue; }
            const int rc = ensemble_launch_segment(h);
            if (rc) { st[i] = rc; state[i] = 2; continue; }
            state[i] = 1;
            any = true;
        }
        if (!any) break;
        for (int i = 0; i < n; i++) {
            if (state[i] != 1) continue;
            const int rc = ensemble_finish_segment(e->mem[i]);
            state[i] = rc ? 2 : 0;
            if (rc) st[i] = rc;
        }
    }
    float ms = 0.0f, t_first = 0.0f, t_last = 0.0f;
    bool timed = false;
    for (int i = 0; i < n; i++) {
        fi_handle* h = e->mem[i];
        h->tstops.insert(h->tstops.end(), rest[i].begin(), rest[i].end());
        h->last_call = 0;
        if (cudaEventRecord(e->ev_end[i], h->stream) != cudaSuccess) continue;
        if (cudaEventSynchronize(e->ev_end[i]) != cudaSuccess) continue;
        float a = 0.0f, b = 0.0f;
        if (cudaEventElapsedTime(&a, e->ev_start[0], e->ev_start[i]) != cudaSuccess) continue;
        if (cudaEventElapsedTime(&b, e->ev_start[0], e->ev_end[i]) != cudaSuccess) continue;
        if (!timed) { t_first = a; t_last = b; timed = true; }
        t_first = std::min(t_first, a);
        t_last = std::max(t_last, b);
    }
    if (timed) ms = t_last - t_first;
    e->last_gpu_ms = ms;
    if (status)
        for (int i = 0; i < n; i++) status[i] = st[i];
    return FI_OK;
}

extern "C" double fi_ensemble_last_gpu_ms(const fi_ensemble* e) { return e ? e->last_gpu_ms : 0.0; }

extern "C" int fi_ensemble_trace(fi_ensemble* e, int32_t on, double* ms, int64_t* counts) {
    if (!e) return FI_ERR_ARG;
    if (!e->persist) return FI_ERR_UNSUPPORTED;
    cudaSetDevice(e->mem[0]->cfg.device);
    if (ms && counts) {
        unsigned long long v[2 * PH_COUNT];
        if (cudaMemcpy(v, e->d_trace, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return FI_ERR_CUDA;
        for (int p = 0; p < PH_COUNT; p++) {
            ms[p] = (double)v[2 * p] * 1e-6;
            counts[p] = (int64_t)v[2 * p + 1];
        }
    }
    if (on >= 0) {
        if (on && cudaMemset(e->d_trace, 0, 2 * PH_COUNT * sizeof(unsigned long long)) != cudaSuccess)
            return FI_ERR_CUDA;
        e->args.trace = on ? e->d_trace : nullptr;
    }
    return FI_OK;
}

extern "C" int fi_get_sealevel(fi_handle* h, fi_sealevel* out) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !out) return FI_ERR_ARG;
    memset(out, 0, sizeof(*out));
    if (!h->initialized) {
        out->z_bsl = h->cfg.z_bsl;
        out->A_bsl = h->cfg.bsl_ref_A;
        return FI_OK;
    }
    RET(read_ctl(h));
    const Ctl& ct = h->ctl;
    out->z_bsl = ct.z_bsl;
    out->A_bsl = ct.A_bsl;
    out->tracked = h->cfg.form == FI_FORM_FP64;
    if (out->tracked) {
        out->V_af = ct.V_af;
        out->V_den = ct.V_den;
        out->V_pov = ct.V_pov;
        out->delta_V = ct.delta_V;
    }
    return FI_OK;
}

extern "C" int fi_get_stats(fi_handle* h, fi_stats* st) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !st) return FI_ERR_ARG;
    memset(st, 0, sizeof(*st));
    if (h->initialized) RET(read_ctl(h));
    const Ctl& ct = h->ctl;
    st->t = ct.t;
    st->dt = ct.dtpropose;
    st->nf = h->cfg.form == FI_FORM_FP32 ? ct.nf : h->nf_plain;
    st->naccept = ct.naccept;
    st->nreject = ct.nreject;
    st->nsparse = ct.count_sparse;
    st->status = ct.status;
    st->form = h->cfg.form;
    st->gpu_ms = h->gpu_ms;
    st->last_gpu_ms = h->last_gpu_ms;
    st->segments = h->segments;
    st->executor = h->cfg.form == FI_FORM_FP32 ? h->executor : -1;
    st->grid = h->executor == EXEC_PERSIST ? h->persist_grid : 0;
    return FI_OK;
}

extern "C" int fi_time_kernels(fi_handle* h, int32_t reps, double* ms) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !ms || reps < 1) return FI_ERR_ARG;
    if (h->cfg.form != FI_FORM_FP32) return set_err(h, FI_ERR_UNSUPPORTED, "kernel timing is for the FP32 form");
    if (!h->initialized) return set_err(h, FI_ERR_STATE, "fi_init not called");
    RET(read_ctl(h));
    h->ctl.active = 1;
    h->ctl.gate = 1;
    h->ctl.status = FI_OK;
    RET(write_ctl(h));
    for (int k = 0; k < 6; k++) {
        for (int r = -3; r < reps; r++) {
            if (r == 0) CK(cudaEventRecord(h->ev0, h->stream));
            switch (k) {
                case 0:
                    k_rows_fwd<<<h->n_rows, ROW_THREADS, rows_fwd_smem(h->mem.fl.bytes, h->nx, (int)h->ice_t.size()), h->stream>>>(
                        h->d_mem, h->t_rows, 3, h->h_rows, nullptr, 1);
                    break;
                case 1:
                    k_cols<<<h->n_cols, ROW_THREADS, cols_smem(h->ny, h->B_cols), h->stream>>>(
                        h->d_mem, h->t_cols, h->B_cols, 0, 0);
                    break;
                case 2:
                    k_rows_inv<<<h->n_rows, ROW_THREADS, rows_inv_smem(h->nx, h->h_rows, h->n_cols), h->stream>>>(
                        h->d_mem, h->t_rows, 1, h->h_rows, nullptr, nullptr, 0, 0);
                    break;
                case 3:
                    k_conv_rows<<<h->n_crow, ROW_THREADS, conv_rows_smem(h->Mx, h->h_conv), h->stream>>>(
                        h->d_mem, h->t_crow, h->h_conv);
                    break;
                case 4:
                    k_conv_cols<<<h->n_ccol, ROW_THREADS, conv_cols_smem(h->My, h->B_conv), h->stream>>>(
                        h->d_mem, h->t_ccol, h->B_conv);
                    break;
                default:
                    k_conv_rows_inv<<<h->n_crowi, ROW_THREADS, conv_rows_smem(h->Mx, h->h_conv), h->stream>>>(
                        h->d_mem, h->t_crowi, h->h_conv);
                    break;
            }
            CKL();
        }
        CK(cudaEventRecord(h->ev1, h->stream));
        CK(cudaEventSynchronize(h->ev1));
        float t = 0.0f;
        CK(cudaEventElapsedTime(&t, h->ev0, h->ev1));
        ms[k] = (double)t / reps;
    }
    return FI_OK;
}

static_assert(FI_NUM_PHASES == PH_COUNT, "phase count mismatch");

extern "C" int fi_trace_phases(fi_handle* h, int32_t on) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h) return FI_ERR_ARG;
    if (h->cfg.form != FI_FORM_FP32) return set_err(h, FI_ERR_UNSUPPORTED, "phase trace is for the FP32 form");
    if (on) CK(cudaMemsetAsync(h->d_trace, 0, 2 * PH_COUNT * sizeof(unsigned long long), h->stream));
    h->pargs.trace = on ? h->d_trace : nullptr;
    CK(cudaStreamSynchronize(h->stream));
    return FI_OK;
}

extern "C" int fi_get_phase_trace(fi_handle* h, double* ms, int64_t* counts) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !ms || !counts) return FI_ERR_ARG;
    if (h->cfg.form != FI_FORM_FP32) return set_err(h, FI_ERR_UNSUPPORTED, "phase trace is for the FP32 form");
    unsigned long long v[2 * PH_COUNT];
    CK(cudaMemcpyAsync(v, h->d_trace, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int p = 0; p < PH_COUNT; p++) {
        ms[p] = (double)v[2 * p] * 1e-6;
        counts[p] = (int64_t)v[2 * p + 1];
    }
    return FI_OK;
}

extern "C" int fi_get_field(fi_handle* h, int32_t field, double* host, size_t n) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !host) return FI_ERR_ARG;
    if (n != N2(h)) return set_err(h, FI_ERR_ARG, "field size %zu != nx*ny", n);
    std::vector<double> v;
    const fi_config& c = h->cfg;
    const bool fused = c.form == FI_FORM_FP32;
    switch (field) {
        case FI_FIELD_LITHO_RIGIDITY: v = h->D; break;
        case FI_FIELD_EFFECTIVE_VISCOSITY: v = h->eta; break;
        case FI_FIELD_MASKACTIVE: v = h->mask; break;
        case FI_FIELD_U_REF: v = h->u_ref; break;
        case FI_FIELD_UE_REF: v = h->ue_ref; break;
        case FI_FIELD_DZ_SS_REF: v = h->dz_ss_ref; break;
        case FI_FIELD_Z_B_REF: v = h->z_b_ref; break;
        case FI_FIELD_TAU: v = h->tau; break;
        case FI_FIELD_PSEUDODIFF_SCALING: RET(download(h, v, h->d_R, n)); break;
        case FI_FIELD_PSEUDODIFF: RET(download(h, v, h->d_pd, n)); break;
        case FI_FIELD_SCALED_PSEUDODIFF_INV: RET(download(h, v, h->d_spinv, n)); break;
        case FI_FIELD_ELASTIC_GREEN: RET(download(h, v, h->d_Ge, n)); break;
        case FI_FIELD_DZ_SS_GREEN: RET(download(h, v, h->d_Gg, n)); break;
        default: {
            if (!h->initialized) return set_err(h, FI_ERR_STATE, "state fields need fi_init");
            RET(read_ctl(h));
            const Ctl& ct = h->ctl;
            if (!fused) {
                const PlainBufs& p = h->p;
                const double* src = nullptr;
                switch (field) {
                    case FI_FIELD_U: src = p.now_u; break;
                    case FI_FIELD_UE: src = p.ue; break;
                    case FI_FIELD_DUDT: src = p.dudt; break;
                    case FI_FIELD_DZ_SS: src = p.dz; break;
                    case FI_FIELD_H_ICE: src = p.H; break;
                    case FI_FIELD_Z_SS: src = p.z_ss; break;
                    case FI_FIELD_Z_B: src = p.z_b; break;
                    case FI_FIELD_COLUMNANOM_LOAD: src = p.s_load; break;
                    case FI_FIELD_COLUMNANOM_FULL: src = p.s_full; break;
                    case FI_FIELD_H_AF: src = p.H_af; break;
                    case FI_FIELD_MASKGROUNDED: src = p.mgr; break;
                    case FI_FIELD_MASKOCEAN: src = p.moc; break;
                    case FI_FIELD_H_WATER: src = p.hwater; break;
                    case FI_FIELD_COLUMNANOM_SEAWATER: src = p.s_sw; break;
                    case FI_FIELD_U_EQ: src = p.u_eq; break;
                    default: return set_err(h, FI_ERR_ARG, "unknown field %d", field);
                }
                RET(download(h, v, src, n));
                break;
            }
            const Member& m = h->mem;
            std::vector<double> ue, dz;
            RET(download(h, ue, m.ue[ct.iue], n));
            const double cue = corner_mean(ct.ue_corner[ct.iue]) - c.bc_elastic_border;
            for (auto& x : ue) x -= cue;
            RET(download(h, dz, m.dz, n));
            const double cdz = corner_mean(ct.dz_corner) - c.bc_sea_surface_border;
            for (auto& x : dz) x -= cdz;
            switch (field) {
                case FI_FIELD_U: RET(download(h, v, m.u[h->last_call == 1 ? ct.ibuf ^ 1 : ct.ibuf], n)); break;
                case FI_FIELD_UE: v = ue; break;
                case FI_FIELD_DZ_SS: v = dz; break;
                case FI_FIELD_DUDT: {
                    const bool scr = h->last_call == 1;
                    RET(download(h, v, scr ? h->d_vscr : m.k14[ct.ik], n));
                    double cc[4];
                    if (scr) {
                        CK(cudaMemcpy(cc, h->d_cscr, 32, cudaMemcpyDeviceToHost));
                    } else {
                        memcpy(cc, ct.kcorner[ct.ik], 32);
                    }
                    const double off = corner_mean(cc) - c.bc_viscous_border;
                    for (auto& x : v) x -= off;
                    break;
                }
                case FI_FIELD_H_ICE: {
                    int st;
                    interp_ice_host(h, h->last_call == 1 ? h->last_rhs_t : ct.t, v, &st);
                    if (c.ice_mode == FI_ICE_EXTERNAL) RET(download(h, v, m.H_ext, n));
                    break;
                }
                case FI_FIELD_Z_SS:
                    v.resize(n);
                    for (size_t k = 0; k < n; k++) v[k] = h->z_ss_ref[k] + dz[k] + ct.z_bsl;
                    break;
                case FI_FIELD_MASKGROUNDED: RET(download(h, v, m.mgr, n)); break;
                case FI_FIELD_MASKOCEAN: RET(download(h, v, m.moc, n)); break;
                case FI_FIELD_H_WATER: RET(download(h, v, m.hwater, n)); break;
                case FI_FIELD_COLUMNANOM_SEAWATER: RET(download(h, v, m.sw, n)); break;
                case FI_FIELD_COLUMNANOM_LOAD: RET(download(h, v, m.sig_load, n)); break;
                case FI_FIELD_COLUMNANOM_FULL:
                    if (m.column_compressible) return set_err(h, FI_ERR_UNSUPPORTED, "full anomaly not kept");
                    RET(download(h, v, m.sig_geo, n));
                    for (auto& x : v) x /= m.A;
                    break;
                default: return set_err(h, FI_ERR_ARG, "field %d not available in the FP32 form", field);
            }
        }
    }
    memcpy(host, v.data(), n * sizeof(double));
    return FI_OK;
}

// ---------------------------------------------------------------------------
// checkpoint / restore: control block + every state buffer
// ---------------------------------------------------------------------------
struct Blob {
    void* d;
    size_t bytes;
};

static std::vector<Blob> state_blobs(fi_handle* h) {
    const size_t n = N2(h);
    std::vector<Blob> b;
    if (h->cfg.form == FI_FORM_FP32) {
        Member& m = h->mem;
        for (int i = 0; i < 2; i++) {
            b.push_back({m.u[i], n * 8});
            b.push_back({m.k14[i], n * 4});
            b.push_back({m.ue[i], n * 4});
        }
        b.push_back({m.k2, n * 4});
        b.push_back({m.k3, n * 4});
        b.push_back({m.dz, n * 4});
        b.push_back({m.sig_load, n * 4});
        b.push_back({m.sig_geo, n * 4});
        b.push_back({m.H_ext, n * 4});
    } else {
        PlainBufs& p = h->p;
        double* bufs[] = {p.u[0], p.u[1], p.k14[0], p.k14[1], p.k2, p.k3, p.now_u, p.ue, p.dz, p.H, p.H_af, p.z_b,
                          p.z_ss, p.s_i, p.s_l, p.s_m, p.s_load, p.s_full, p.dudt};
        for (double* q : bufs) b.push_back({q, n * 8});
    }
    return b;
}

// Checkpoint layout: CkHeader, the control block, nf_plain, last_call, the tstops
// (CkHeader::nts doubles), then the state blobs of the handle's form in order.
struct CkHeader {
    char magic[8];        // "FICKPT\0\0"
    uint32_t version;     // CK_VERSION
    int32_t form;         // FI_FORM_*
    int32_t nx, ny;
    uint32_t ctl_bytes;   // sizeof(Ctl)
    uint32_t nblobs;
    uint64_t nts;         // tstops
    uint64_t total;       // bytes of the whole checkpoint
};
static const char CK_MAGIC[8] = {'F', 'I', 'C', 'K', 'P', 'T', 0, 0};
constexpr uint32_t CK_VERSION = 2;

static size_t ck_size(const std::vector<Blob>& blobs, size_t nts) {
    size_t need = sizeof(CkHeader) + sizeof(Ctl) + sizeof(long long) + sizeof(int) + nts * sizeof(double);
    for (auto& b : blobs) need += b.bytes;
    return need;
}

extern "C" int fi_checkpoint(fi_handle* h, void* buf, size_t* size) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !size) return FI_ERR_ARG;
    if (!h->initialized) return set_err(h, FI_ERR_STATE, "fi_init not called");
    auto blobs = state_blobs(h);
    const size_t need = ck_size(blobs, h->tstops.size());
    if (!buf) { *size = need; return FI_OK; }
    if (*size < need) return set_err(h, FI_ERR_ARG, "checkpoint buffer too small");
    RET(read_ctl(h));
    CkHeader hd{};
    memcpy(hd.magic, CK_MAGIC, sizeof(CK_MAGIC));
    hd.version = CK_VERSION;
    hd.form = h->cfg.form;
    hd.nx = h->nx;
    hd.ny = h->ny;
    hd.ctl_bytes = (uint32_t)sizeof(Ctl);
    hd.nblobs = (uint32_t)blobs.size();
    hd.nts = h->tstops.size();
    hd.total = need;
    char* w = (char*)buf;
    memcpy(w, &hd, sizeof(hd)); w += sizeof(hd);
    memcpy(w, &h->ctl, sizeof(Ctl)); w += sizeof(Ctl);
    memcpy(w, &h->nf_plain, sizeof(long long)); w += sizeof(long long);
    int ls = h->last_call;
    memcpy(w, &ls, sizeof(int)); w += sizeof(int);
    memcpy(w, h->tstops.data(), h->tstops.size() * sizeof(double)); w += h->tstops.size() * sizeof(double);
    for (auto& b : blobs) {
        CK(cudaMemcpyAsync(w, b.d, b.bytes, cudaMemcpyDeviceToHost, h->stream));
        w += b.bytes;
    }
    CK(cudaStreamSynchronize(h->stream));
    *size = need;
    return FI_OK;
}

// Every check runs on the caller's bytes before any handle state changes: a rejected
// checkpoint leaves the handle as it was.
extern "C" int fi_restore(fi_handle* h, const void* buf, size_t size) {
    if (h) cudaSetDevice(h->cfg.device);
    if (!h || !buf) return FI_ERR_ARG;
    if (!h->initialized) return set_err(h, FI_ERR_STATE, "fi_init must precede fi_restore");
    if (size < sizeof(CkHeader)) return set_err(h, FI_ERR_ARG, "checkpoint truncated: %zu bytes", size);
    CkHeader hd;
    memcpy(&hd, buf, sizeof(hd));
    if (memcmp(hd.magic, CK_MAGIC, sizeof(CK_MAGIC)) || hd.version != CK_VERSION)
        return set_err(h, FI_ERR_ARG, "not a checkpoint of this library version");
    if (hd.form != h->cfg.form || hd.nx != h->nx || hd.ny != h->ny || hd.ctl_bytes != sizeof(Ctl))
        return set_err(h, FI_ERR_ARG, "checkpoint of form %d on %d x %d does not match this handle (form %d, %d x %d)",
                       hd.form, hd.nx, hd.ny, h->cfg.form, h->nx, h->ny);
    auto blobs = state_blobs(h);
    if (hd.nblobs != blobs.size()) return set_err(h, FI_ERR_ARG, "checkpoint state layout mismatch");
    const size_t fixed = ck_size(blobs, 0);
    if (size < fixed || hd.nts > (size - fixed) / sizeof(double) || hd.nts > (uint64_t)MAX_TSTOPS + 8)
        return set_err(h, FI_ERR_ARG, "checkpoint truncated or tstop count %llu out of range",
                       (unsigned long long)hd.nts);
    const size_t need = ck_size(blobs, (size_t)hd.nts);
    if (size < need || hd.total != need) return set_err(h, FI_ERR_ARG, "checkpoint size mismatch");
    const char* r = (const char*)buf + sizeof(hd);
    Ctl ct;
    memcpy(&ct, r, sizeof(Ctl)); r += sizeof(Ctl);
    long long nf_plain;
    memcpy(&nf_plain, r, sizeof(long long)); r += sizeof(long long);
    int ls;
    memcpy(&ls, r, sizeof(int)); r += sizeof(int);
    std::vector<double> ts((size_t)hd.nts);
    memcpy(ts.data(), r, ts.size() * sizeof(double)); r += ts.size() * sizeof(double);
    // the step record / replay buffers belong to this handle, not to the checkpoint
    if (h->cfg.form == FI_FORM_FP32) RET(read_ctl(h));
    ct.replay_dt = h->ctl.replay_dt;
    ct.rec_dt = h->ctl.rec_dt;
    ct.replay_n = h->ctl.replay_n;
    ct.replay_i = h->ctl.replay_i;
    ct.rec_cap = h->ctl.rec_cap;
    ct.rec_n = h->ctl.rec_n;
    for (auto& b : blobs) {
        CK(cudaMemcpyAsync(b.d, r, b.bytes, cudaMemcpyHostToDevice, h->stream));
        r += b.bytes;
    }
    h->ctl = ct;
    h->nf_plain = nf_plain;
    h->last_call = ls;
    h->tstops.swap(ts);
    RET(write_ctl(h));
    CK(cudaStreamSynchronize(h->stream));
    h->integ_started = true;
    return FI_OK;
}

namespace fi {
void tc_set_wait_polls(long long polls);  // fno_gemm.cu
}

extern "C" int fi_debug_set_wait_limit(int32_t which, int64_t value) {
    switch (which) {
        case FI_WAIT_GRID_POLLS: g_grid_polls.store(value < 0 ? -1 : value); return FI_OK;
        case FI_WAIT_GRID_EXTRA_ARRIVALS:
            if (value > 1024) return FI_ERR_ARG;
            g_grid_extra.store(value < 0 ? 0 : value);
            return FI_OK;
        case FI_WAIT_TC_POLLS: fi::tc_set_wait_polls(value < 0 ? -1 : value); return FI_OK;
        default: return FI_ERR_ARG;
    }
}
