// capi.cu -- host runtime behind the C-ABI of include/gacelle_b200.h.
//
// A gx_context owns one device, one stream and a grow-only device workspace
// reused across calls.  gx_askadam lays the volumes out as one padded SoA
// work-list, runs the fused kernels (or, for opts.path == GX_PATH_PLAIN, the
// op-by-op kernels with a host read of the loss every epoch, mirroring the
// reference loop), and restates the reference's host-side bookkeeping
// (min-loss tracking, convergence signals, stopping; utils/askadam.m:433-671)
// on the per-epoch sums the kernels record.  States the fused kernels do not
// keep (the minimum-loss parameters, the state at a stopping epoch) are rebuilt
// bit-exactly by replaying from the nearest checkpoint.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <mutex>
#include <string>
#include <vector>
#include <map>
#include <array>

#include "../../include/gacelle_b200.h"
#include "gx_internal.h"

using namespace gx;

static thread_local std::string g_err;

static gx_status fail(gx_status s, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? GX_ENOMEM : GX_ECUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                   \
    } while (0)

#define TRY(expr)                         \
    do {                                          \
        gx_status s_ = (expr);                    \
        if (s_ != GX_OK) return s_;               \
    } while (0)

// ---------------------------------------------------------------------------
// Autotuner cache: launch shapes chosen by trial runs, per key, for the
// process (GACELLE_B200_AUTOTUNE=0 turns tuning off: the defaults are used).
// ---------------------------------------------------------------------------
struct TuneKey {
    std::array<long long, 13> k;
    bool operator<(const TuneKey& o) const { return k < o.k; }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, int> g_tune;

static bool autotune_enabled() {
    const char* e = getenv("GACELLE_B200_AUTOTUNE");
    return !(e && strcmp(e, "0") == 0);
}

static int tune_lookup(const TuneKey& key) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    return it == g_tune.end() ? 0 : it->second;
}

static void tune_store(const TuneKey& key, int v) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = v;
}

constexpr int kTuneLayoutBlock = 512;  // layout block of tuned fused jobs: every candidate divides it

// ---------------------------------------------------------------------------
// Context and workspace
// ---------------------------------------------------------------------------
enum Slot {
    S_DATA, S_W, S_B1, S_SIG, S_TH0, S_Z, S_M1, S_M2, S_ZP, S_ZR, S_M1R, S_M2R, S_HIST, S_SCHED,
    S_CKPT, S_RESF, S_RESM, S_THF, S_THM, S_RLF, S_RLM, S_BLK, S_VOLS, S_GIDX, S_MASK, S_GRID0,
    S_GRID1, S_P_TH, S_P_DTH, S_P_SIG, S_P_DSIG, S_P_RES, S_P_GTH, S_P_GZ, S_P_ACC, S_ZMIN,
    S_MC_PART, S_MC_SUM, S_MC_SUMSQ, S_MC_SHIFT, S_MC_X0, S_MC_POST, S_MC_ACC, S_MC_MEAN,
    S_MC_STD, S_FWD_TH, S_FWD_SIG, S_FWD_B1, S_BAR, S_MC_GLOB, S_ROBUST, S_DICT_SIG, S_DICT_D,
    S_DICT_W, S_DICT_E, S_DICT_C, S_DICT_B, S_DICT_S, S_FLAGS, S_DATA_QUADS, S_PRIOR_MU, S_PRIOR_SD, S_SURF_NB, S_SURF_LEN,
    S_MC_STATS, S_TUNE, S_TUNE_HIST, S_BLK_L, S_HGRID0, S_HGRID1, S_NSLOTS
};

struct gx_context {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    volatile int32_t* cancel = nullptr;
    gx_timing timing{};
    void* buf[S_NSLOTS] = {};
    size_t cap[S_NSLOTS] = {};
    cudaEvent_t ev[6] = {};  // call, main kernel, post-processing kernels
    // pinned staging of the small per-call tables, so that their copies are
    // queued without draining the stream (every call ends with a sync, so the
    // next call may refill it)
    void* pin = nullptr;
    size_t pin_cap = 0;
    cudaEvent_t pin_ev = nullptr;  // recorded after the copies out of `pin`
    gx_test_hooks hooks{};         // fault injection (tests); all zero = off
    int ws_requests = 0;           // workspace requests of the current call
};

// The context's pinned staging buffer, once the copies queued from it by an
// earlier call (which may have failed before its final sync) have run.
static gx_status pinned(gx_context* c, size_t bytes, void** out) {
    if (c->pin_ev) CK(cudaEventSynchronize(c->pin_ev));
    else CK(cudaEventCreateWithFlags(&c->pin_ev, cudaEventDisableTiming));
    if (c->pin_cap < bytes) {
        if (c->pin) {
            cudaStreamSynchronize(c->stream);
            cudaFreeHost(c->pin);
            c->pin = nullptr;
            c->pin_cap = 0;
        }
        size_t b = bytes + bytes / 8 + 256;
        CK(cudaMallocHost(&c->pin, b));
        c->pin_cap = b;
    }
    *out = c->pin;
    return GX_OK;
}

static gx_status ws(gx_context* c, Slot s, size_t bytes, void** out) {
    if (bytes == 0) bytes = 16;
    if (c->hooks.fail_alloc_at > 0 && ++c->ws_requests == c->hooks.fail_alloc_at)
        return fail(GX_ENOMEM, "device workspace request %d (%zu bytes): allocation failure injected by the "
                               "context's test hooks", c->ws_requests, bytes);
    if (c->cap[s] < bytes) {
        if (c->buf[s]) {
            cudaStreamSynchronize(c->stream);
            cudaFree(c->buf[s]);
            c->buf[s] = nullptr;
            c->cap[s] = 0;
        }
        size_t b = bytes + bytes / 8;
        CK(cudaMalloc(&c->buf[s], b));
        c->cap[s] = b;
    }
    *out = c->buf[s];
    return GX_OK;
}

template <class T>
static gx_status wsT(gx_context* c, Slot s, size_t n, T** out) {
    void* p;
    TRY(ws(c, s, n * sizeof(T), &p));
    *out = (T*)p;
    return GX_OK;
}

// Opt-in phase trace (environment variable GACELLE_B200_TRACE=1): the host
// wall time of each phase of a call, with the stream drained at every phase
// boundary so that the device work of the phase is included; printed to
// stderr when the call returns.  Off, it costs one branch per phase.
struct PhaseTrace {
    bool on = false;
    cudaStream_t s = nullptr;
    const char* call = "";
    std::chrono::steady_clock::time_point t0, last;
    std::string line;
    PhaseTrace(const char* name, cudaStream_t st) : s(st), call(name) {
        const char* e = getenv("GACELLE_B200_TRACE");
        on = e && e[0] && e[0] != '0';
        if (on) {
            cudaStreamSynchronize(s);
            t0 = last = std::chrono::steady_clock::now();
        }
    }
    void mark(const char* phase) {
        if (!on) return;
        cudaStreamSynchronize(s);
        auto now = std::chrono::steady_clock::now();
        char b[96];
        snprintf(b, sizeof(b), " %s %.3f", phase, std::chrono::duration<double, std::milli>(now - last).count());
        line += b;
        last = now;
    }
    ~PhaseTrace() {
        if (!on) return;
        double tot = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        fprintf(stderr, "[gacelle_b200] %s ms:%s | total %.3f\n", call, line.c_str(), tot);
    }
};

struct CallScope {
    gx_context* c;
    std::lock_guard<std::mutex> lk;
    long long launches0;
    explicit CallScope(gx_context* ctx) : c(ctx), lk(ctx->mu), launches0(g_kernel_launches) {
        cudaSetDevice(ctx->device);
        c->timing = gx_timing{};
        c->ws_requests = 0;
    }
};

extern "C" {

const char* gx_version(void) { return "gacelle_b200 0.1.0 (sm_100a)"; }
int32_t gx_abi_version(void) { return GX_ABI_VERSION; }
const char* gx_last_error(void) { return g_err.c_str(); }

size_t gx_struct_size(const char* name) {
    if (!name) return 0;
    std::string n(name);
    if (n == "gx_model") return sizeof(gx_model);
    if (n == "gx_volume") return sizeof(gx_volume);
    if (n == "gx_askadam_opts") return sizeof(gx_askadam_opts);
    if (n == "gx_askadam_result") return sizeof(gx_askadam_result);
    if (n == "gx_mcmc_opts") return sizeof(gx_mcmc_opts);
    if (n == "gx_mcmc_result") return sizeof(gx_mcmc_result);
    if (n == "gx_timing") return sizeof(gx_timing);
    if (n == "gx_test_hooks") return sizeof(gx_test_hooks);
    return 0;
}

gx_status gx_context_create(int32_t device, gx_context** out) {
    if (!out) return fail(GX_EINVAL, "gx_context_create: out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(GX_ECUDA, "gx_context_create: no CUDA device (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= n) return fail(GX_EINVAL, "gx_context_create: device %d of %d", device, n);
    CK(cudaSetDevice(device));
    gx_context* c = new gx_context();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return fail(GX_ECUDA, "gx_context_create: stream creation failed");
    }
    c->stream = c->own;
    for (auto& ev : c->ev) cudaEventCreate(&ev);
    *out = c;
    return GX_OK;
}

gx_status gx_context_destroy(gx_context* c) {
    if (!c) return GX_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (int s = 0; s < S_NSLOTS; ++s)
        if (c->buf[s]) cudaFree(c->buf[s]);
    if (c->pin) cudaFreeHost(c->pin);
    if (c->pin_ev) cudaEventDestroy(c->pin_ev);
    for (auto& ev : c->ev) cudaEventDestroy(ev);
    cudaStreamDestroy(c->own);
    delete c;
    return GX_OK;
}

gx_status gx_context_set_stream(gx_context* c, void* s) {
    if (!c) return fail(GX_EINVAL, "context is NULL");
    std::lock_guard<std::mutex> lk(c->mu);
    c->stream = s ? (cudaStream_t)s : c->own;
    return GX_OK;
}

gx_status gx_last_timing(gx_context* c, gx_timing* out) {
    if (!c || !out) return fail(GX_EINVAL, "gx_last_timing: NULL argument");
    *out = c->timing;
    return GX_OK;
}

gx_status gx_set_cancel_flag(gx_context* c, volatile int32_t* flag) {
    if (!c) return fail(GX_EINVAL, "context is NULL");
    c->cancel = flag;
    return GX_OK;
}

gx_status gx_context_set_test_hooks(gx_context* c, const gx_test_hooks* h) {
    if (!c) return fail(GX_EINVAL, "context is NULL");
    if (h && (h->fail_alloc_at < 0 || h->wait_limit_cycles < 0 || h->barrier_extra_arrivals < 0))
        return fail(GX_EINVAL, "gx_context_set_test_hooks: negative setting");
    std::lock_guard<std::mutex> lk(c->mu);
    c->hooks = h ? *h : gx_test_hooks{};
    return GX_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Model / protocol
// ---------------------------------------------------------------------------
static gx_status model_sizes(const gx_model* m, int* np, int* nm, int* id) {
    if (!m) return fail(GX_EINVAL, "model is NULL");
    switch (m->kind) {
    case GX_MODEL_R2S:
        if (m->n_te < 1 || m->n_te > kMaxTE || !m->te) return fail(GX_EINVAL, "R2*: need 1..%d echo times", kMaxTE);
        *np = 2; *nm = m->n_te; *id = kR2S;
        return GX_OK;
    case GX_MODEL_R1R2S:
        if (m->n_te < 1 || m->n_te > kMaxTE || !m->te) return fail(GX_EINVAL, "R1R2*: need 1..%d echo times", kMaxTE);
        if (m->n_fa < 1 || m->n_fa > kMaxFA || !m->fa_deg) return fail(GX_EINVAL, "R1R2*: need 1..%d flip angles", kMaxFA);
        if (m->n_te * m->n_fa > kMaxMeas) return fail(GX_EINVAL, "R1R2*: at most %d measurements", kMaxMeas);
        *np = 3; *nm = m->n_te * m->n_fa; *id = kR1R2S;
        return GX_OK;
    case GX_MODEL_NEXI:
        if (m->n_shell < 1 || m->n_shell > kMaxShell || !m->bval || !m->big_delta)
            return fail(GX_EINVAL, "NEXI: need 1..%d shells with b and Delta", kMaxShell);
        if (m->lmax != 0 && m->lmax != 2) return fail(GX_EINVAL, "NEXI: lmax must be 0 or 2");
        if (m->nx < 2 || m->nx > 4096) return fail(GX_EINVAL, "NEXI: nx must be in [2, 4096]");
        *np = m->lmax == 2 ? 5 : 4;
        *nm = m->n_shell * (m->lmax / 2 + 1);
        *id = m->lmax == 2 ? kNEXI2 : kNEXI;
        return GX_OK;
    case GX_MODEL_NEXI_RICE:
        if (m->n_shell < 1 || m->n_shell > kMaxShell || !m->bval || !m->big_delta)
            return fail(GX_EINVAL, "NEXI Rice: need 1..%d shells with b and Delta", kMaxShell);
        // gpuNEXIrice.FWD returns the lmax-0 signal only (NEXI/gpuNEXIrice.m:645-650)
        if (m->lmax != 0) return fail(GX_EUNSUPPORTED, "NEXI Rice: the reference's FWD computes lmax 0 only");
        if (m->nx < 2 || m->nx > 4096) return fail(GX_EINVAL, "NEXI: nx must be in [2, 4096]");
        *np = 4;
        *nm = m->n_shell;
        *id = kNEXI;
        return GX_OK;
    }
    return fail(GX_EUNSUPPORTED, "unknown model kind %d (custom FWD handles are not accelerated)", m->kind);
}

extern "C" gx_status gx_model_sizes(const gx_model* m, int32_t* np, int32_t* nm) {
    int a, b, id;
    TRY(model_sizes(m, &a, &b, &id));
    if (np) *np = a;
    if (nm) *nm = b;
    return GX_OK;
}

static DevProtocol make_protocol(const gx_model* m, int id, int np, int nm, const double* lb,
                                 const double* ub, int nbound) {
    DevProtocol P;
    memset(&P, 0, sizeof(P));
    P.model = id;
    P.nm = nm;
    P.np = np;
    P.n_te = m->n_te;
    P.n_fa = m->n_fa;
    P.n_shell = m->n_shell;
    P.nx = m->nx;
    P.tr = (float)m->tr;
    P.h = m->nx > 1 ? (float)(1.0 / (m->nx - 1)) : 0.0f;
    if (m->te)
        for (int i = 0; i < m->n_te && i < kMaxTE; ++i) {
            P.te[i] = (float)m->te[i];
            P.te_l2e[i] = (float)(m->te[i] * M_LOG2E);
            if (i < kPairTE) {
                P.te_pair[i] = make_float2(P.te[i], P.te[i]);
                P.nl2e_pair[i] = make_float2(-P.te_l2e[i], -P.te_l2e[i]);
            }
        }
    if (m->fa_deg) for (int i = 0; i < m->n_fa && i < kMaxFA; ++i) P.fa_rad[i] = (float)(m->fa_deg[i] * M_PI / 180.0);
    if (m->bval) for (int i = 0; i < m->n_shell && i < kMaxShell; ++i) P.bval[i] = (float)m->bval[i];
    if (m->big_delta) for (int i = 0; i < m->n_shell && i < kMaxShell; ++i) P.delta[i] = (float)m->big_delta[i];
    for (int i = 0; i < nbound && i < kMaxParam; ++i) {
        P.lb[i] = lb ? (float)lb[i] : 0.0f;
        P.ub[i] = ub ? (float)ub[i] : 1.0f;
    }
    if (m->kind == GX_MODEL_NEXI_RICE) {
        P.rice = 1;
        for (int i = 1; i < kRiceNodes - 1; ++i) {  // t_i = i pi / 33 (mybesseli nodes)
            double t = i * M_PI / (kRiceNodes - 1);
            P.rice_cm1[i - 1] = (float)(cos(t) - 1.0);
            P.rice_s2[i - 1] = (float)(sin(t) * sin(t));
        }
    }
    return P;
}

// ---------------------------------------------------------------------------
// Host restatement of the reference's per-epoch bookkeeping
// (update_min_loss :433-446, update_convergence_signals :512-632,
// check_stopping :634-671 of utils/askadam.m; robustConvergence off).
// ---------------------------------------------------------------------------
struct Tracker {
    const gx_askadam_opts* o = nullptr;
    double minLoss = 0, minFid = 0, minReg = 0;
    int minIter = 0;
    double ema = 0;
    std::vector<double> buf;
    double ewic = 0, ewis = 0, ewig = 0;
    bool stopped = false;
    int stop_epoch = 0, reason = GX_STOP_NONE;
    int reprime = 0;  // robustConvergence: epochs until the convergence window is clean again

    void init(const gx_askadam_opts* opts, double fid0, double reg0) {
        o = opts;
        minLoss = fid0 + reg0; minFid = fid0; minReg = reg0; minIter = 0;
        ema = minLoss;
        buf.assign(o->convergence_window > 0 ? o->convergence_window : 1, 1.0);
    }
    // Returns true if the loop stops at epoch e (before the update).  With
    // robustConvergence, lconv is the mean loss of the convergence voxel set
    // and refreshed tells that the set was renewed at this epoch
    // (utils/askadam.m:530-581).
    bool epoch(int e, double fid, double reg, double g2, double z2, double d2, double lconv = 0.0,
               bool refreshed = false) {
        double L = fid + reg;
        if (minLoss > L) { minLoss = L; minFid = fid; minReg = reg; minIter = e; }
        const bool robust = o->robust_convergence != 0;
        if (robust && refreshed) reprime = o->convergence_window;
        const double Lc = robust ? lconv : L;
        double conv;
        if (o->convergence_model == GX_CONV_EMA) {
            double en = o->ema_decay * ema + (1.0 - o->ema_decay) * Lc;
            conv = std::fabs(en - ema) / (std::fabs(ema) + 1e-8);
            ema = en;
        } else {
            int W = (int)buf.size();
            for (int i = 0; i < W - 1; ++i) buf[i] = buf[i + 1];
            buf[W - 1] = Lc;
            double xm = (W + 1) / 2.0, ym = 0, sxy = 0, sxx = 0;
            for (int i = 0; i < W; ++i) ym += buf[i];
            ym /= W;
            for (int i = 0; i < W; ++i) {
                sxy += (i + 1 - xm) * (buf[i] - ym);
                sxx += (i + 1 - xm) * (i + 1 - xm);
            }
            conv = sxx > 0 ? -(sxy / sxx) : 0.0;
        }
        if (reprime > 0) { reprime -= 1; ewic = 0; }
        else if (conv > o->convergence_value || e <= o->convergence_window) ewic = 0;
        else if (!robust && (minLoss - L) > o->convergence_value) ewic = 0;
        else ewic += 1;
        if (o->step_tol > 0) {
            double sn = std::sqrt(d2) / (1.0 + std::sqrt(z2));
            ewis = sn < o->step_tol ? ewis + 1 : 0;
        }
        if (o->grad_tol > 0) {
            double gn = std::sqrt(g2);
            ewig = gn < o->grad_tol ? ewig + 1 : 0;
        }
        int r = GX_STOP_NONE;
        if (ewic > o->patience_convergence) r = GX_STOP_CONVERGENCE;
        else if (L < o->tol) r = GX_STOP_TOL;
        else if (o->step_tol > 0 && ewis > o->patience_step) r = GX_STOP_STEP;
        else if (o->grad_tol > 0 && ewig > o->patience_grad) r = GX_STOP_GRAD;
        if (r != GX_STOP_NONE) { stopped = true; stop_epoch = e; reason = r; }
        return stopped;
    }
};

// ---------------------------------------------------------------------------
// askAdam
// ---------------------------------------------------------------------------
// Checks of the options every askAdam entry point makes: iteration count,
// bounds, and the loss / optimiser / transform enumerations.
static gx_status validate_adam_common(const gx_askadam_opts* o, int np) {
    if (!o) return fail(GX_EINVAL, "opts is NULL");
    if (o->iteration < 0) return fail(GX_EINVAL, "iteration must be >= 0");
    if (!o->lb || !o->ub) return fail(GX_EINVAL, "lb/ub are required");
    for (int k = 0; k < np; ++k)
        if (!(o->ub[k] > o->lb[k])) return fail(GX_EINVAL, "ub[%d] must exceed lb[%d]", k, k);
    if (o->loss < GX_LOSS_L1 || o->loss > GX_LOSS_RICIAN_LOGP) return fail(GX_EINVAL, "unknown loss %d", o->loss);
    if (o->optimiser < GX_OPT_ADAM || o->optimiser > GX_OPT_RMSPROP) return fail(GX_EINVAL, "unknown optimiser %d", o->optimiser);
    if (o->transform != GX_TRANSFORM_SIGMOID && o->transform != GX_TRANSFORM_LINEAR)
        return fail(GX_EINVAL, "unknown parameterTransform %d", o->transform);
    return GX_OK;
}

static gx_status validate_adam(const gx_askadam_opts* o, int np, const gx_volume* vols, int nvol,
                               int nm) {
    if (!o) return fail(GX_EINVAL, "opts is NULL");
    if (!vols || nvol < 1) return fail(GX_EINVAL, "need at least one volume");
    TRY(validate_adam_common(o, np));
    if (o->n_reg < 0 || o->n_reg > kMaxReg) return fail(GX_EINVAL, "n_reg must be in [0, %d]", kMaxReg);
    for (int r = 0; r < o->n_reg; ++r)
        if (o->reg_param[r] < 0 || o->reg_param[r] >= np) return fail(GX_EINVAL, "regmap index %d out of range", o->reg_param[r]);
    if (o->robust_convergence && (o->weight_update_interval < 1 || o->outlier_check_window < 1 ||
                                  o->convergence_window < 1))
        return fail(GX_EINVAL, "robustConvergence needs weightUpdateInterval, outlierCheckWindow and "
                               "convergenceWindow >= 1");
    if (o->reg_type != GX_REG_TV && o->reg_type != GX_REG_PRIOR && o->reg_type != GX_REG_SURFACE_TV)
        return fail(GX_EINVAL, "unknown regularisation type %d", o->reg_type);
    const bool reg = o->n_reg > 0 && o->lambda[0] > 0;
    const bool prior = reg && o->reg_type == GX_REG_PRIOR;
    const bool surf = reg && o->reg_type == GX_REG_SURFACE_TV;
    const bool tv = reg && !prior && !surf;
    if (tv)
        for (int d = 0; d < (o->tv_3d ? 3 : 2); ++d)
            if (!(o->voxel_size[d] > 0)) return fail(GX_EINVAL, "voxel_size must be positive");
    if ((o->loss == GX_LOSS_GAUSS_LOGP || o->loss == GX_LOSS_RICIAN_LOGP) && !(o->sigma > 0)) {
        for (int i = 0; i < nvol; ++i)
            if (!vols[i].sigma) return fail(GX_EINVAL, "likelihood loss needs sigma > 0 or a sigma map");
    }
    for (int i = 0; i < nvol; ++i) {
        const gx_volume& v = vols[i];
        if (v.nvox < 1) return fail(GX_EINVAL, "volume %d: nvox must be >= 1", i);
        if (!v.data) return fail(GX_EINVAL, "volume %d: data is NULL", i);
        if (prior && (!v.prior_mu || !v.prior_sd))
            return fail(GX_EINVAL, "volume %d: the prior regulariser needs prior_mu and prior_sd", i);
        if (surf && (!v.neighbours || !v.edge_length || v.max_neighbours < 1 || v.max_neighbours > 64))
            return fail(GX_EINVAL, "volume %d: surface TV needs neighbours, edge_length and max_neighbours "
                                   "in [1, 64]", i);
        if (tv || surf) {
            if (!v.grid_index) return fail(GX_EINVAL, "volume %d: TV needs grid_index", i);
            long long g = (long long)v.dims[0] * v.dims[1] * v.dims[2];
            if (v.dims[0] < 1 || v.dims[1] < 1 || v.dims[2] < 1 || g < v.nvox || g > (1LL << 31) - 1)
                return fail(GX_EINVAL, "volume %d: bad grid dims", i);
        }
    }
    (void)nm;
    return GX_OK;
}

static bool copy_kind_host(int mem) { return mem == GX_MEM_HOST; }

// Copy a [rows][n] array into a padded [rows][stride] device array at offset off.
static gx_status upload_rows(gx_context* c, float* dst, size_t stride, size_t off, const float* src,
                             int rows, int n, int mem, long long* bytes) {
    cudaMemcpyKind kind = copy_kind_host(mem) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (rows > 0 && n > 0)  // one strided copy of the whole matrix
        CK(cudaMemcpy2DAsync(dst + off, sizeof(float) * stride, src, sizeof(float) * n, sizeof(float) * n, rows,
                             kind, c->stream));
    if (copy_kind_host(mem)) *bytes += (long long)rows * n * sizeof(float);
    return GX_OK;
}

static gx_status download_rows(gx_context* c, float* dst, const float* src, size_t stride, size_t off,
                               int rows, int n, int mem, long long* bytes) {
    if (!dst) return GX_OK;
    cudaMemcpyKind kind = copy_kind_host(mem) ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (rows > 0 && n > 0)
        CK(cudaMemcpy2DAsync(dst, sizeof(float) * n, src + off, sizeof(float) * stride, sizeof(float) * n, rows,
                             kind, c->stream));
    if (copy_kind_host(mem)) *bytes += (long long)rows * n * sizeof(float);
    return GX_OK;
}

static bool cancelled(gx_context* c) { return c->cancel && *c->cancel; }

struct AdamJob {
    gx_context* c;
    const gx_model* model;
    const gx_askadam_opts* o;
    int mem;
    const gx_volume* vols;
    int nvol;
    int np, nm, id;
    int B;
    bool tv, stats, want_min, want_res_f, want_res_m;
    bool prior = false;                   // prior-distribution regulariser (instead of TV)
    bool surf = false;                    // surface TV: TV grids with mesh neighbour tables
    std::vector<DevVol> hv;
    std::vector<int> hblk;
    int nvtot = 0, nblocks = 0;
    long long grid_total = 0;
    long long hgrid_total = 0;            // haloed maps of the persistent kernel (per map)
    int hlayout = 0;                      // their strides (PersistArgs::hlayout)
    float* hgrid[2] = {nullptr, nullptr};
    AdamParams a;
    int ckpt_every = 0, nslots = 0;
    std::vector<double> hist;   // [nvol][N+1][kHistW]
    long long h2d = 0, d2h = 0;
    DevVol* local_vols = nullptr;   // per-volume copies with off = 0 (volume views)
    float* grid[2] = {nullptr, nullptr};  // TV grids, alternating by epoch parity
    PhaseTrace* trace = nullptr;
    float *zr = nullptr, *m1r = nullptr, *m2r = nullptr;  // replay / plain min-loss state
    bool use_persist = false;             // TV main pass as one cooperative launch
    PersistPlan plan{};
    PersistBarrier* barrier = nullptr;
    float4* data_quads = nullptr;         // echo quads of the measurements for the persistent kernel
    bool allow_tune = false;              // gx_askadam with block_size 0: the fused kernel's block is tuned
    bool autotune = false;                // ... and this job tunes it (fused path, no TV)
    int Bl = 0;                           // launch block of the fused kernel's main pass (0: B)
    int* blk_l = nullptr;                 // block -> volume table for Bl
    bool tuned_now = false;               // a trial ran in this call
};

static double sched_pow(double b, int e) { return std::pow(b, (double)e); }

// Mesh neighbour tables of the surface TV, [maxnb][nvtot] in the work-list
// layout; a volume with fewer slots than the widest repeats its own grid
// index (a zero difference) with length 1 in the extra rows.
static gx_status upload_surface(AdamJob& J, int* gidx) {
    gx_context* c = J.c;
    int maxnb = 0;
    for (int i = 0; i < J.nvol; ++i) maxnb = std::max(maxnb, (int)J.vols[i].max_neighbours);
    const size_t nv = J.nvtot;
    int* nb;
    float* len;
    TRY(wsT(c, S_SURF_NB, (size_t)maxnb * nv, &nb));
    TRY(wsT(c, S_SURF_LEN, (size_t)maxnb * nv, &len));
    CK(cudaMemsetAsync(nb, 0, sizeof(int) * maxnb * nv, c->stream));
    CK(cudaMemsetAsync(len, 0, sizeof(float) * maxnb * nv, c->stream));
    const cudaMemcpyKind kind = copy_kind_host(J.mem) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int i = 0; i < J.nvol; ++i) {
        const gx_volume& v = J.vols[i];
        const size_t off = J.hv[i].off;
        for (int j = 0; j < maxnb; ++j) {
            if (j < v.max_neighbours) {
                CK(cudaMemcpyAsync(nb + j * nv + off, v.neighbours + (size_t)j * v.nvox, sizeof(int32_t) * v.nvox,
                                   kind, c->stream));
                TRY(upload_rows(c, len + j * nv, nv, off, v.edge_length + (size_t)j * v.nvox, 1, v.nvox, J.mem,
                                &J.h2d));
                if (J.mem == GX_MEM_HOST) J.h2d += sizeof(int32_t) * v.nvox;
            } else {
                CK(cudaMemcpyAsync(nb + j * nv + off, gidx + off, sizeof(int) * v.nvox, cudaMemcpyDeviceToDevice,
                                   c->stream));
                std::vector<float> ones((size_t)v.nvox, 1.0f);
                CK(cudaMemcpyAsync(len + j * nv + off, ones.data(), sizeof(float) * v.nvox, cudaMemcpyHostToDevice,
                                   c->stream));
                CK(cudaStreamSynchronize(c->stream));
            }
        }
    }
    J.a.surf_nb = nb;
    J.a.surf_len = len;
    J.a.surf_maxnb = maxnb;
    return GX_OK;
}

static gx_status adam_setup(AdamJob& J) {
    gx_context* c = J.c;
    const gx_askadam_opts* o = J.o;
    int N = o->iteration;
    J.prior = o->n_reg > 0 && o->lambda[0] > 0 && o->reg_type == GX_REG_PRIOR;
    J.surf = o->n_reg > 0 && o->lambda[0] > 0 && o->reg_type == GX_REG_SURFACE_TV;
    J.tv = o->n_reg > 0 && o->lambda[0] > 0 && !J.prior;   // grid TV or surface TV
    J.stats = o->step_tol > 0 || o->grad_tol > 0;
    // the fused (no TV) path with block_size 0 tunes its launch block among
    // the divisors of a 512-voxel layout block; every other path lays out and
    // launches with block_size (default 128)
    J.autotune = J.allow_tune && o->block_size == 0 && autotune_enabled() && o->path == GX_PATH_FUSED &&
                 !o->robust_convergence && !J.tv;
    J.B = o->block_size > 0 ? o->block_size : (J.autotune ? kTuneLayoutBlock : 128);
    if (J.B % 32 || J.B < 32 || J.B > 1024) return fail(GX_EINVAL, "block_size must be a multiple of 32 in [32,1024]");
    // work-list layout
    J.hv.resize(J.nvol);
    int off = 0;
    long long goff = 0, hgoff = 0;
    // haloed map layout: power-of-two strides when every volume's x and y
    // extents (with the halo) fit, so that the neighbour offsets are constants
    if (J.tv) {
        int dmax = 0, zmax = 0;
        for (int i = 0; i < J.nvol; ++i) {
            dmax = std::max(dmax, std::max(J.vols[i].dims[0], J.vols[i].dims[1]) + 2);
            zmax = std::max(zmax, J.vols[i].dims[2] + 2);
        }
        J.hlayout = dmax <= 128 && zmax <= (1 << 16) ? 7
                    : dmax <= 256 && zmax <= (1 << 14) ? 8
                    : dmax <= 512 && zmax <= (1 << 12) ? 9 : 0;
    }
    for (int i = 0; i < J.nvol; ++i) {
        const gx_volume& v = J.vols[i];
        DevVol& d = J.hv[i];
        memset(&d, 0, sizeof(d));
        d.off = off;
        d.nvox = v.nvox;
        d.npad = (v.nvox + J.B - 1) / J.B * J.B;
        d.normd = 1.0 / ((double)J.nm * (double)v.nvox);
        d.norm = (float)d.normd;
        for (int q = 0; q < 3; ++q) d.dims[q] = J.tv ? v.dims[q] : (q == 0 ? v.nvox : 1);
        d.grid_off = goff;
        d.hgrid_off = hgoff;
        for (int r = 0; r < o->n_reg && r < kMaxReg; ++r) d.tv_scale[r] = (float)(o->lambda[r] / (double)v.nvox);
        d.prior_off = J.prior ? (float)v.prior_offset : 0.0f;
        if (J.tv) {
            goff += (long long)v.dims[0] * v.dims[1] * v.dims[2];
            hgoff += J.hlayout > 0 ? (long long)(v.dims[2] + 2) << (2 * J.hlayout)
                                   : (long long)(v.dims[0] + 2) * (v.dims[1] + 2) * (v.dims[2] + 2);
        }
        for (int b = 0; b < d.npad / J.B; ++b) J.hblk.push_back(i);
        off += d.npad;
    }
    J.nvtot = off;
    J.nblocks = off / J.B;
    J.grid_total = goff;
    J.hgrid_total = hgoff;

    AdamParams& a = J.a;
    memset(&a, 0, sizeof(a));
    a.P = make_protocol(J.model, J.id, J.np, J.nm, o->lb, o->ub, J.np);
    a.nm = J.nm;
    a.np = J.np;
    a.nvtot = J.nvtot;
    a.nvol = J.nvol;
    a.niter = N;
    a.optimiser = o->optimiser;
    a.transform = o->transform;
    a.beta1 = (float)o->beta1; a.beta2 = (float)o->beta2; a.eps = (float)o->epsilon;
    a.momentum = (float)o->momentum; a.rms_decay = (float)o->rms_decay; a.rms_eps = (float)o->rms_epsilon;
    a.mse_scale = (float)o->mse_scale;
    a.huber_delta = (float)o->huber_delta;
    a.sigma_default = (float)o->sigma;
    a.n_reg = (J.tv || J.prior) ? o->n_reg : 0;
    for (int r = 0; r < a.n_reg; ++r) a.reg_param[r] = o->reg_param[r];
    a.tv_3d = o->tv_3d;
    for (int d = 0; d < 3; ++d) a.inv_vs[d] = o->voxel_size[d] > 0 ? (float)(1.0 / o->voxel_size[d]) : 0.0f;
    a.grid_total = J.grid_total;

    size_t nv = J.nvtot;
    bool anyw = false, anyb1 = false, anysig = false, anyth0 = false;
    for (int i = 0; i < J.nvol; ++i) {
        anyw |= J.vols[i].weights != nullptr;
        anyb1 |= J.vols[i].b1 != nullptr;
        anysig |= J.vols[i].sigma != nullptr;
        anyth0 |= J.vols[i].theta0 != nullptr;
    }
    float *data, *w = nullptr, *b1 = nullptr, *sig = nullptr, *th0 = nullptr;
    TRY(wsT(c, S_DATA, (size_t)J.nm * nv, &data));
    CK(cudaMemsetAsync(data, 0, sizeof(float) * J.nm * nv, c->stream));
    if (anyw) {
        TRY(wsT(c, S_W, (size_t)J.nm * nv, &w));
        CK(cudaMemsetAsync(w, 0, sizeof(float) * J.nm * nv, c->stream));
    }
    if (anyb1) TRY(wsT(c, S_B1, nv, &b1));
    if (anysig) TRY(wsT(c, S_SIG, nv, &sig));
    if (anyth0) TRY(wsT(c, S_TH0, (size_t)J.np * nv, &th0));
    for (int i = 0; i < J.nvol; ++i) {
        const gx_volume& v = J.vols[i];
        const DevVol& d = J.hv[i];
        TRY(upload_rows(c, data, nv, d.off, v.data, J.nm, v.nvox, J.mem, &J.h2d));
        if (anyw) {
            if (v.weights) TRY(upload_rows(c, w, nv, d.off, v.weights, J.nm, v.nvox, J.mem, &J.h2d));
            else {
                std::vector<float> ones((size_t)v.nvox, 1.0f);
                for (int m = 0; m < J.nm; ++m)
                    CK(cudaMemcpyAsync(w + (size_t)m * nv + d.off, ones.data(), sizeof(float) * v.nvox, cudaMemcpyHostToDevice, c->stream));
                CK(cudaStreamSynchronize(c->stream));
            }
        }
        if (anyb1) {
            if (v.b1) TRY(upload_rows(c, b1, nv, d.off, v.b1, 1, v.nvox, J.mem, &J.h2d));
            else {
                std::vector<float> ones((size_t)v.nvox, 1.0f);
                CK(cudaMemcpyAsync(b1 + d.off, ones.data(), sizeof(float) * v.nvox, cudaMemcpyHostToDevice, c->stream));
                CK(cudaStreamSynchronize(c->stream));
            }
        }
        if (anysig) {
            if (v.sigma) TRY(upload_rows(c, sig, nv, d.off, v.sigma, 1, v.nvox, J.mem, &J.h2d));
            else {
                std::vector<float> s((size_t)v.nvox, (float)o->sigma);
                CK(cudaMemcpyAsync(sig + d.off, s.data(), sizeof(float) * v.nvox, cudaMemcpyHostToDevice, c->stream));
                CK(cudaStreamSynchronize(c->stream));
            }
        }
        if (anyth0 && v.theta0) TRY(upload_rows(c, th0, nv, d.off, v.theta0, J.np, v.nvox, J.mem, &J.h2d));
    }
    if (J.prior) {
        // mean and SD maps of the regularised parameters; padding voxels get 0 / 0
        float *mu, *sd;
        TRY(wsT(c, S_PRIOR_MU, (size_t)o->n_reg * nv, &mu));
        TRY(wsT(c, S_PRIOR_SD, (size_t)o->n_reg * nv, &sd));
        CK(cudaMemsetAsync(mu, 0, sizeof(float) * o->n_reg * nv, c->stream));
        CK(cudaMemsetAsync(sd, 0, sizeof(float) * o->n_reg * nv, c->stream));
        for (int i = 0; i < J.nvol; ++i) {
            const gx_volume& v = J.vols[i];
            TRY(upload_rows(c, mu, nv, J.hv[i].off, v.prior_mu, o->n_reg, v.nvox, J.mem, &J.h2d));
            TRY(upload_rows(c, sd, nv, J.hv[i].off, v.prior_sd, o->n_reg, v.nvox, J.mem, &J.h2d));
        }
        a.prior_mu = mu;
        a.prior_sd = sd;
    }
    a.data = data; a.weights = w; a.b1 = b1; a.sigma = sig;
    if (J.trace) J.trace->mark("upload");
    TRY(wsT(c, S_Z, (size_t)J.np * nv, &a.z));
    TRY(wsT(c, S_M1, (size_t)J.np * nv, &a.m1));
    TRY(wsT(c, S_M2, (size_t)J.np * nv, &a.m2));
    if (J.stats || J.prior) TRY(wsT(c, S_ZP, (size_t)J.np * nv, &a.zprev));
    int* blk;
    DevVol* dvols;
    TRY(wsT(c, S_BLK, J.hblk.size(), &blk));
    TRY(wsT(c, S_VOLS, 2 * J.hv.size(), &dvols));
    // block map, volume table (+ per-volume copies with off = 0) and the
    // optimiser schedule staged in the context's pinned buffer: three queued copies
    const size_t nblk = J.hblk.size(), nvt = 2 * J.hv.size();
    const size_t o_vols = (sizeof(int) * nblk + 15) / 16 * 16;
    const size_t o_sched = o_vols + (sizeof(DevVol) * nvt + 15) / 16 * 16;
    // every destination exists before the stage is filled, so that no return
    // path leaves copies out of the stage queued without pin_ev behind them
    float2* dsched;
    TRY(wsT(c, S_SCHED, (size_t)N + 1, &dsched));
    unsigned char* stage;
    TRY(pinned(c, o_sched + sizeof(float2) * ((size_t)N + 1), (void**)&stage));
    memcpy(stage, J.hblk.data(), sizeof(int) * nblk);
    DevVol* sv = reinterpret_cast<DevVol*>(stage + o_vols);
    for (size_t i = 0; i < J.hv.size(); ++i) {
        sv[i] = J.hv[i];
        sv[J.hv.size() + i] = J.hv[i];
        sv[J.hv.size() + i].off = 0;
    }
    J.local_vols = dvols + J.hv.size();
    a.blk_vol = blk;
    a.vols = dvols;
    // optimiser schedule per epoch (update_learn_rate :1180-1183, adamupdate bias correction)
    float2* sched = reinterpret_cast<float2*>(stage + o_sched);
    sched[0] = float2{0.f, 0.f};
    for (int e = 1; e <= N; ++e) {
        double lr = o->initial_learn_rate / (1.0 + o->decay_rate * (e - 1));
        if (o->optimiser == GX_OPT_ADAM)
            sched[e] = float2{(float)(lr / (1.0 - sched_pow(o->beta1, e))), (float)(1.0 / (1.0 - sched_pow(o->beta2, e)))};
        else
            sched[e] = float2{(float)lr, 0.f};
    }
    {
        // the three copies out of the stage; pin_ev is recorded behind them
        // even when one fails, so the next call's pinned() waits for the
        // copies that were queued
        cudaError_t e = cudaMemcpyAsync(blk, stage, sizeof(int) * nblk, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dvols, sv, sizeof(DevVol) * nvt, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dsched, sched, sizeof(float2) * ((size_t)N + 1), cudaMemcpyHostToDevice, c->stream);
        const cudaError_t er = cudaEventRecord(c->pin_ev, c->stream);
        if (e == cudaSuccess && er != cudaSuccess) e = er;
        if (e != cudaSuccess) {
            if (er != cudaSuccess) cudaStreamSynchronize(c->stream);  // no event: drain instead
            CK(e);
        }
    }
    a.sched = dsched;
    TRY(wsT(c, S_HIST, (size_t)J.nvol * (N + 1) * kHistW, &a.hist));
    CK(cudaMemsetAsync(a.hist, 0, sizeof(double) * J.nvol * (N + 1) * kHistW, c->stream));
    // checkpoints: slot c holds the state after c*ckpt_every updates, every
    // 16 updates within a budget of min(4 GB, free/4); free memory is only
    // queried when the context's buffer cannot already hold that plan (the
    // query can stall for milliseconds on a shared device)
    size_t slot_bytes = sizeof(float) * 3 * (size_t)J.np * nv;
    const size_t cap4 = (size_t)4 << 30;
    int K = 16;
    const size_t want16 = ((size_t)(N / 16) + 1) * slot_bytes;
    if (!(want16 <= cap4 && c->cap[S_CKPT] >= want16)) {
        size_t budget = cap4;
        size_t freeb = 0, totalb = 0;
        if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess && freeb / 4 < budget) budget = freeb / 4;
        long long max_slots = budget / slot_bytes;
        if (max_slots < 2) max_slots = 2;
        while ((long long)(N / K) + 1 > max_slots) K *= 2;
    }
    J.ckpt_every = K;
    J.nslots = N / K + 1;
    TRY(wsT(c, S_CKPT, (size_t)J.nslots * 3 * J.np * nv, &a.ckpt));
    a.ckpt_every = K;
    if (J.trace) J.trace->mark("tables");
    // TV grids and masks
    if (J.tv) {
        int* gidx;
        unsigned char* mk;
        float *g0, *g1;
        TRY(wsT(c, S_GIDX, nv, &gidx));
        TRY(wsT(c, S_MASK, ((size_t)J.grid_total + 3) & ~(size_t)3, &mk));  // word-aligned for the mask kernel
        TRY(wsT(c, S_GRID0, (size_t)a.n_reg * J.grid_total, &g0));
        TRY(wsT(c, S_GRID1, (size_t)a.n_reg * J.grid_total, &g1));
        CK(cudaMemsetAsync(gidx, 0, sizeof(int) * nv, c->stream));
        CK(cudaMemsetAsync(g0, 0, sizeof(float) * a.n_reg * J.grid_total, c->stream));
        CK(cudaMemsetAsync(g1, 0, sizeof(float) * a.n_reg * J.grid_total, c->stream));
        CK(cudaMemsetAsync(mk, 0, ((size_t)J.grid_total + 3) & ~(size_t)3, c->stream));
        const cudaMemcpyKind kind = copy_kind_host(J.mem) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
        for (int i = 0; i < J.nvol; ++i) {
            const gx_volume& v = J.vols[i];
            CK(cudaMemcpyAsync(gidx + J.hv[i].off, v.grid_index, sizeof(int32_t) * v.nvox, kind, c->stream));
            if (J.mem == GX_MEM_HOST) J.h2d += sizeof(int32_t) * v.nvox;
        }
        a.gidx = gidx;
        a.maskgrid = mk;
        if (J.surf) TRY(upload_surface(J, gidx));
        // mask grid and index checks on the device
        int* flags;
        TRY(wsT(c, S_FLAGS, 2, &flags));
        const int init[2] = {0, 0x7fffffff};
        CK(cudaMemcpyAsync(flags, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
        CK(launch_tv_mask(a, mk, flags, flags + 1, J.B, J.nblocks, c->stream));
        int hf[2];
        CK(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (hf[0] & 1) return fail(GX_EINVAL, "volume %d: grid_index out of range", hf[1]);
        if (hf[0] & 2) return fail(GX_EINVAL, "volume %d: duplicate grid_index", hf[1]);
        if (hf[0] & 4) return fail(GX_EINVAL, "volume %d: mesh neighbour index out of range", hf[1]);
        a.grid_cur = g0;
        a.grid_next = g1;
        J.grid[0] = g0;
        J.grid[1] = g1;
    }
    if (J.trace) J.trace->mark("tv_grid");
    // initial state + checkpoint slot 0
    CK(launch_init_state(a, anyth0 ? th0 : nullptr, o->randomness, o->seed, J.B, c->stream));
    if (anyth0) {
        // volumes without theta0 start from the no-start-point initialisation
        for (int i = 0; i < J.nvol; ++i)
            if (!J.vols[i].theta0) return fail(GX_EUNSUPPORTED, "mixing volumes with and without theta0");
    }
    CK(launch_copy_state(a, a.ckpt, a.z, a.m1, a.m2, true, J.B, J.nblocks, c->stream));
    if (J.trace) J.trace->mark("init");
    return GX_OK;
}

// A view of the work-list restricted to one volume: pointers are offset to
// the volume's first (padded) voxel and the volume table entry has off = 0,
// so every kernel runs unchanged on that volume alone.
struct View {
    AdamParams a;
    int nblocks;
};

static gx_status make_view(AdamJob& J, int i, const AdamParams& base, View* out) {
    const DevVol& d = J.hv[i];
    AdamParams a = base;
    size_t o = d.off;
    a.data += o;
    if (a.weights) a.weights += o;
    if (a.b1) a.b1 += o;
    if (a.sigma) a.sigma += o;
    a.z += o; a.m1 += o; a.m2 += o;
    if (a.zprev) a.zprev += o;
    if (a.ckpt) a.ckpt += o;
    if (a.gidx) a.gidx += o;
    if (a.prior_mu) { a.prior_mu += o; a.prior_sd += o; }
    if (a.surf_nb) { a.surf_nb += o; a.surf_len += o; }
    a.blk_vol += d.off / J.B;
    a.vols = J.local_vols;
    out->a = a;
    out->nblocks = d.npad / J.B;
    return GX_OK;
}

// Run epochs [e0, e1] on the (sub)list described by `a` (TV: one launch per
// epoch, alternating the two grids by epoch parity).
static gx_status run_epochs(AdamJob& J, AdamParams a, int nblocks, int e0, int e1, int update_last,
                            bool record, float* res_out, bool persistent_ok = false) {
    gx_context* c = J.c;
    a.res_out = res_out;
    if (!record) a.hist = nullptr;
    if (!J.tv) {
        // the main pass (the whole work-list) launches with the tuned block
        int B = J.B;
        if (J.Bl > 0 && a.blk_vol == J.a.blk_vol && nblocks == J.nblocks) {
            B = J.Bl;
            nblocks = J.nvtot / J.Bl;
            a.blk_vol = J.blk_l;
        }
        // the prior's loss is recorded in the statistics columns of the history
        CK(launch_fused(a, J.id, J.o->loss, (J.stats || J.prior) && record, e0, e1, update_last, record, B,
                        nblocks, c->stream));
        return GX_OK;
    }
    if (persistent_ok && J.use_persist) {
        PersistArgs p;
        memset(&p, 0, sizeof(p));
        p.e_begin = e0;
        p.e_end = e1;
        p.update_last = update_last;
        p.record = record ? 1 : 0;
        p.want_res = res_out != nullptr;
        p.stats = (J.stats && record) ? 1 : 0;
        p.loss = J.o->loss;
        p.grid0 = J.hgrid[0];
        p.grid1 = J.hgrid[1];
        p.hgrid_total = J.hgrid_total;
        p.hlayout = J.hlayout;
        p.barrier = J.barrier;
        p.pad_block = J.B;
        p.data_quads = J.data_quads;
        p.spin_cycles = c->hooks.wait_limit_cycles > 0 ? c->hooks.wait_limit_cycles : kBarrierSpinCycles;
        p.extra_arrivals = (unsigned int)c->hooks.barrier_extra_arrivals;
        CK(cudaMemsetAsync(J.barrier, 0, sizeof(PersistBarrier), c->stream));
        CK(launch_tv_persistent(a, J.plan, p, c->stream));
        return GX_OK;
    }
    float* g[2] = {J.grid[0], J.grid[1]};
    for (int e = e0; e <= e1; ++e) {
        a.grid_cur = g[e >= 1 ? (e - 1) & 1 : 0];  // epoch 0 evaluates the start, like epoch 1
        a.grid_next = g[e & 1];
        CK(launch_tv_step(a, J.id, J.o->loss, J.stats && record, e, e <= update_last, record,
                          e == e1 && res_out != nullptr, J.B, nblocks, c->stream));
        if ((e & 63) == 0 && cancelled(c)) return fail(GX_ECANCELLED, "cancelled");
    }
    return GX_OK;
}

// Rebuild, for volume i, the state after `target` updates into the replay
// buffers (J.zr, J.m1r, J.m2r), the residuals at it into res_out (may be
// NULL) and theta into th_out (padded layout, rows of the volume only).
static gx_status replay_volume(AdamJob& J, int i, int target, float* th_out, float* res_out) {
    gx_context* c = J.c;
    AdamParams base = J.a;
    base.z = J.zr; base.m1 = J.m1r; base.m2 = J.m2r;
    base.zprev = nullptr;
    base.ckpt_every = 0;
    View V;
    TRY(make_view(J, i, base, &V));
    int slot = target / J.ckpt_every;
    float* src = J.a.ckpt + (size_t)slot * 3 * J.np * J.nvtot + J.hv[i].off;
    V.a.ckpt = nullptr;
    CK(launch_copy_state(V.a, src, nullptr, nullptr, nullptr, false, J.B, V.nblocks, c->stream));
    int e0 = slot * J.ckpt_every + 1;
    // a job of one volume replays through the cooperative TV kernel (its plan
    // covers exactly this view; it computes bit for bit what the per-epoch
    // kernel does, and writes its own start map); a view of a larger job runs
    // one launch per epoch, from the map of its start state
    const bool persist = J.nvol == 1 && J.use_persist;
    if (J.tv && !persist) CK(launch_tv_scatter(V.a, J.grid[(e0 - 1) & 1], J.B, V.nblocks, c->stream));  // e0 >= 1
    size_t o = J.hv[i].off;
    TRY(run_epochs(J, V.a, V.nblocks, e0, target + 1, target, false, res_out ? res_out + o : nullptr,
                   J.nvol == 1));
    CK(launch_finalize(V.a, V.a.z, th_out + o, nullptr, nullptr, J.B, V.nblocks, c->stream));
    return GX_OK;
}

struct AdamOut {
    std::vector<Tracker> tr;
    std::vector<int> final_epoch;
    float *thf = nullptr, *thm = nullptr, *resf = nullptr, *resm = nullptr;
};

static gx_status alloc_outputs(AdamJob& J, AdamOut& out) {
    gx_context* c = J.c;
    size_t pn = (size_t)J.np * J.nvtot, mn = (size_t)J.nm * J.nvtot;
    TRY(wsT(c, S_THF, pn, &out.thf));
    TRY(wsT(c, S_THM, pn, &out.thm));
    if (J.want_res_f) TRY(wsT(c, S_RESF, mn, &out.resf));
    if (J.want_res_m) TRY(wsT(c, S_RESM, mn, &out.resm));
    TRY(wsT(c, S_ZR, pn, &J.zr));
    TRY(wsT(c, S_M1R, pn, &J.m1r));
    TRY(wsT(c, S_M2R, pn, &J.m2r));
    return GX_OK;
}

static bool can_stop(const gx_askadam_opts* o) {
    bool signed_loss = o->loss == GX_LOSS_GAUSS_LOGP || o->loss == GX_LOSS_RICIAN_LOGP;
    return std::isfinite(o->patience_convergence) || o->step_tol > 0 || o->grad_tol > 0 ||
           o->tol > 0 || (signed_loss && o->tol > -INFINITY);
}

// Block -> volume table of launch block Bl (a divisor of the layout block B).
static gx_status upload_blk_table(AdamJob& J, int Bl, int** out) {
    const int k = J.B / Bl;
    std::vector<int> t(J.hblk.size() * (size_t)k);
    for (size_t b = 0; b < J.hblk.size(); ++b)
        for (int j = 0; j < k; ++j) t[b * k + j] = J.hblk[b];
    TRY(wsT(J.c, S_BLK_L, t.size(), out));
    CK(cudaMemcpyAsync(*out, t.data(), sizeof(int) * t.size(), cudaMemcpyHostToDevice, J.c->stream));
    CK(cudaStreamSynchronize(J.c->stream));  // t is freed on return
    return GX_OK;
}

// Autotuner of the fused kernel's launch block.  Key: device, model, loss,
// measurements, statistics / prior / weights / b1 / sigma-map variants,
// optimiser, transform and the voxel-count class (log2 of the work-list).
// On a miss every candidate (64, 128, 256, 512 threads, and 32 for short
// work-lists, within the kernel's thread and shared-memory limits) runs a
// few epochs of this job's own
// kernel on its own data from a scratch copy of the start state (the job's
// state and history untouched); the fastest is cached for the process.
static gx_status tune_fused(AdamJob& J) {
    gx_context* c = J.c;
    const gx_askadam_opts* o = J.o;
    const bool stats = J.stats || J.prior;
    int cls = 0;
    while ((1LL << (cls + 1)) <= (long long)J.nvtot) ++cls;
    const TuneKey key{{1, c->device, J.id, o->loss, J.nm, stats ? 1 : 0, J.prior ? 1 : 0, J.a.weights ? 1 : 0,
                       J.a.b1 ? 1 : 0, J.a.sigma ? 1 : 0, o->optimiser, o->transform, cls}};
    int Bl = o->iteration < 2 ? 128 : tune_lookup(key);  // trials need two epochs of history rows
    if (Bl <= 0) {
        const int N = o->iteration;
        AdamParams t = J.a;
        const size_t pn = (size_t)J.np * J.nvtot;
        float* sc;
        TRY(wsT(c, S_TUNE, 4 * pn, &sc));
        t.z = sc; t.m1 = sc + pn; t.m2 = sc + 2 * pn; t.zprev = J.a.zprev ? sc + 3 * pn : nullptr;
        CK(cudaMemcpyAsync(t.z, J.a.z, sizeof(float) * pn, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaMemcpyAsync(t.m1, J.a.m1, sizeof(float) * pn, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaMemcpyAsync(t.m2, J.a.m2, sizeof(float) * pn, cudaMemcpyDeviceToDevice, c->stream));
        if (t.zprev) CK(cudaMemcpyAsync(t.zprev, J.a.zprev, sizeof(float) * pn, cudaMemcpyDeviceToDevice, c->stream));
        TRY(wsT(c, S_TUNE_HIST, (size_t)J.nvol * (N + 1) * kHistW, &t.hist));
        t.ckpt = nullptr;
        t.ckpt_every = 0;
        t.res_out = nullptr;
        // epochs per trial: about 1 ms of work (at least 2), so that the
        // kernel's one-time staging of the measurements is amortised as in a fit
        int E = 1;
        {
            int* blk;
            TRY(upload_blk_table(J, 128, &blk));
            t.blk_vol = blk;
            float m = 0.f;
            for (int rep = 0; rep < 2; ++rep) {
                CK(cudaEventRecord(c->ev[2], c->stream));
                CK(launch_fused(t, J.id, o->loss, stats, 1, 1, 0, true, 128, J.nvtot / 128, c->stream));
                CK(cudaEventRecord(c->ev[3], c->stream));
                CK(cudaEventSynchronize(c->ev[3]));
                cudaEventElapsedTime(&m, c->ev[2], c->ev[3]);
            }
            E = (int)std::min(64.0, std::max(2.0, 1.0 / std::max((double)m, 1e-3)));
            E = std::max(1, std::min(E, N));
        }
        float best = 0.f;
        for (int cand : {32, 64, 128, 256, 512}) {
            // one-warp blocks only for work-lists that leave SMs idle with 64-thread blocks
            if (cand == 32 && J.nvtot > 64 * 148) continue;
            if (J.B % cand || fused_block_limit(t, J.id, o->loss, stats) < cand) continue;
            int* blk;
            TRY(upload_blk_table(J, cand, &blk));
            t.blk_vol = blk;
            float ms = 0.f;
            for (int rep = 0; rep < 3; ++rep) {  // the first run warms the code and caches
                CK(cudaEventRecord(c->ev[2], c->stream));
                CK(launch_fused(t, J.id, o->loss, stats, 1, E, E - 1, true, cand, J.nvtot / cand, c->stream));
                CK(cudaEventRecord(c->ev[3], c->stream));
                CK(cudaEventSynchronize(c->ev[3]));
                float m = 0.f;
                cudaEventElapsedTime(&m, c->ev[2], c->ev[3]);
                if (rep == 1 || (rep > 1 && m < ms)) ms = m;
            }
            if (Bl <= 0 || ms < best) { best = ms; Bl = cand; }
        }
        if (Bl <= 0) return fail(GX_ECUDA, "autotuner: no launch block fits the fused kernel");
        tune_store(key, Bl);
        J.tuned_now = true;
    }
    J.Bl = Bl;
    TRY(upload_blk_table(J, Bl, &J.blk_l));
    return GX_OK;
}

static gx_status adam_fused(AdamJob& J, AdamOut& out) {
    gx_context* c = J.c;
    const gx_askadam_opts* o = J.o;
    const int N = o->iteration;
    const bool stop_possible = can_stop(o);
    const int chunk = stop_possible ? (o->chunk > 0 ? o->chunk : 200) : (N > 0 ? N : 1);
    TRY(alloc_outputs(J, out));
    if (J.autotune) TRY(tune_fused(J));
    if (J.tv) {
        const char* env = getenv("GACELLE_B200_TV_KERNEL");
        bool want = !(env && strcmp(env, "step") == 0);
        std::vector<int> npad(J.nvol);
        for (int i = 0; i < J.nvol; ++i) {
            npad[i] = J.hv[i].npad;
            const gx_volume& v = J.vols[i];
            // map positions are 32-bit in the persistent kernel
            if ((long long)(v.dims[0] + 2) * (v.dims[1] + 2) * (v.dims[2] + 2) >= (1LL << 31)) want = false;
        }
        J.use_persist = want && !J.surf &&
                        plan_persistent(J.a, J.id, o->loss, J.stats, J.B, npad.data(), J.nvol, &J.plan);
        if (J.use_persist) {
            TRY(wsT(c, S_BAR, 1, &J.barrier));
            const size_t hn = (size_t)J.a.n_reg * J.hgrid_total;
            TRY(wsT(c, S_HGRID0, hn, &J.hgrid[0]));
            TRY(wsT(c, S_HGRID1, hn, &J.hgrid[1]));
            CK(cudaMemsetAsync(J.hgrid[0], 0, sizeof(float) * hn, c->stream));
            CK(cudaMemsetAsync(J.hgrid[1], 0, sizeof(float) * hn, c->stream));
        }
        if (J.use_persist && J.plan.quad_width > 0) {
            TRY(wsT(c, S_DATA_QUADS, (size_t)J.nvtot * (J.plan.quad_width / 4), &J.data_quads));
            CK(launch_echo_quads(J.a.data, J.nm, J.nvtot, J.plan.quad_width, J.plan.quad_pairs != 0, J.data_quads,
                                 c->stream));
        }
        // the per-epoch kernel reads the start map from the plain grid (the
        // persistent kernel writes its own)
        if (!J.use_persist) CK(launch_tv_scatter(J.a, J.grid[0], J.B, J.nblocks, c->stream));
    }

    out.tr.assign(J.nvol, Tracker());
    out.final_epoch.assign(J.nvol, N);
    J.hist.assign((size_t)J.nvol * (N + 1) * kHistW, 0.0);
    std::vector<bool> started(J.nvol, false);
    int n_main = 0;
    if (J.trace) J.trace->mark("plan");
    CK(cudaEventRecord(c->ev[2], c->stream));
    if (N == 0) {
        TRY(run_epochs(J, J.a, J.nblocks, 0, 0, -1, true, out.resf, true));
        ++n_main;
    } else {
        bool all_stopped = false;
        for (int eb = 1; eb <= N && !all_stopped; eb += chunk) {
            int ee = std::min(eb + chunk - 1, N);
            TRY(run_epochs(J, J.a, J.nblocks, eb, ee, std::min(ee, N - 1), true, ee == N ? out.resf : nullptr,
                           true));
            n_main += (J.tv && !J.use_persist) ? (ee - eb + 1) : 1;
            if (cancelled(c)) return fail(GX_ECANCELLED, "cancelled");
            if (!stop_possible) continue;
            CK(cudaStreamSynchronize(c->stream));
            all_stopped = true;
            for (int i = 0; i < J.nvol; ++i) {
                size_t base = (size_t)i * (N + 1) * kHistW;
                CK(cudaMemcpy(J.hist.data() + base + (size_t)eb * kHistW, J.a.hist + base + (size_t)eb * kHistW,
                              sizeof(double) * (ee - eb + 1) * kHistW, cudaMemcpyDeviceToHost));
                Tracker& t = out.tr[i];
                if (!started[i]) {
                    t.init(o, J.hist[base + kHistW], J.hist[base + kHistW + 1]);
                    started[i] = true;
                }
                for (int e = eb; e <= ee && !t.stopped; ++e) {
                    const double* h = J.hist.data() + base + (size_t)e * kHistW;
                    t.epoch(e, h[0], h[1], h[2], h[3], h[4]);
                }
                all_stopped = all_stopped && t.stopped;
            }
        }
    }
    CK(cudaEventRecord(c->ev[3], c->stream));
    if (!stop_possible || N == 0) {
        CK(cudaMemcpyAsync(J.hist.data(), J.a.hist, sizeof(double) * J.hist.size(), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < J.nvol; ++i) {
            size_t base = (size_t)i * (N + 1) * kHistW;
            Tracker& t = out.tr[i];
            if (N == 0) {
                t.init(o, J.hist[base], J.hist[base + 1]);
                continue;
            }
            t.init(o, J.hist[base + kHistW], J.hist[base + kHistW + 1]);
            for (int e = 1; e <= N && !t.stopped; ++e) {
                const double* h = J.hist.data() + base + (size_t)e * kHistW;
                t.epoch(e, h[0], h[1], h[2], h[3], h[4]);
            }
        }
    }
    CK(cudaEventSynchronize(c->ev[3]));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
    c->timing.main_kernel_ms = ms;
    c->timing.main_launches = n_main;
    c->timing.block_size = J.Bl > 0 ? J.Bl : (J.use_persist ? J.plan.threads : J.B);
    c->timing.autotuned = J.tuned_now ? 1 : 0;
    c->timing.tv_path = !J.use_persist ? 0
                        : GX_TV_PERSISTENT | (J.plan.quad_pairs ? GX_TV_PAIRS : 0) |
                              (J.plan.data_in_smem ? GX_TV_DATA_SMEM : 0) | (J.data_quads ? GX_TV_DATA_QUADS : 0);
    if (J.use_persist) {
        PersistBarrier hb;
        CK(cudaMemcpy(&hb, J.barrier, sizeof(hb), cudaMemcpyDeviceToHost));
        if (hb.error) return fail(GX_ETIMEOUT, "askAdam TV kernel: a grid barrier wait expired");
    }
    for (int i = 0; i < J.nvol && N > 0; ++i) {  // the initial evaluation equals epoch 1's
        size_t base = (size_t)i * (N + 1) * kHistW;
        for (int q = 0; q < kHistW; ++q) J.hist[base + q] = J.hist[base + kHistW + q];
    }
    for (int i = 0; i < J.nvol; ++i)
        if (out.tr[i].stopped) out.final_epoch[i] = out.tr[i].stop_epoch;

    if (J.trace) J.trace->mark("main");
    // final state: the live z holds z_{N-1}; volumes that stopped at e* are replayed to z_{e*-1}
    CK(launch_finalize(J.a, J.a.z, out.thf, nullptr, nullptr, J.B, J.nblocks, c->stream));
    for (int i = 0; i < J.nvol; ++i)
        if (out.final_epoch[i] != N) TRY(replay_volume(J, i, std::max(out.final_epoch[i] - 1, 0), out.thf, out.resf));
    // minimum-loss state (z_{minIter-1}); equal to the final state when the loss never rose
    for (int i = 0; i < J.nvol; ++i) {
        int tmin = std::max(out.tr[i].minIter - 1, 0);
        int tfin = std::max(out.final_epoch[i] - 1, 0);
        const DevVol& d = J.hv[i];
        if (tmin == tfin && out.tr[i].minIter == out.final_epoch[i]) {
            for (int k = 0; k < J.np; ++k)
                CK(cudaMemcpyAsync(out.thm + (size_t)k * J.nvtot + d.off, out.thf + (size_t)k * J.nvtot + d.off,
                                   sizeof(float) * d.npad, cudaMemcpyDeviceToDevice, c->stream));
            if (out.resm && out.resf)
                for (int m = 0; m < J.nm; ++m)
                    CK(cudaMemcpyAsync(out.resm + (size_t)m * J.nvtot + d.off, out.resf + (size_t)m * J.nvtot + d.off,
                                       sizeof(float) * d.npad, cudaMemcpyDeviceToDevice, c->stream));
        } else {
            TRY(replay_volume(J, i, tmin, out.thm, out.resm));
        }
    }
    if (J.trace) J.trace->mark("final_min");
    return GX_OK;
}

// Plain path: op-by-op kernels, one volume at a time, with the loss read back
// every epoch and the reference's bookkeeping run on the host in the loop.
static gx_status adam_plain(AdamJob& J, AdamOut& out) {
    gx_context* c = J.c;
    const gx_askadam_opts* o = J.o;
    const int N = o->iteration;
    TRY(alloc_outputs(J, out));
    size_t pn = (size_t)J.np * J.nvtot, mn = (size_t)J.nm * J.nvtot;
    PlainBufs pb;
    TRY(wsT(c, S_P_TH, pn, &pb.theta));
    TRY(wsT(c, S_P_DTH, pn, &pb.dth));
    TRY(wsT(c, S_P_SIG, mn, &pb.signal));
    TRY(wsT(c, S_P_DSIG, mn, &pb.dsig));
    TRY(wsT(c, S_P_RES, mn, &pb.res));
    TRY(wsT(c, S_P_GTH, pn, &pb.gth));
    TRY(wsT(c, S_P_GZ, pn, &pb.gz));
    TRY(wsT(c, S_P_ACC, 8, &pb.acc));
    pb.r = RobustBufs{};
    const bool robust = o->robust_convergence != 0;
    const int RW = robust ? o->outlier_check_window : 0;
    RobustOpts ro{(float)o->outlier_weight, (float)o->outlier_voxel_thres, (float)o->outlier_pop_thres,
                  (float)o->outlier_init_thres, (float)o->outlier_init_pop_thres};
    if (robust) {
        const size_t nv = J.nvtot;
        auto al = [](size_t b) { return (b + 255) / 256 * 256; };
        size_t of[11];
        of[0] = 0;
        of[1] = of[0] + al(sizeof(float) * nv);              // vmod
        of[2] = of[1] + al(sizeof(float) * nv);              // vloss
        of[3] = of[2] + al(sizeof(float) * nv);              // vinit
        of[4] = of[3] + al(sizeof(float) * nv * RW);         // ring
        of[5] = of[4] + al(sizeof(float) * nv);              // imp_a
        of[6] = of[5] + al(sizeof(float) * nv);              // imp_b
        of[7] = of[6] + al(sizeof(int) * nv);                // flagcnt
        of[8] = of[7] + al(nv);                              // mainmask
        of[9] = of[8] + al(nv);                              // convmask
        of[10] = of[9] + al(sizeof(RobustStat));
        unsigned char* rb;
        TRY(wsT(c, S_ROBUST, of[10], &rb));
        pb.r.vmod = reinterpret_cast<float*>(rb + of[0]);
        pb.r.vloss = reinterpret_cast<float*>(rb + of[1]);
        pb.r.vinit = reinterpret_cast<float*>(rb + of[2]);
        pb.r.ring = reinterpret_cast<float*>(rb + of[3]);
        pb.r.imp_a = reinterpret_cast<float*>(rb + of[4]);
        pb.r.imp_b = reinterpret_cast<float*>(rb + of[5]);
        pb.r.flagcnt = reinterpret_cast<int*>(rb + of[6]);
        pb.r.mainmask = rb + of[7];
        pb.r.convmask = rb + of[8];
        pb.r.stat = reinterpret_cast<RobustStat*>(rb + of[9]);
    }
    if (!J.stats) {
        // plain_zgrad only touches zprev when statistics are requested
        J.a.zprev = nullptr;
    }
    out.tr.assign(J.nvol, Tracker());
    out.final_epoch.assign(J.nvol, N);
    J.hist.assign((size_t)J.nvol * (N + 1) * kHistW, 0.0);
    int n_main = 0;
    CK(cudaEventRecord(c->ev[2], c->stream));
    for (int i = 0; i < J.nvol; ++i) {
        View V;
        TRY(make_view(J, i, J.a, &V));
        AdamParams& a = V.a;
        const size_t off = J.hv[i].off;
        PlainBufs b = pb;
        b.theta += off; b.dth += off; b.signal += off; b.dsig += off; b.res += off;
        b.gth += off; b.gz += off;
        int rhead = 0;  // oldest row of the robust loss history
        if (robust) {
            b.r.vmod += off; b.r.vloss += off; b.r.vinit += off; b.r.ring += off; b.r.imp_a += off;
            b.r.imp_b += off; b.r.flagcnt += off; b.r.mainmask += off; b.r.convmask += off;
            CK(launch_robust_reset(a, b, J.B, V.nblocks, c->stream));
        }
        Tracker& t = out.tr[i];
        float* zmin = J.zr + off;
        float* resm = out.resm ? out.resm + off : nullptr;
        size_t base = (size_t)i * (N + 1) * kHistW;
        int last = 0;
        for (int e = (N == 0 ? 0 : 1); e <= N; ++e) {
            last = e;
            CK(cudaMemsetAsync(pb.acc, 0, sizeof(double) * 8, c->stream));
            CK(launch_plain_unscale(a, b, J.B, V.nblocks, c->stream));
            CK(launch_plain_forward(a, J.id, b, J.B, V.nblocks, c->stream));
            CK(launch_plain_loss(a, o->loss, b, J.B, V.nblocks, c->stream));
            CK(launch_plain_adjoint(a, J.id, b, J.B, V.nblocks, c->stream));
            if (J.tv) CK(launch_plain_tv(a, b, J.grid[0], J.B, V.nblocks, c->stream));
            if (J.prior) CK(launch_plain_prior(a, b, J.B, V.nblocks, c->stream));
            CK(launch_plain_zgrad(a, b, J.stats, J.B, V.nblocks, c->stream));
            n_main += J.tv ? 7 : (J.prior ? 6 : 5);
            if (robust && e >= 1) {
                // perVoxelLossInit is the starting point's evaluation, equal to epoch 1's
                if (e == 1) CK(launch_robust_seed(a, b, RW, J.B, V.nblocks, c->stream));
                if (e % o->weight_update_interval == 0) {
                    const int slot = rhead;
                    rhead = (rhead + 1) % RW;
                    CK(launch_robust_check(a, b, slot, rhead, ro, J.hv[i].nvox, J.B, V.nblocks, c->stream));
                }
                if (e % o->convergence_window == 0) CK(launch_robust_window(a, b, J.B, V.nblocks, c->stream));
                CK(launch_robust_conv(a, b, J.B, V.nblocks, c->stream));
            }
            double acc[8];
            CK(cudaMemcpyAsync(acc, pb.acc, sizeof(acc), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            double* h = J.hist.data() + base + (size_t)e * kHistW;
            h[0] = acc[0]; h[1] = acc[1]; h[2] = acc[2]; h[3] = acc[3]; h[4] = acc[4];
            bool snap = false;
            if (e <= 1) {
                t.init(o, acc[0], acc[1]);
                for (int q = 0; q < kHistW; ++q) J.hist[base + q] = h[q];
                snap = true;  // parameters_minLoss = initial parameters (askadam.m:203-208)
            }
            if (e >= 1) {
                int before = t.minIter;
                if (robust) t.epoch(e, acc[0], acc[1], acc[2], acc[3], acc[4], acc[5] / acc[6], acc[7] != 0.0);
                else t.epoch(e, acc[0], acc[1], acc[2], acc[3], acc[4]);
                snap = snap || t.minIter != before;
            }
            if (snap) {
                for (int k = 0; k < J.np; ++k)
                    CK(cudaMemcpyAsync(zmin + (size_t)k * J.nvtot, a.z + (size_t)k * J.nvtot, sizeof(float) * J.hv[i].npad,
                                       cudaMemcpyDeviceToDevice, c->stream));
                if (resm)
                    for (int m = 0; m < J.nm; ++m)
                        CK(cudaMemcpyAsync(resm + (size_t)m * J.nvtot, b.res + (size_t)m * J.nvtot, sizeof(float) * J.hv[i].npad,
                                           cudaMemcpyDeviceToDevice, c->stream));
            }
            if (t.stopped) break;
            if (e >= 1 && e < N) {
                CK(launch_plain_update(a, b, e, J.B, V.nblocks, c->stream));
                ++n_main;
            }
            if (cancelled(c)) return fail(GX_ECANCELLED, "cancelled");
        }
        out.final_epoch[i] = last;
        CK(launch_finalize(a, a.z, out.thf + off, nullptr, nullptr, J.B, V.nblocks, c->stream));
        CK(launch_finalize(a, zmin, out.thm + off, nullptr, nullptr, J.B, V.nblocks, c->stream));
        if (out.resf)
            for (int m = 0; m < J.nm; ++m)
                CK(cudaMemcpyAsync(out.resf + off + (size_t)m * J.nvtot, b.res + (size_t)m * J.nvtot,
                                   sizeof(float) * J.hv[i].npad, cudaMemcpyDeviceToDevice, c->stream));
    }
    CK(cudaEventRecord(c->ev[3], c->stream));
    CK(cudaEventSynchronize(c->ev[3]));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
    c->timing.main_kernel_ms = ms;
    c->timing.main_launches = n_main;
    return GX_OK;
}

static gx_status adam_write_results(AdamJob& J, AdamOut& out, gx_askadam_result* results) {
    gx_context* c = J.c;
    const int N = J.o->iteration;
    float *rlf = nullptr, *rlm = nullptr;
    bool want_rlf = false, want_rlm = false;
    for (int i = 0; i < J.nvol; ++i) {
        want_rlf |= results[i].final_resloss != nullptr;
        want_rlm |= results[i].min_resloss != nullptr;
    }
    if (want_rlf && out.resf) {
        TRY(wsT(c, S_RLF, J.nvtot, &rlf));
        CK(launch_finalize(J.a, nullptr, nullptr, out.resf, rlf, J.B, J.nblocks, c->stream));
    }
    if (want_rlm && out.resm) {
        TRY(wsT(c, S_RLM, J.nvtot, &rlm));
        CK(launch_finalize(J.a, nullptr, nullptr, out.resm, rlm, J.B, J.nblocks, c->stream));
    }
    for (int i = 0; i < J.nvol; ++i) {
        gx_askadam_result& r = results[i];
        const DevVol& d = J.hv[i];
        int n = d.nvox;
        TRY(download_rows(c, r.final_theta, out.thf, J.nvtot, d.off, J.np, n, J.mem, &J.d2h));
        TRY(download_rows(c, r.min_theta, out.thm, J.nvtot, d.off, J.np, n, J.mem, &J.d2h));
        if (out.resf) TRY(download_rows(c, r.final_residual, out.resf, J.nvtot, d.off, J.nm, n, J.mem, &J.d2h));
        if (out.resm) TRY(download_rows(c, r.min_residual, out.resm, J.nvtot, d.off, J.nm, n, J.mem, &J.d2h));
        if (rlf) TRY(download_rows(c, r.final_resloss, rlf, J.nvtot, d.off, 1, n, J.mem, &J.d2h));
        if (rlm) TRY(download_rows(c, r.min_resloss, rlm, J.nvtot, d.off, 1, n, J.mem, &J.d2h));
        const Tracker& t = out.tr[i];
        int fe = out.final_epoch[i];
        size_t base = (size_t)i * (N + 1) * kHistW;
        const double* hf = J.hist.data() + base + (size_t)fe * kHistW;
        r.final_loss = hf[0] + hf[1];
        r.final_loss_fidelity = hf[0];
        r.final_loss_reg = hf[1];
        r.min_loss = t.minLoss;
        r.min_loss_fidelity = t.minFid;
        r.min_loss_reg = t.minReg;
        r.final_niteration = fe;
        r.min_niteration = t.minIter;
        r.stop_reason = t.reason;
        if (r.loss_history)
            for (int e = 0; e <= N; ++e) {
                const double* h = J.hist.data() + base + (size_t)e * kHistW;
                r.loss_history[e] = e <= fe ? h[0] + h[1] : NAN;
            }
    }
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < J.nvol; ++i)
        if (!std::isfinite(results[i].final_loss))
            return fail(GX_ENUMERIC, "volume %d: non-finite loss", i);
    return GX_OK;
}

extern "C" gx_status gx_askadam(gx_context* c, const gx_model* model, int32_t mem,
                                const gx_volume* vols, int32_t nvol, const gx_askadam_opts* opts,
                                gx_askadam_result* results) {
    if (!c) return fail(GX_EINVAL, "context is NULL");
    if (!results) return fail(GX_EINVAL, "results is NULL");
    if (mem != GX_MEM_HOST && mem != GX_MEM_DEVICE) return fail(GX_EINVAL, "mem must be GX_MEM_HOST or GX_MEM_DEVICE");
    CallScope scope(c);
    AdamJob J;
    J.c = c; J.model = model; J.o = opts; J.mem = mem; J.vols = vols; J.nvol = nvol;
    J.allow_tune = true;
    TRY(model_sizes(model, &J.np, &J.nm, &J.id));
    TRY(validate_adam(opts, J.np, vols, nvol, J.nm));
    for (int i = 0; i < nvol; ++i)
        if (!results[i].final_theta) return fail(GX_EINVAL, "volume %d: final_theta is NULL", i);
    J.want_min = true;
    J.want_res_f = J.want_res_m = false;
    for (int i = 0; i < nvol; ++i) {
        J.want_res_f |= results[i].final_residual || results[i].final_resloss;
        J.want_res_m |= results[i].min_residual || results[i].min_resloss;
    }
    PhaseTrace trace("gx_askadam", c->stream);
    J.trace = trace.on ? &trace : nullptr;
    CK(cudaEventRecord(c->ev[0], c->stream));
    TRY(adam_setup(J));
    AdamOut out;
    // robustConvergence couples every epoch to per-voxel losses and a
    // readback, as the reference's loop does: it runs on the op-by-op path
    if (opts->path == GX_PATH_PLAIN || opts->robust_convergence) TRY(adam_plain(J, out));
    else TRY(adam_fused(J, out));
    gx_status st = adam_write_results(J, out, results);
    trace.mark("write");
    CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaEventSynchronize(c->ev[1]));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->timing.total_ms = ms;
    c->timing.kernel_launches = g_kernel_launches - scope.launches0;
    c->timing.h2d_bytes = J.h2d;
    c->timing.d2h_bytes = J.d2h;
    return st;
}

// One evaluation of loss and d loss / d theta at physical parameters theta
// (askadam.model_gradient, utils/askadam.m:23-117).
extern "C" gx_status gx_model_gradient(gx_context* c, const gx_model* model, int32_t mem,
                                       const gx_volume* vol, const gx_askadam_opts* opts,
                                       const float* theta, float* gtheta, float* residual,
                                       double* loss, double* loss_fid, double* loss_reg) {
    if (!c || !theta) return fail(GX_EINVAL, "NULL argument");
    CallScope scope(c);
    AdamJob J;
    J.c = c; J.model = model; J.o = opts; J.mem = mem; J.vols = vol; J.nvol = 1;
    TRY(model_sizes(model, &J.np, &J.nm, &J.id));
    TRY(validate_adam(opts, J.np, vol, 1, J.nm));
    gx_askadam_opts o2 = *opts;
    o2.iteration = 0;
    J.o = &o2;
    TRY(adam_setup(J));
    size_t pn = (size_t)J.np * J.nvtot, mn = (size_t)J.nm * J.nvtot;
    PlainBufs b;
    TRY(wsT(c, S_P_TH, pn, &b.theta));
    TRY(wsT(c, S_P_DTH, pn, &b.dth));
    TRY(wsT(c, S_P_SIG, mn, &b.signal));
    TRY(wsT(c, S_P_DSIG, mn, &b.dsig));
    TRY(wsT(c, S_P_RES, mn, &b.res));
    TRY(wsT(c, S_P_GTH, pn, &b.gth));
    TRY(wsT(c, S_P_GZ, pn, &b.gz));
    TRY(wsT(c, S_P_ACC, 8, &b.acc));
    CK(cudaMemsetAsync(b.theta, 0, sizeof(float) * pn, c->stream));
    TRY(upload_rows(c, b.theta, J.nvtot, 0, theta, J.np, vol->nvox, mem, &J.h2d));
    CK(cudaMemsetAsync(b.acc, 0, sizeof(double) * 8, c->stream));
    AdamParams a = J.a;
    a.zprev = nullptr;
    CK(launch_plain_forward(a, J.id, b, J.B, J.nblocks, c->stream));
    CK(launch_plain_loss(a, opts->loss, b, J.B, J.nblocks, c->stream));
    CK(launch_plain_adjoint(a, J.id, b, J.B, J.nblocks, c->stream));
    if (J.tv) CK(launch_plain_tv(a, b, J.grid[0], J.B, J.nblocks, c->stream));
    if (J.prior) CK(launch_plain_prior(a, b, J.B, J.nblocks, c->stream));
    double acc[8];
    CK(cudaMemcpyAsync(acc, b.acc, sizeof(acc), cudaMemcpyDeviceToHost, c->stream));
    TRY(download_rows(c, gtheta, b.gth, J.nvtot, 0, J.np, vol->nvox, mem, &J.d2h));
    if (residual) TRY(download_rows(c, residual, b.res, J.nvtot, 0, J.nm, vol->nvox, mem, &J.d2h));
    CK(cudaStreamSynchronize(c->stream));
    if (loss) *loss = acc[0] + acc[1];
    if (loss_fid) *loss_fid = acc[0];
    if (loss_reg) *loss_reg = acc[1];
    c->timing.kernel_launches = g_kernel_launches - scope.launches0;
    return GX_OK;
}

extern "C" gx_status gx_forward(gx_context* c, const gx_model* model, int32_t mem, const float* theta,
                                const float* b1, int32_t nvox, float* signal) {
    if (!c || !theta || !signal) return fail(GX_EINVAL, "NULL argument");
    if (nvox < 1) return fail(GX_EINVAL, "nvox must be >= 1");
    CallScope scope(c);
    int np, nm, id;
    TRY(model_sizes(model, &np, &nm, &id));
    if (model->kind == GX_MODEL_NEXI_RICE && !b1)
        return fail(GX_EINVAL, "NEXI Rice: the per-voxel noise sigma (aux) is required");
    DevProtocol P = make_protocol(model, id, np, nm, nullptr, nullptr, 0);
    const float *dth = theta, *db1 = b1;
    float* dsig = signal;
    long long h2d = 0, d2h = 0;
    if (mem == GX_MEM_HOST) {
        float *t, *s, *bb = nullptr;
        TRY(wsT(c, S_FWD_TH, (size_t)np * nvox, &t));
        TRY(wsT(c, S_FWD_SIG, (size_t)nm * nvox, &s));
        CK(cudaMemcpyAsync(t, theta, sizeof(float) * np * nvox, cudaMemcpyHostToDevice, c->stream));
        h2d += sizeof(float) * np * nvox;
        if (b1) {
            TRY(wsT(c, S_FWD_B1, (size_t)nvox, &bb));
            CK(cudaMemcpyAsync(bb, b1, sizeof(float) * nvox, cudaMemcpyHostToDevice, c->stream));
            h2d += sizeof(float) * nvox;
        }
        dth = t; db1 = bb; dsig = s;
    }
    CK(cudaEventRecord(c->ev[2], c->stream));
    CK(launch_forward_only(P, id, dth, db1, nvox, dsig, c->stream));
    CK(cudaEventRecord(c->ev[3], c->stream));
    if (mem == GX_MEM_HOST) {
        CK(cudaMemcpyAsync(signal, dsig, sizeof(float) * nm * nvox, cudaMemcpyDeviceToHost, c->stream));
        d2h += sizeof(float) * nm * nvox;
    }
    CK(cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
    c->timing.main_kernel_ms = ms;
    c->timing.main_launches = 1;
    c->timing.kernel_launches = g_kernel_launches - scope.launches0;
    c->timing.h2d_bytes = h2d;
    c->timing.d2h_bytes = d2h;
    return GX_OK;
}

// ---------------------------------------------------------------------------
// MCMC
// ---------------------------------------------------------------------------
static int mcmc_nsamples(int iteration, int nb, int thinning) {
    if (nb + 1 > iteration) return 0;
    return (iteration - nb - 1) / thinning + 1;  // numel(Nburnin+1:thinning:iteration)
}

// Autotuner of the MCMC kernels' block shape (Goodman-Weare: voxels per CTA;
// MH: threads per CTA).  Key: device, model, algorithm, walkers, update
// scheme, variables, measurements, weights / b1 variants and the voxel-count
// class.  On a miss each candidate runs a few steps from the start on the
// first voxels of this job (scratch walker state and sums; the job's buffers
// untouched) and the fastest is cached for the process.
static gx_status tune_mcmc(gx_context* c, const McmcParams& p, int model, int* block, bool* tuned) {
    int cls = 0;
    while ((1LL << (cls + 1)) <= (long long)p.nvox) ++cls;
    const int W = p.algorithm == 1 ? p.nwalker : 1;
    const TuneKey key{{2, c->device, model, p.algorithm, W, p.update, p.nvar, p.nm, p.weights ? 1 : 0,
                       p.b1 ? 1 : 0, cls, 0, 0}};
    int b = tune_lookup(key);
    if (b <= 0) {
        McmcParams t = p;
        t.nvox = std::min(p.nvox, std::max(256, (1 << 19) / W));
        t.posterior = nullptr;
        const int k1 = std::min(p.iteration, 8);
        const size_t nx = (size_t)t.nvar * t.nvox * W, nl = (size_t)t.nvox * W, ns = (size_t)t.nvar * t.nvox;
        const size_t o_lp = (sizeof(float) * nx + 255) / 256 * 256;
        const size_t o_s1 = o_lp + (sizeof(double) * nl + 255) / 256 * 256;
        const size_t o_s2 = o_s1 + sizeof(double) * ns;
        const size_t o_acc = o_s2 + sizeof(double) * ns;
        unsigned char* sc;
        TRY(wsT(c, S_TUNE, o_acc + sizeof(unsigned long long), &sc));
        float* xs = reinterpret_cast<float*>(sc);
        double* lps = reinterpret_cast<double*>(sc + o_lp);
        double* s1 = reinterpret_cast<double*>(sc + o_s1);
        double* s2 = reinterpret_cast<double*>(sc + o_s2);
        t.n_acc = reinterpret_cast<unsigned long long*>(sc + o_acc);
        int cand[8];
        const int nc = mcmc_block_candidates(t, cand, 8);
        float best = 0.f;
        for (int j = 0; j < nc; ++j) {
            float ms = 0.f;
            bool ok = true;
            for (int rep = 0; rep < 3 && ok; ++rep) {  // the first run warms the code and caches
                CK(cudaEventRecord(c->ev[2], c->stream));
                cudaError_t e = launch_mcmc_trial(t, model, cand[j], k1, xs, lps, s1, s2, c->stream);
                if (e == cudaErrorInvalidConfiguration || e == cudaErrorLaunchOutOfResources) {
                    cudaGetLastError();  // a shape this kernel cannot take: skipped
                    ok = false;
                    break;
                }
                CK(e);
                CK(cudaEventRecord(c->ev[3], c->stream));
                CK(cudaEventSynchronize(c->ev[3]));
                float m = 0.f;
                cudaEventElapsedTime(&m, c->ev[2], c->ev[3]);
                if (rep == 1 || (rep > 1 && m < ms)) ms = m;
            }
            if (ok && (b <= 0 || ms < best)) { best = ms; b = cand[j]; }
        }
        if (b <= 0) return fail(GX_ECUDA, "autotuner: no block shape fits the MCMC kernel");
        tune_store(key, b);
        *tuned = true;
    }
    *block = b;
    return GX_OK;
}

extern "C" gx_status gx_mcmc(gx_context* c, const gx_model* model, int32_t mem, const gx_volume* vols,
                             int32_t nvol, const gx_mcmc_opts* o, gx_mcmc_result* results) {
    if (!c || !o || !vols || !results || nvol < 1) return fail(GX_EINVAL, "NULL argument");
    if (mem != GX_MEM_HOST && mem != GX_MEM_DEVICE) return fail(GX_EINVAL, "bad mem");
    CallScope scope(c);
    int np, nm, id;
    TRY(model_sizes(model, &np, &nm, &id));
    if (model->kind == GX_MODEL_NEXI_RICE)
        return fail(GX_EUNSUPPORTED, "NEXI Rice: the reference samples gpuNEXIrice with askAdam only");
    int nvar = np + 1;
    if (o->algorithm != GX_MCMC_MH && o->algorithm != GX_MCMC_ENSEMBLE) return fail(GX_EINVAL, "unknown algorithm");
    if (o->iteration < 1 || o->thinning < 1 || o->repetition < 1) return fail(GX_EINVAL, "iteration, thinning and repetition must be >= 1");
    if (!o->lb || !o->ub) return fail(GX_EINVAL, "lb/ub required");
    for (int q = 0; q < nvar; ++q)
        if (!(o->ub[q] >= o->lb[q])) return fail(GX_EINVAL, "ub[%d] < lb[%d]", q, q);
    if (o->lb[nvar - 1] <= 0) return fail(GX_EINVAL, "noise lower bound must be positive");
    if (o->algorithm == GX_MCMC_ENSEMBLE) {
        if (o->nwalker < 2 || o->nwalker > 256) return fail(GX_EINVAL, "nwalker must be in [2, 256]");
        if (!(o->step_size > 1.0)) return fail(GX_EINVAL, "StepSize must exceed 1");
        if (o->ensemble_update != GX_GW_SIMULTANEOUS && o->ensemble_update != GX_GW_REDBLACK)
            return fail(GX_EINVAL, "unknown Ensembleupdate");
    } else if (!o->x_step) {
        return fail(GX_EINVAL, "MH needs x_step (xStepSize)");
    }
    if (o->nbin < 0 || o->nbin == 1 || o->nbin > (1 << 15)) return fail(GX_EINVAL, "Nbin must be in [2, 32768] (0 = 1001)");
    int ng = 0;
    if (o->is_global)
        for (int q = 0; q < nvar; ++q) ng += o->is_global[q] != 0;
    if (ng > 0) {
        // goodman_weare_wglobal_constant's partition check (utils/mcmc.m:462-466)
        if (o->algorithm != GX_MCMC_ENSEMBLE)
            return fail(GX_EINVAL, "global parameters need the ensemble (Goodman-Weare) algorithm");
        if (ng == nvar)
            return fail(GX_EINVAL, "need at least one local and one global parameter (NND=0, NGlobal=%d)", ng);
        if (o->global_warmup < 0) return fail(GX_EINVAL, "globalWarmup must be >= 0");
    }
    int nb = o->burnin < 1 ? (int)std::floor(o->iteration * o->burnin) : (int)o->burnin;
    int ns = mcmc_nsamples(o->iteration, nb, o->thinning);
    int W = o->algorithm == GX_MCMC_ENSEMBLE ? o->nwalker : 1;
    long long h2d = 0, d2h = 0;
    double kernel_ms = 0.0;
    int launches = 0;
    bool tuned_now = false;
    int block_used = 0;
    bool aux_pending = false;
    double aux_ms = 0.0;
    CK(cudaEventRecord(c->ev[0], c->stream));
    for (int i = 0; i < nvol; ++i) {
        const gx_volume& v = vols[i];
        gx_mcmc_result& r = results[i];
        if (v.nvox < 1 || !v.data || !v.theta0) return fail(GX_EINVAL, "volume %d: need nvox, data and theta0 (pars0)", i);
        int nv = v.nvox;
        McmcParams p;
        memset(&p, 0, sizeof(p));
        p.P = make_protocol(model, id, np, nm, nullptr, nullptr, 0);
        p.nm = nm; p.nvar = nvar; p.nvox = nv;
        for (int q = 0; q < nvar; ++q) {
            p.lb[q] = (float)o->lb[q];
            p.ub[q] = (float)o->ub[q];
            p.xstep[q] = o->x_step ? (float)o->x_step[q] : 0.0f;
        }
        p.algorithm = o->algorithm; p.nwalker = W; p.iteration = o->iteration; p.thinning = o->thinning;
        p.nburnin = nb; p.ns = ns; p.repetition = o->repetition; p.update = o->ensemble_update;
        p.a = (float)o->step_size; p.start_range = (float)o->start_range; p.seed = o->seed;
        float *data, *w = nullptr, *b1 = nullptr, *x0, *shift, *post = nullptr;
        double *sum, *sumsq;
        unsigned long long* nacc;
        int* partner = nullptr;
        TRY(wsT(c, S_DATA, (size_t)nm * nv, &data));
        TRY(upload_rows(c, data, nv, 0, v.data, nm, nv, mem, &h2d));
        if (v.weights) { TRY(wsT(c, S_W, (size_t)nm * nv, &w)); TRY(upload_rows(c, w, nv, 0, v.weights, nm, nv, mem, &h2d)); }
        if (v.b1) { TRY(wsT(c, S_B1, (size_t)nv, &b1)); TRY(upload_rows(c, b1, nv, 0, v.b1, 1, nv, mem, &h2d)); }
        TRY(wsT(c, S_MC_X0, (size_t)nvar * nv, &x0));
        TRY(upload_rows(c, x0, nv, 0, v.theta0, nvar, nv, mem, &h2d));
        TRY(wsT(c, S_MC_SHIFT, (size_t)nvar * nv, &shift));
        TRY(wsT(c, S_MC_SUM, (size_t)nvar * nv, &sum));
        TRY(wsT(c, S_MC_SUMSQ, (size_t)nvar * nv, &sumsq));
        TRY(wsT(c, S_MC_ACC, 1, &nacc));
        CK(cudaMemsetAsync(sum, 0, sizeof(double) * nvar * nv, c->stream));
        CK(cudaMemsetAsync(sumsq, 0, sizeof(double) * nvar * nv, c->stream));
        CK(cudaMemsetAsync(nacc, 0, sizeof(unsigned long long), c->stream));
        // the kept samples stay on the device when the posterior is returned or
        // summarised there (median / iqr / mode)
        const bool want_stats = r.median || r.iqr || r.mode;
        const size_t npost = (size_t)nvar * o->repetition * ns * W * nv;
        if (r.posterior || want_stats) {
            if (mem == GX_MEM_DEVICE && r.posterior) post = r.posterior;
            else TRY(wsT(c, S_MC_POST, npost, &post));
        }
        if (o->algorithm == GX_MCMC_ENSEMBLE) TRY(wsT(c, S_MC_PART, (size_t)o->repetition * o->iteration * W, &partner));
        p.data = data; p.weights = w; p.b1 = b1; p.x0 = x0; p.shift = shift; p.sum = sum; p.sumsq = sumsq;
        p.posterior = post; p.n_acc = nacc; p.partner = partner;
        if (ng > 0) {
            p.ng = ng;
            p.nnd = nvar - ng;
            p.global_warmup = o->global_warmup;
            p.nsteps_g = o->iteration + o->global_warmup;
            for (int q = 0; q < nvar; ++q) p.is_global[q] = o->is_global[q] != 0;
            int vpb, block, nbk;
            size_t smem;
            gwg_launch_shape(p, o->block_size, &vpb, &block, &nbk, &smem);
            // one allocation, carved at 256-byte boundaries
            auto al = [](size_t b) { return (b + 255) / 256 * 256; };
            size_t o_gs = 0;
            size_t o_ga = o_gs + al(sizeof(float) * nvar * W);
            size_t o_sum = o_ga + al(sizeof(int) * W);
            size_t o_sq = o_sum + al(sizeof(double) * nvar * W);
            size_t o_na = o_sq + al(sizeof(double) * nvar * W);
            size_t o_pr = o_na + al(sizeof(unsigned long long));
            size_t o_zz = o_pr + al(sizeof(float) * nvar * W);
            size_t o_lu = o_zz + al(sizeof(float) * W);
            size_t o_ob = o_lu + al(sizeof(float) * W);
            size_t o_gp = o_ob + al(sizeof(int) * W);
            size_t o_lpg = o_gp + al(sizeof(int) * (size_t)o->repetition * p.nsteps_g * W);
            size_t o_part = o_lpg + al(sizeof(double) * (size_t)nv * W);
            size_t total = o_part + al(sizeof(double) * (size_t)W * nbk);
            unsigned char* gb;
            TRY(wsT(c, S_MC_GLOB, total, &gb));
            p.gstate = reinterpret_cast<float*>(gb + o_gs);
            p.gacc = reinterpret_cast<int*>(gb + o_ga);
            p.gsum = reinterpret_cast<double*>(gb + o_sum);
            p.gsumsq = reinterpret_cast<double*>(gb + o_sq);
            p.n_gacc = reinterpret_cast<unsigned long long*>(gb + o_na);
            p.gprop = reinterpret_cast<float*>(gb + o_pr);
            p.gzz = reinterpret_cast<float*>(gb + o_zz);
            p.glu = reinterpret_cast<float*>(gb + o_lu);
            p.goob = reinterpret_cast<int*>(gb + o_ob);
            p.gpartner = reinterpret_cast<int*>(gb + o_gp);
            p.lpg = reinterpret_cast<double*>(gb + o_lpg);
            p.partial = reinterpret_cast<double*>(gb + o_part);
            CK(cudaMemsetAsync(gb, 0, o_gp, c->stream));  // state, decisions, sums, counter
        }
        // slots that no step fills stay zero (res2out counts them)
        if (post && mcmc_missing_slots(p) > 0) CK(cudaMemsetAsync(post, 0, sizeof(float) * npost, c->stream));
        if (partner) CK(launch_mcmc_partners(p, partner, c->stream));
        int block = o->block_size;
        if (block == 0 && ng == 0 && autotune_enabled()) TRY(tune_mcmc(c, p, id, &block, &tuned_now));
        block_used = block > 0 ? block : 128;
        CK(cudaEventRecord(c->ev[2], c->stream));
        CK(launch_mcmc(p, id, block, c->stream));
        CK(cudaEventRecord(c->ev[3], c->stream));
        launches += ng > 0 ? (o->ensemble_update == GX_GW_REDBLACK ? 4 : 2) * (o->iteration + o->global_warmup) *
                                 o->repetition
                           : (o->iteration + 249) / 250 * o->repetition;
        float *mean = nullptr, *stdv = nullptr;
        if (mem == GX_MEM_DEVICE) { mean = r.mean; stdv = r.std; }
        else {
            TRY(wsT(c, S_MC_MEAN, (size_t)nvar * nv, &mean));
            TRY(wsT(c, S_MC_STD, (size_t)nvar * nv, &stdv));
        }
        CK(launch_mcmc_finalize(p, mean, stdv, c->stream));
        float *dmed = nullptr, *diqr = nullptr, *dmode = nullptr;
        if (want_stats) {
            const int nbin = o->nbin > 0 ? o->nbin : 1001;
            // [3][nvar][nv] outputs (host calls) and the bounds [nvar][2] in one buffer
            const size_t nst = (size_t)nvar * nv;
            const size_t o_lb = (sizeof(float) * 3 * nst + 15) / 16 * 16;
            unsigned char* sb;
            TRY(wsT(c, S_MC_STATS, o_lb + sizeof(double) * 2 * nvar, &sb));
            float* st = reinterpret_cast<float*>(sb);
            double* lbub = reinterpret_cast<double*>(sb + o_lb);
            double hb[2 * kMaxParam];
            for (int q = 0; q < nvar; ++q) { hb[2 * q] = o->lb[q]; hb[2 * q + 1] = o->ub[q]; }
            CK(cudaMemcpyAsync(lbub, hb, sizeof(double) * 2 * nvar, cudaMemcpyHostToDevice, c->stream));
            if (mem == GX_MEM_DEVICE) { dmed = r.median; diqr = r.iqr; dmode = r.mode; }
            else {
                dmed = r.median ? st : nullptr;
                diqr = r.iqr ? st + nst : nullptr;
                dmode = r.mode ? st + 2 * nst : nullptr;
            }
            CK(cudaEventRecord(c->ev[4], c->stream));
            CK(launch_posterior_stats(post, nvar, nv, o->repetition * ns * W, nbin, lbub, dmed, diqr, dmode,
                                      c->stream));
            CK(cudaEventRecord(c->ev[5], c->stream));
            aux_pending = true;
        }
        if (mem == GX_MEM_HOST) {
            const size_t nst = (size_t)nvar * nv;
            float* hs[3] = {r.median, r.iqr, r.mode};
            float* ds[3] = {dmed, diqr, dmode};
            for (int j = 0; j < 3; ++j)
                if (hs[j]) {
                    CK(cudaMemcpyAsync(hs[j], ds[j], sizeof(float) * nst, cudaMemcpyDeviceToHost, c->stream));
                    d2h += sizeof(float) * nst;
                }
            if (r.mean) { CK(cudaMemcpyAsync(r.mean, mean, sizeof(float) * nvar * nv, cudaMemcpyDeviceToHost, c->stream)); d2h += sizeof(float) * nvar * nv; }
            if (r.std) { CK(cudaMemcpyAsync(r.std, stdv, sizeof(float) * nvar * nv, cudaMemcpyDeviceToHost, c->stream)); d2h += sizeof(float) * nvar * nv; }
            if (r.posterior) {
                CK(cudaMemcpyAsync(r.posterior, post, sizeof(float) * npost, cudaMemcpyDeviceToHost, c->stream));
                d2h += sizeof(float) * npost;
            }
        }
        unsigned long long acc = 0, gacc = 0;
        CK(cudaMemcpyAsync(&acc, nacc, sizeof(acc), cudaMemcpyDeviceToHost, c->stream));
        if (ng > 0) CK(cudaMemcpyAsync(&gacc, p.n_gacc, sizeof(gacc), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        r.n_global_accepted = (int64_t)gacc;
        r.n_global_proposals = ng > 0 ? (int64_t)W * (o->iteration + o->global_warmup) * o->repetition : 0;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
        kernel_ms += ms;
        if (aux_pending) {
            cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]);
            aux_ms += ms;
            aux_pending = false;
        }
        r.n_accepted = (int64_t)acc;
        r.n_proposals = (int64_t)nv * W * o->iteration * o->repetition;
        r.ns = ns;
    }
    CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaEventSynchronize(c->ev[1]));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->timing.total_ms = ms;
    c->timing.main_kernel_ms = kernel_ms;
    c->timing.main_launches = launches;
    c->timing.block_size = block_used;
    c->timing.autotuned = tuned_now ? 1 : 0;
    c->timing.aux_kernel_ms = aux_ms;
    c->timing.kernel_launches = g_kernel_launches - scope.launches0;
    c->timing.h2d_bytes = h2d;
    c->timing.d2h_bytes = d2h;
    return GX_OK;
}

extern "C" gx_status gx_dictionary_match(gx_context* c, int32_t mem, const float* signals, int32_t nvox,
                                         const float* dict, int32_t ndict, int32_t nm, const float* wt,
                                         int32_t* best, float* best_sse) {
    if (!c || !signals || !dict || !best) return fail(GX_EINVAL, "NULL argument");
    if (mem != GX_MEM_HOST && mem != GX_MEM_DEVICE) return fail(GX_EINVAL, "bad mem");
    if (nvox < 1 || ndict < 1) return fail(GX_EINVAL, "nvox and ndict must be >= 1");
    if (nm < 1 || nm > kMaxMeas) return fail(GX_EINVAL, "nm must be in [1, %d]", kMaxMeas);
    CallScope scope(c);
    const float *ds = signals, *dd = dict, *dw = wt;
    int* db = best;
    float* dsse = best_sse;
    long long h2d = 0, d2h = 0;
    if (mem == GX_MEM_HOST) {
        float *s1, *s2, *s3 = nullptr, *s5 = nullptr;
        int* s4;
        TRY(wsT(c, S_DICT_SIG, (size_t)nm * nvox, &s1));
        TRY(wsT(c, S_DICT_D, (size_t)nm * ndict, &s2));
        CK(cudaMemcpyAsync(s1, signals, sizeof(float) * nm * nvox, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(s2, dict, sizeof(float) * nm * ndict, cudaMemcpyHostToDevice, c->stream));
        h2d += sizeof(float) * ((long long)nm * nvox + (long long)nm * ndict);
        if (wt) {
            TRY(wsT(c, S_DICT_W, (size_t)nm, &s3));
            CK(cudaMemcpyAsync(s3, wt, sizeof(float) * nm, cudaMemcpyHostToDevice, c->stream));
            h2d += sizeof(float) * nm;
        }
        TRY(wsT(c, S_DICT_B, (size_t)nvox, &s4));
        if (best_sse) TRY(wsT(c, S_DICT_S, (size_t)nvox, &s5));
        ds = s1; dd = s2; dw = s3; db = s4; dsse = s5;
    }
    double *ie, *cj;
    TRY(wsT(c, S_DICT_E, (size_t)ndict, &ie));
    TRY(wsT(c, S_DICT_C, (size_t)ndict, &cj));
    CK(cudaEventRecord(c->ev[2], c->stream));
    CK(launch_dictionary_match(ds, nvox, dd, ndict, nm, dw, ie, cj, db, dsse, c->stream));
    CK(cudaEventRecord(c->ev[3], c->stream));
    if (mem == GX_MEM_HOST) {
        CK(cudaMemcpyAsync(best, db, sizeof(int32_t) * nvox, cudaMemcpyDeviceToHost, c->stream));
        d2h += sizeof(int32_t) * nvox;
        if (best_sse) {
            CK(cudaMemcpyAsync(best_sse, dsse, sizeof(float) * nvox, cudaMemcpyDeviceToHost, c->stream));
            d2h += sizeof(float) * nvox;
        }
    }
    CK(cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
    c->timing.total_ms = ms;
    c->timing.main_kernel_ms = ms;
    c->timing.main_launches = 1;
    c->timing.kernel_launches = g_kernel_launches - scope.launches0;
    c->timing.h2d_bytes = h2d;
    c->timing.d2h_bytes = d2h;
    return GX_OK;
}

// ---------------------------------------------------------------------------
// Helpers for other translation units of the library (no new behaviour).
// ---------------------------------------------------------------------------
namespace gx {
gx_status internal_fail(gx_status s, const char* msg) { return fail(s, "%s", msg); }

gx_status internal_model(const gx_model* m, const double* lb, const double* ub, DevProtocol* P,
                         int* np, int* nm, int* id) {
    gx_status st = model_sizes(m, np, nm, id);
    if (st != GX_OK) return st;
    *P = make_protocol(m, *id, *np, *nm, lb, ub, *np);
    return GX_OK;
}

bool internal_can_stop(const gx_askadam_opts* o) { return can_stop(o); }

gx_status internal_validate_opts(const gx_askadam_opts* o, int np) { return validate_adam_common(o, np); }
}  // namespace gx
