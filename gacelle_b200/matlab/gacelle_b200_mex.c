/*
 * gacelle_b200_mex.c -- MATLAB MEX gateway to libgacelle_b200.so.
 *
 * The reference's built-in model classes call askadam().optimisation(...) and
 * mcmc().optimisation(...) with @this.FWD (R2star/gpuR2starMapping.m:237,243,
 * R1R2s/gpuJointR1R2starMapping.m:272,279, NEXI/gpuNEXI.m:435,440).  This
 * gateway lets those classes call the engine instead: it marshals mxArrays
 * into the structs of include/gacelle_b200.h and maps a non-zero gx_status to
 * the error identifier GACELLE:b200:<status>, as the reference raises
 * GACELLE:... identifiers (e.g. NEXI/gpuNEXI.m:565).
 *
 * Build (MATLAB, with the library next to this file):
 *   mex -I../../include gacelle_b200_mex.c -L.. -lgacelle_b200
 *
 * Calls (masked data in G-D form, voxel fastest: y is [Nvox, Nmeas] single,
 * which in memory is the engine's [Nmeas][Nvox]; parameters likewise
 * [Nvox, Nparam] single):
 *   ctx = gacelle_b200_mex('context', device)            % uint64 handle
 *   gacelle_b200_mex('destroy', ctx)
 *   S   = gacelle_b200_mex('forward', ctx, model, theta [, aux])
 *   out = gacelle_b200_mex('askadam', ctx, model, y, theta0, gidx, dims, fitting, lb, ub [, weights])
 *   out = gacelle_b200_mex('mcmc', ctx, model, y, x0, fitting, lb, ub [, xstep])
 * model:   struct with kind (1 R2*, 2 joint R1-R2*, 3 NEXI, 4 NEXI Rician
 *          mean), te [s], fa [deg], tr [s], b, Delta, lmax, Nx;
 * gidx:    int32 [Nvox] 0-based column-major grid index (TV), dims int32 [3];
 * fitting: the struct after askadam.check_set_default_basic /
 *          mcmc.check_set_default_basic (utils/askadam.m:735-878,
 *          utils/mcmc.m:633-679); regmap entries are 1-based parameter
 *          indices in fitting.regmapIndex.
 * Outputs: askadam -> struct final_theta, min_theta ([Nvox, Nparam] single),
 * final_loss, min_loss, final_Niteration, min_Niteration, lossHistory; mcmc ->
 * struct mean, std (and median, iqr, mode when fitting.metric asks for them).
 */
#include <stdint.h>
#include <string.h>

#include "mex.h"
#include "gacelle_b200.h"

static const char* status_id(gx_status s) {
    switch (s) {
    case GX_EINVAL: return "GACELLE:b200:invalidArgument";
    case GX_ENOMEM: return "GACELLE:b200:outOfMemory";
    case GX_ECUDA: return "GACELLE:b200:cuda";
    case GX_EUNSUPPORTED: return "GACELLE:b200:unsupported";
    case GX_ETIMEOUT: return "GACELLE:b200:timeout";
    case GX_ENUMERIC: return "GACELLE:b200:numeric";
    case GX_ECANCELLED: return "GACELLE:b200:cancelled";
    default: return "GACELLE:b200:error";
    }
}

static void check(gx_status s) {
    if (s != GX_OK) mexErrMsgIdAndTxt(status_id(s), "%s", gx_last_error());
}

static void need(int ok, const char* what) {
    if (!ok) mexErrMsgIdAndTxt("GACELLE:b200:invalidArgument", "%s", what);
}

/* ---- field readers (missing or empty fields give the default) ---------- */
static const mxArray* field(const mxArray* s, const char* name) {
    if (!s || !mxIsStruct(s)) return NULL;
    const mxArray* f = mxGetField(s, 0, name);
    return (f && !mxIsEmpty(f)) ? f : NULL;
}

static double fdouble(const mxArray* s, const char* name, double dflt) {
    const mxArray* f = field(s, name);
    return f ? mxGetScalar(f) : dflt;
}

static int fint(const mxArray* s, const char* name, int dflt) { return (int)fdouble(s, name, (double)dflt); }

static int fstr_is(const mxArray* s, const char* name, const char* value, int dflt) {
    const mxArray* f = field(s, name);
    char buf[64];
    if (!f || !mxIsChar(f) || mxGetString(f, buf, sizeof(buf)) != 0) return dflt;
    for (char* c = buf; *c; ++c)
        if (*c >= 'A' && *c <= 'Z') *c = (char)(*c - 'A' + 'a');
    return strcmp(buf, value) == 0;
}

/* a double vector field copied into a caller buffer; returns its length */
static int fvec(const mxArray* s, const char* name, double* out, int maxn) {
    const mxArray* f = field(s, name);
    if (!f) return 0;
    need(mxIsDouble(f), "numeric model / fitting fields must be double");
    int n = (int)mxGetNumberOfElements(f);
    need(n <= maxn, "model / fitting vector field too long");
    memcpy(out, mxGetPr(f), sizeof(double) * (size_t)n);
    return n;
}

static const float* single_arg(const mxArray* a, size_t rows, size_t cols, const char* what) {
    need(mxIsSingle(a) && !mxIsComplex(a), what);
    need(mxGetM(a) == rows && mxGetN(a) == cols, what);
    return (const float*)mxGetData(a);
}

static gx_context* ctx_arg(const mxArray* a) {
    need(mxIsUint64(a) && mxGetNumberOfElements(a) == 1, "context handle must be the uint64 from 'context'");
    gx_context* c = (gx_context*)(uintptr_t)(*(const uint64_t*)mxGetData(a));
    need(c != NULL, "context handle is empty");
    return c;
}

/* ---- model --------------------------------------------------------------- */
typedef struct {
    gx_model m;
    double te[128], fa[16], b[256], delta[256];
} model_buf;

static void model_arg(const mxArray* s, model_buf* mb, int* np, int* nm) {
    need(mxIsStruct(s), "model must be a struct");
    memset(mb, 0, sizeof(*mb));
    mb->m.kind = fint(s, "kind", 0);
    mb->m.lmax = fint(s, "lmax", 0);
    mb->m.nx = fint(s, "Nx", 14);
    mb->m.n_te = fvec(s, "te", mb->te, 128);
    mb->m.te = mb->te;
    mb->m.n_fa = fvec(s, "fa", mb->fa, 16);
    mb->m.fa_deg = mb->fa;
    mb->m.tr = fdouble(s, "tr", 0.0);
    mb->m.n_shell = fvec(s, "b", mb->b, 256);
    need(fvec(s, "Delta", mb->delta, 256) == mb->m.n_shell, "model.b and model.Delta must have equal length");
    mb->m.bval = mb->b;
    mb->m.big_delta = mb->delta;
    int32_t p = 0, q = 0;
    check(gx_model_sizes(&mb->m, &p, &q));
    *np = p;
    *nm = q;
}

/* ---- askadam ------------------------------------------------------------- */
static void askadam_opts(const mxArray* f, const double* lb, const double* ub, gx_askadam_opts* o) {
    memset(o, 0, sizeof(*o));
    o->iteration = fint(f, "iteration", 10000);
    o->initial_learn_rate = fdouble(f, "initialLearnRate", 0.001);
    o->decay_rate = fdouble(f, "decayRate", 0.0);
    o->optimiser = fstr_is(f, "optimiser", "sgdm", 0) ? GX_OPT_SGDM
                   : fstr_is(f, "optimiser", "rmsprop", 0) ? GX_OPT_RMSPROP : GX_OPT_ADAM;
    o->beta1 = fdouble(f, "adamupdateGradDecay", 0.9);
    o->beta2 = fdouble(f, "adamupdateSqGradDecay", 0.999);
    o->epsilon = fdouble(f, "adamupdateEpsilon", 1e-8);
    o->momentum = fdouble(f, "sgdmupdateMomentum", 0.9);
    o->rms_decay = fdouble(f, "rmspropupdateSqGradDecay", 0.9);
    o->rms_epsilon = fdouble(f, "rmspropupdateEpsilon", 1e-8);
    o->loss = fstr_is(f, "lossFunction", "l2", 0) ? GX_LOSS_L2
              : fstr_is(f, "lossFunction", "huber", 0) ? GX_LOSS_HUBER
              : fstr_is(f, "lossFunction", "mse", 0) ? GX_LOSS_MSE
              : fstr_is(f, "lossFunction", "gauss", 0) ? GX_LOSS_GAUSS_LOGP
              : fstr_is(f, "lossFunction", "rician", 0) ? GX_LOSS_RICIAN_LOGP : GX_LOSS_L1;
    o->mse_scale = fdouble(f, "mseScale", 0.5);
    o->huber_delta = fdouble(f, "huberTransitionPoint", 1.0);
    o->sigma = fdouble(f, "noiseSigma", 0.0);
    o->transform = fstr_is(f, "parameterTransform", "linear", 0) ? GX_TRANSFORM_LINEAR : GX_TRANSFORM_SIGMOID;
    o->randomness = fdouble(f, "randomness", 0.0);
    o->seed = (uint64_t)fdouble(f, "seed", 0.0);
    o->lb = lb;
    o->ub = ub;
    o->tol = fdouble(f, "tol", 1e-3);
    o->convergence_value = fdouble(f, "convergenceValue", 1e-8);
    o->convergence_window = fint(f, "convergenceWindow", 20);
    o->patience_convergence = fdouble(f, "patienceConvergence", 5.0);
    o->convergence_model = fstr_is(f, "convergenceModel", "linear", 0) ? GX_CONV_LINEAR : GX_CONV_EMA;
    o->ema_decay = fdouble(f, "emaDecay", 0.95);
    o->step_tol = fdouble(f, "convergenceStepTol", 1e-6);
    o->grad_tol = fdouble(f, "convergenceGradTol", 1e-6);
    o->patience_step = fdouble(f, "patienceStep", 5.0);
    o->patience_grad = fdouble(f, "patienceGrad", 5.0);
    double lam[8] = {0}, idx[8] = {0};
    int nl = fvec(f, "lambda", lam, 8), ni = fvec(f, "regmapIndex", idx, 8);
    if (nl > 0 && lam[0] > 0) {
        need(ni >= nl, "fitting.regmapIndex needs one 1-based parameter index per lambda");
        o->n_reg = nl;
        for (int r = 0; r < nl; ++r) {
            o->lambda[r] = lam[r];
            o->reg_param[r] = (int32_t)idx[r] - 1;
        }
    }
    o->reg_type = fstr_is(f, "regularisationType", "prior", 0) ? GX_REG_PRIOR
                  : fstr_is(f, "dataType", "surface", 0) ? GX_REG_SURFACE_TV : GX_REG_TV;
    o->tv_3d = fstr_is(f, "TVmode", "3d", 0);
    double vs[3] = {2.0, 2.0, 2.0};
    fvec(f, "voxelSize", vs, 3);
    for (int d = 0; d < 3; ++d) o->voxel_size[d] = vs[d];
    o->path = fstr_is(f, "path", "plain", 0) ? GX_PATH_PLAIN : GX_PATH_FUSED;
    o->robust_convergence = fint(f, "robustConvergence", 0);
    o->outlier_weight = fdouble(f, "outlierWeight", 0.1);
    o->weight_update_interval = fint(f, "weightUpdateInterval", 5);
    o->outlier_check_window = fint(f, "outlierCheckWindow", 5);
    o->outlier_min_flag_duration = fint(f, "outlierMinFlagDuration", 5);
    o->outlier_voxel_thres = fdouble(f, "outlierVoxelThres", 0.01);
    o->outlier_pop_thres = fdouble(f, "outlierPopThres", 0.05);
    o->outlier_init_thres = fdouble(f, "outlierInitThres", 0.05);
    o->outlier_init_pop_thres = fdouble(f, "outlierInitPopThres", 0.20);
}

static mxArray* single_out(size_t rows, size_t cols, float** data) {
    mxArray* a = mxCreateNumericMatrix(rows, cols, mxSINGLE_CLASS, mxREAL);
    *data = (float*)mxGetData(a);
    return a;
}

static void do_askadam(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 10, "askadam: ctx, model, y, theta0, gidx, dims, fitting, lb, ub [, weights]");
    gx_context* c = ctx_arg(prhs[1]);
    model_buf mb;
    int np, nm;
    model_arg(prhs[2], &mb, &np, &nm);
    const size_t nv = mxGetM(prhs[3]);
    gx_volume v;
    memset(&v, 0, sizeof(v));
    v.nvox = (int32_t)nv;
    v.data = single_arg(prhs[3], nv, (size_t)nm, "y must be single [Nvox, Nmeas]");
    v.theta0 = single_arg(prhs[4], nv, (size_t)np, "theta0 must be single [Nvox, Nparam]");
    if (!mxIsEmpty(prhs[5])) {
        need(mxIsInt32(prhs[5]) && mxGetNumberOfElements(prhs[5]) == nv, "gidx must be int32 [Nvox] (0-based)");
        v.grid_index = (const int32_t*)mxGetData(prhs[5]);
    }
    v.dims[0] = (int32_t)nv;
    v.dims[1] = v.dims[2] = 1;
    if (!mxIsEmpty(prhs[6])) {
        need(mxIsInt32(prhs[6]) && mxGetNumberOfElements(prhs[6]) == 3, "dims must be int32 [3]");
        memcpy(v.dims, mxGetData(prhs[6]), sizeof(int32_t) * 3);
    }
    need(mxIsDouble(prhs[8]) && mxIsDouble(prhs[9]) && (int)mxGetNumberOfElements(prhs[8]) >= np &&
             (int)mxGetNumberOfElements(prhs[9]) >= np,
         "lb / ub must be double with one entry per parameter");
    if (nrhs > 10 && !mxIsEmpty(prhs[10])) v.weights = single_arg(prhs[10], nv, (size_t)nm, "weights: single [Nvox, Nmeas]");
    gx_askadam_opts o;
    askadam_opts(prhs[7], mxGetPr(prhs[8]), mxGetPr(prhs[9]), &o);
    gx_askadam_result r;
    memset(&r, 0, sizeof(r));
    const char* names[] = {"final_theta", "min_theta", "final_loss", "min_loss", "final_Niteration",
                           "min_Niteration", "lossHistory", "stopReason"};
    mxArray* out = mxCreateStructMatrix(1, 1, 8, names);
    mxArray* hist = mxCreateDoubleMatrix((size_t)o.iteration + 1, 1, mxREAL);
    mxSetField(out, 0, "final_theta", single_out(nv, (size_t)np, &r.final_theta));
    mxSetField(out, 0, "min_theta", single_out(nv, (size_t)np, &r.min_theta));
    r.loss_history = mxGetPr(hist);
    gx_status st = gx_askadam(c, &mb.m, GX_MEM_HOST, &v, 1, &o, &r);
    mxSetField(out, 0, "lossHistory", hist);
    mxSetField(out, 0, "final_loss", mxCreateDoubleScalar(r.final_loss));
    mxSetField(out, 0, "min_loss", mxCreateDoubleScalar(r.min_loss));
    mxSetField(out, 0, "final_Niteration", mxCreateDoubleScalar(r.final_niteration));
    mxSetField(out, 0, "min_Niteration", mxCreateDoubleScalar(r.min_niteration));
    mxSetField(out, 0, "stopReason", mxCreateDoubleScalar(r.stop_reason));
    if (st == GX_ENUMERIC && nlhs > 0) {  /* the partial result is returned with a warning */
        mexWarnMsgIdAndTxt(status_id(st), "%s", gx_last_error());
        plhs[0] = out;
        return;
    }
    if (st != GX_OK) mxDestroyArray(out);
    check(st);
    plhs[0] = out;
}

/* ---- mcmc ---------------------------------------------------------------- */
static void do_mcmc(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 8, "mcmc: ctx, model, y, x0, fitting, lb, ub [, xstep]");
    gx_context* c = ctx_arg(prhs[1]);
    model_buf mb;
    int np, nm;
    model_arg(prhs[2], &mb, &np, &nm);
    const int nvar = np + 1;
    const size_t nv = mxGetM(prhs[3]);
    gx_volume v;
    memset(&v, 0, sizeof(v));
    v.nvox = (int32_t)nv;
    v.dims[0] = (int32_t)nv;
    v.dims[1] = v.dims[2] = 1;
    v.data = single_arg(prhs[3], nv, (size_t)nm, "y must be single [Nvox, Nmeas]");
    v.theta0 = single_arg(prhs[4], nv, (size_t)nvar, "x0 must be single [Nvox, Nparam + 1] (noise last)");
    const mxArray* f = prhs[5];
    need(mxIsDouble(prhs[6]) && mxIsDouble(prhs[7]) && (int)mxGetNumberOfElements(prhs[6]) >= nvar &&
             (int)mxGetNumberOfElements(prhs[7]) >= nvar,
         "lb / ub must be double with one entry per variable (noise last)");
    gx_mcmc_opts o;
    memset(&o, 0, sizeof(o));
    o.algorithm = (fstr_is(f, "algorithm", "ensemble", 0) || fstr_is(f, "algorithm", "gw", 0)) ? GX_MCMC_ENSEMBLE
                                                                                              : GX_MCMC_MH;
    o.iteration = fint(f, "iteration", 200000);
    o.thinning = fint(f, "thinning", 20);
    o.burnin = fdouble(f, "burnin", 0.1);
    o.repetition = fint(f, "repetition", 1);
    o.nwalker = o.algorithm == GX_MCMC_ENSEMBLE ? fint(f, "Nwalker", 50) : 1;
    o.step_size = fdouble(f, "StepSize", 2.0);
    o.start_range = fdouble(f, "startRange", 0.001);
    o.ensemble_update = fstr_is(f, "Ensembleupdate", "redblack", 0) ? GX_GW_REDBLACK : GX_GW_SIMULTANEOUS;
    o.x_step = (nrhs > 8 && !mxIsEmpty(prhs[8])) ? mxGetPr(prhs[8]) : NULL;
    need(o.algorithm == GX_MCMC_ENSEMBLE || o.x_step != NULL, "MH needs xstep");
    o.lb = mxGetPr(prhs[6]);
    o.ub = mxGetPr(prhs[7]);
    o.seed = (uint64_t)fdouble(f, "seed", 0.0);
    o.nbin = fint(f, "Nbin", 1001);
    int want_med = 0, want_iqr = 0, want_mode = 0;
    const mxArray* met = mxGetField(f, 0, "metric");
    if (met && mxIsCell(met))
        for (size_t i = 0; i < mxGetNumberOfElements(met); ++i) {
            char buf[16];
            const mxArray* e = mxGetCell(met, i);
            if (e && mxIsChar(e) && mxGetString(e, buf, sizeof(buf)) == 0) {
                want_med |= strcmp(buf, "median") == 0;
                want_iqr |= strcmp(buf, "iqr") == 0;
                want_mode |= strcmp(buf, "mode") == 0;
            }
        }
    gx_mcmc_result r;
    memset(&r, 0, sizeof(r));
    const char* names[] = {"mean", "std", "median", "iqr", "mode", "acceptance"};
    mxArray* out = mxCreateStructMatrix(1, 1, 6, names);
    mxSetField(out, 0, "mean", single_out(nv, (size_t)nvar, &r.mean));
    mxSetField(out, 0, "std", single_out(nv, (size_t)nvar, &r.std));
    if (want_med) mxSetField(out, 0, "median", single_out(nv, (size_t)nvar, &r.median));
    if (want_iqr) mxSetField(out, 0, "iqr", single_out(nv, (size_t)nvar, &r.iqr));
    if (want_mode) mxSetField(out, 0, "mode", single_out(nv, (size_t)nvar, &r.mode));
    gx_status st = gx_mcmc(c, &mb.m, GX_MEM_HOST, &v, 1, &o, &r);
    if (st != GX_OK) mxDestroyArray(out);
    check(st);
    mxSetField(out, 0, "acceptance",
               mxCreateDoubleScalar(r.n_proposals > 0 ? (double)r.n_accepted / (double)r.n_proposals : 0.0));
    plhs[0] = out;
}

/* ---- forward ------------------------------------------------------------- */
static void do_forward(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    need(nrhs >= 4, "forward: ctx, model, theta [, aux]");
    gx_context* c = ctx_arg(prhs[1]);
    model_buf mb;
    int np, nm;
    model_arg(prhs[2], &mb, &np, &nm);
    const size_t nv = mxGetM(prhs[3]);
    const float* th = single_arg(prhs[3], nv, (size_t)np, "theta must be single [Nvox, Nparam]");
    const float* aux = (nrhs > 4 && !mxIsEmpty(prhs[4])) ? single_arg(prhs[4], nv, 1, "aux: single [Nvox, 1]") : NULL;
    float* s;
    mxArray* out = single_out(nv, (size_t)nm, &s);
    gx_status st = gx_forward(c, &mb.m, GX_MEM_HOST, th, aux, (int32_t)nv, s);
    if (st != GX_OK) mxDestroyArray(out);
    check(st);
    plhs[0] = out;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    char cmd[16];
    need(nrhs >= 1 && mxIsChar(prhs[0]) && mxGetString(prhs[0], cmd, sizeof(cmd)) == 0,
         "first argument: 'context', 'destroy', 'forward', 'askadam' or 'mcmc'");
    if (strcmp(cmd, "context") == 0) {
        gx_context* c = NULL;
        check(gx_context_create(nrhs > 1 ? (int32_t)mxGetScalar(prhs[1]) : 0, &c));
        plhs[0] = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
        *(uint64_t*)mxGetData(plhs[0]) = (uint64_t)(uintptr_t)c;
    } else if (strcmp(cmd, "destroy") == 0) {
        need(nrhs >= 2, "destroy: ctx");
        check(gx_context_destroy(ctx_arg(prhs[1])));
    } else if (strcmp(cmd, "forward") == 0) {
        do_forward(plhs, nrhs, prhs);
    } else if (strcmp(cmd, "askadam") == 0) {
        do_askadam(nlhs, plhs, nrhs, prhs);
    } else if (strcmp(cmd, "mcmc") == 0) {
        do_mcmc(plhs, nrhs, prhs);
    } else {
        mexErrMsgIdAndTxt("GACELLE:b200:invalidArgument", "unknown command '%s'", cmd);
    }
}
