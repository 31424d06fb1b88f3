"""ctypes front end of the FP64 oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, always as
the checker or the timed CPU restatement, never as the product path.

PARITY UNPINNED against MATLAB runs of the reference (kschan0214/gacelle is
MATLAB-only, depends on closed toolboxes, and ships no golden vectors); see
``oracle.h`` for what pins the restatement instead.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

MODEL_R2S, MODEL_R1R2S, MODEL_NEXI, MODEL_NEXI_RICE = 1, 2, 3, 4
LOSS = {"l1": 0, "l2": 1, "huber": 2, "mse": 3, "gauss": 4, "rician": 5}
OPTIMISER = {"adam": 0, "sgdm": 1, "rmsprop": 2}
TRANSFORM = {"sigmoid": 0, "linear": 1}
CONV_MODEL = {"ema": 0, "linear": 1}
STOP_REASONS = {0: "none", 1: "convergence", 2: "tol", 3: "step", 4: "grad"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)


class OrcModel(C.Structure):
    _fields_ = [("model", C.c_int), ("lmax", C.c_int), ("nx", C.c_int),
                ("n_te", C.c_int), ("te", _dp), ("n_fa", C.c_int), ("fa_deg", _dp),
                ("tr", C.c_double), ("n_shell", C.c_int), ("bval", _dp), ("delta", _dp)]


class OrcAdamOpts(C.Structure):
    _fields_ = [("iteration", C.c_int), ("lr", C.c_double), ("decay", C.c_double),
                ("optimiser", C.c_int), ("beta1", C.c_double), ("beta2", C.c_double),
                ("eps", C.c_double), ("momentum", C.c_double), ("rms_decay", C.c_double),
                ("rms_eps", C.c_double), ("loss", C.c_int), ("mse_scale", C.c_double),
                ("huber_delta", C.c_double), ("sigma", C.c_double), ("transform", C.c_int),
                ("randomness", C.c_double), ("seed", C.c_uint64), ("lb", _dp), ("ub", _dp),
                ("tol", C.c_double), ("conv_value", C.c_double), ("conv_window", C.c_int),
                ("patience_conv", C.c_double), ("conv_model", C.c_int), ("ema_decay", C.c_double),
                ("step_tol", C.c_double), ("grad_tol", C.c_double), ("patience_step", C.c_double),
                ("patience_grad", C.c_double), ("n_reg", C.c_int), ("reg_param", C.c_int * 8),
                ("lambda_", C.c_double * 8), ("tv_3d", C.c_int), ("voxel_size", C.c_double * 3),
                ("nthreads", C.c_int), ("state_f32", C.c_int), ("robust", C.c_int),
                ("outlier_weight", C.c_double), ("weight_update_interval", C.c_int),
                ("outlier_check_window", C.c_int), ("outlier_voxel_thres", C.c_double),
                ("outlier_pop_thres", C.c_double), ("outlier_init_thres", C.c_double),
                ("outlier_init_pop_thres", C.c_double), ("reg_type", C.c_int)]


class OrcVolume(C.Structure):
    _fields_ = [("dims", C.c_int * 3), ("nvox", C.c_int), ("grid_index", _ip),
                ("data", _dp), ("weights", _dp), ("theta0", _dp), ("b1", _dp), ("sigma", _dp),
                ("norm_nvox", C.c_double), ("prior_mu", _dp), ("prior_sd", _dp), ("prior_offset", C.c_double),
                ("max_neighbours", C.c_int), ("neighbours", _ip), ("edge_length", _dp)]


class OrcAdamResult(C.Structure):
    _fields_ = [("final_theta", _dp), ("min_theta", _dp), ("final_residual", _dp),
                ("min_residual", _dp), ("loss_history", _dp), ("final_loss", C.c_double),
                ("final_fid", C.c_double), ("final_reg", C.c_double), ("min_loss", C.c_double),
                ("min_fid", C.c_double), ("min_reg", C.c_double), ("final_niter", C.c_int),
                ("min_niter", C.c_int), ("stop_reason", C.c_int), ("ever_flagged", C.POINTER(C.c_ubyte))]


class OrcMcmcOpts(C.Structure):
    _fields_ = [("algorithm", C.c_int), ("iteration", C.c_int), ("thinning", C.c_int),
                ("burnin", C.c_double), ("repetition", C.c_int), ("nwalker", C.c_int),
                ("step_size", C.c_double), ("start_range", C.c_double),
                ("ensemble_update", C.c_int), ("x_step", _dp), ("lb", _dp), ("ub", _dp),
                ("seed", C.c_uint64), ("nthreads", C.c_int), ("is_global", _ip),
                ("global_warmup", C.c_int)]


class OrcMcmcResult(C.Structure):
    _fields_ = [("mean", _dp), ("std", _dp), ("posterior", _fp), ("n_accepted", C.c_longlong),
                ("n_proposals", C.c_longlong), ("ns", C.c_int)]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(os.path.join(_HERE, f))
                                              for f in ("oracle.c", "oracle.h"))):
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "liboracle.so"], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.orc_nparams.argtypes = [C.POINTER(OrcModel)]
        L.orc_nmeas.argtypes = [C.POINTER(OrcModel)]
        L.orc_forward.argtypes = [C.POINTER(OrcModel), _dp, _dp, C.c_int, _dp]
        L.orc_forward_voxel.argtypes = [C.POINTER(OrcModel), _dp, C.c_double, _dp]
        L.orc_vjp_voxel.argtypes = [C.POINTER(OrcModel), _dp, C.c_double, _dp, _dp]
        for f in ("orc_loss_value", "orc_loss_deriv"):
            getattr(L, f).argtypes = [C.c_int] + [C.c_double] * 6
            getattr(L, f).restype = C.c_double
        for f in ("orc_i0e", "orc_i1e"):
            getattr(L, f).argtypes = [C.c_double]
            getattr(L, f).restype = C.c_double
        L.orc_besseli_trapz.argtypes = [C.c_int, C.c_double, C.c_int]
        L.orc_besseli_trapz.restype = C.c_double
        L.orc_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_u01.argtypes = [C.c_uint32]
        L.orc_u01.restype = C.c_double
        L.orc_askadam.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcVolume), C.POINTER(OrcAdamOpts),
                                  C.POINTER(OrcAdamResult)]
        L.orc_model_gradient.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcVolume),
                                         C.POINTER(OrcAdamOpts), _dp, _dp, _dp, _dp, _dp]
        L.orc_model_gradient.restype = C.c_double
        L.orc_mcmc.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcVolume), _dp,
                               C.POINTER(OrcMcmcOpts), C.POINTER(OrcMcmcResult)]
        L.orc_mcmc_nsamples.argtypes = [C.c_int, C.c_double, C.c_int]
        L.orc_gw_partner.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, _ip]
        L.orc_dictionary_match.argtypes = [_dp, C.c_int, _dp, C.c_int, C.c_int, _dp, _ip, _dp]
        L.orc_dictionary_match.restype = None
        L.orc_tv_cost.argtypes = [_ip, C.POINTER(C.c_ubyte), _dp, C.c_int, _dp]
        L.orc_tv_cost.restype = C.c_double
        L.orc_tv_grad.argtypes = [_ip, C.POINTER(C.c_ubyte), _dp, C.c_int, _dp, _dp]
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Model:
    """Protocol + model choice.  Keeps the numpy arrays alive for the struct."""

    def __init__(self, model: int, te=None, fa_deg=None, tr=0.0, bval=None, delta=None,
                 lmax=0, nx=14):
        self.model = model
        self.te = _f64(te) if te is not None else np.zeros(1)
        self.fa_deg = _f64(fa_deg) if fa_deg is not None else np.zeros(1)
        self.bval = _f64(bval) if bval is not None else np.zeros(1)
        self.delta = _f64(delta) if delta is not None else np.zeros(1)
        self.s = OrcModel(model, lmax, nx, len(self.te) if te is not None else 0, _d(self.te),
                          len(self.fa_deg) if fa_deg is not None else 0, _d(self.fa_deg), tr,
                          len(self.bval) if bval is not None else 0, _d(self.bval), _d(self.delta))

    @property
    def np(self):
        return lib().orc_nparams(C.byref(self.s))

    @property
    def nm(self):
        return lib().orc_nmeas(C.byref(self.s))


def r2s(te):
    return Model(MODEL_R2S, te=te)


def r1r2s(te, fa_deg, tr):
    return Model(MODEL_R1R2S, te=te, fa_deg=fa_deg, tr=tr)


def nexi(bval, delta, lmax=0, nx=14):
    return Model(MODEL_NEXI, bval=bval, delta=delta, lmax=lmax, nx=nx)


def nexi_rice(bval, delta, nx=14):
    """gpuNEXIrice (NEXI/gpuNEXIrice.m): Rician mean of the lmax-0 NEXI signal;
    the per-voxel noise sigma is passed where R1R2* takes b1."""
    return Model(MODEL_NEXI_RICE, bval=bval, delta=delta, lmax=0, nx=nx)


def forward(model: Model, theta, b1=None):
    """b1: per-voxel model input (b1 for R1R2*, sigma for the NEXI Rician mean)."""
    theta = _f64(theta)
    nv = theta.shape[1]
    out = np.empty((model.nm, nv))
    b1 = _f64(b1)
    lib().orc_forward(C.byref(model.s), _d(theta), _d(b1), nv, _d(out))
    return out


def vjp_voxel(model: Model, theta, sbar, b1=1.0):
    theta = _f64(theta)
    sbar = _f64(sbar)
    tb = np.zeros(model.np)
    lib().orc_vjp_voxel(C.byref(model.s), _d(theta), b1, _d(sbar), _d(tb))
    return tb


def loss_value(loss, s, y, w=1.0, sigma=1.0, mse_scale=0.5, huber_delta=1.0):
    return lib().orc_loss_value(LOSS[loss], s, y, w, sigma, mse_scale, huber_delta)


def loss_deriv(loss, s, y, w=1.0, sigma=1.0, mse_scale=0.5, huber_delta=1.0):
    return lib().orc_loss_deriv(LOSS[loss], s, y, w, sigma, mse_scale, huber_delta)


def i0e(x):
    return lib().orc_i0e(float(x))


def i1e(x):
    return lib().orc_i1e(float(x))


def besseli_trapz(nu, z, nx=34):
    return lib().orc_besseli_trapz(nu, float(z), nx)


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox(c, k, o)
    return list(o)


def u01(x):
    return lib().orc_u01(x)


def gw_partner(seed, step, rep, nwalker):
    p = np.zeros(nwalker, dtype=np.int32)
    lib().orc_gw_partner(seed, step, rep, nwalker, p.ctypes.data_as(_ip))
    return p


def dictionary_match(signals, dictionary, wt=None):
    """gpuNEXI.likelihood (NEXI/gpuNEXI.m:813-836) on the FP64 oracle:
    signals [nm][nvox], dictionary [nm][ndict]; returns (best index, best sse)."""
    s = np.ascontiguousarray(signals, dtype=np.float64)
    d = np.ascontiguousarray(dictionary, dtype=np.float64)
    nm, nv = s.shape
    w = None if wt is None else np.ascontiguousarray(wt, dtype=np.float64)
    best = np.zeros(nv, dtype=np.int32)
    sse = np.zeros(nv)
    lib().orc_dictionary_match(_d(s), nv, _d(d), d.shape[1], nm, _d(w), best.ctypes.data_as(_ip), _d(sse))
    return best, sse


def tv_cost(mask3d, img3d, tv_3d=True, voxel_size=(2.0, 2.0, 2.0)):
    dims = np.array(mask3d.shape, dtype=np.int32)
    m = np.asfortranarray(mask3d.astype(np.uint8))
    im = np.asfortranarray(img3d.astype(np.float64))
    vs = np.array(voxel_size, dtype=np.float64)
    return lib().orc_tv_cost(dims.ctypes.data_as(_ip), m.ctypes.data_as(C.POINTER(C.c_ubyte)),
                             im.ctypes.data_as(_dp), int(tv_3d), _d(vs))


def tv_grad(mask3d, img3d, tv_3d=True, voxel_size=(2.0, 2.0, 2.0)):
    dims = np.array(mask3d.shape, dtype=np.int32)
    m = np.asfortranarray(mask3d.astype(np.uint8))
    im = np.asfortranarray(img3d.astype(np.float64))
    vs = np.array(voxel_size, dtype=np.float64)
    g = np.zeros(im.shape, order="F")
    lib().orc_tv_grad(dims.ctypes.data_as(_ip), m.ctypes.data_as(C.POINTER(C.c_ubyte)),
                      im.ctypes.data_as(_dp), int(tv_3d), _d(vs), g.ctypes.data_as(_dp))
    return g


class Volume:
    """One masked volume in the oracle's SoA layout: arrays are [k][nvox]."""

    def __init__(self, data, dims=None, grid_index=None, weights=None, theta0=None, b1=None,
                 sigma=None, norm_nvox=0.0, prior_mu=None, prior_sd=None, prior_offset=0.0,
                 neighbours=None, edge_length=None):
        self.data = _f64(data)
        nv = self.data.shape[1]
        self.grid_index = None if grid_index is None else np.ascontiguousarray(grid_index, np.int32)
        self.weights = _f64(weights)
        self.theta0 = _f64(theta0)
        self.b1 = _f64(b1)
        self.sigma = _f64(sigma)
        dims = dims if dims is not None else (nv, 1, 1)
        self.s = OrcVolume((C.c_int * 3)(*dims), nv,
                           None if self.grid_index is None else self.grid_index.ctypes.data_as(_ip),
                           _d(self.data), _d(self.weights), _d(self.theta0), _d(self.b1),
                           _d(self.sigma), float(norm_nvox))
        self.prior_mu = _f64(prior_mu)
        self.prior_sd = _f64(prior_sd)
        self.s.prior_mu = _d(self.prior_mu)
        self.s.prior_sd = _d(self.prior_sd)
        self.s.prior_offset = float(prior_offset)
        self.neighbours = None if neighbours is None else np.ascontiguousarray(neighbours, np.int32)
        self.edge_length = _f64(edge_length)
        if self.neighbours is not None:
            self.s.max_neighbours = self.neighbours.shape[0]
            self.s.neighbours = self.neighbours.ctypes.data_as(_ip)
            self.s.edge_length = _d(self.edge_length)

    @property
    def nvox(self):
        return self.data.shape[1]


def adam_opts(lb, ub, fitting: dict):
    """Map a GACELLE ``fitting`` dict (askadam defaults already applied) to
    the oracle's option struct."""
    f = fitting
    o = OrcAdamOpts()
    o.iteration = int(f["iteration"])
    o.lr = f["initialLearnRate"]
    o.decay = f["decayRate"]
    o.optimiser = OPTIMISER[f["optimiser"].lower()]
    o.beta1 = f.get("adamupdateGradDecay", 0.9)
    o.beta2 = f.get("adamupdateSqGradDecay", 0.999)
    o.eps = f.get("adamupdateEpsilon", 1e-8)
    o.momentum = f.get("sgdmupdateMomentum", 0.9)
    o.rms_decay = f.get("rmspropupdateSqGradDecay", 0.9)
    o.rms_eps = f.get("rmspropupdateEpsilon", 1e-8)
    o.loss = LOSS[f["lossFunction"].lower()]
    o.mse_scale = f.get("mseScale", 0.5)
    o.huber_delta = f.get("huberTransitionPoint", 1.0)
    o.sigma = f.get("noiseSigma", 1.0)
    o.transform = TRANSFORM[f["parameterTransform"]]
    o.randomness = f["randomness"]
    o.seed = int(f.get("seed", 0))
    lb = _f64(lb)
    ub = _f64(ub)
    o._keep = (lb, ub)
    o.lb = _d(lb)
    o.ub = _d(ub)
    o.tol = f["tol"]
    o.conv_value = f["convergenceValue"]
    o.conv_window = int(f["convergenceWindow"])
    o.patience_conv = float(f["patienceConvergence"])
    o.conv_model = CONV_MODEL[f["convergenceModel"]]
    o.ema_decay = f["emaDecay"]
    o.step_tol = f["convergenceStepTol"]
    o.grad_tol = f["convergenceGradTol"]
    o.patience_step = float(f["patienceStep"])
    o.patience_grad = float(f["patienceGrad"])
    o.robust = 1 if f.get("robustConvergence") else 0
    o.outlier_weight = f.get("outlierWeight", 0.1)
    o.weight_update_interval = int(f.get("weightUpdateInterval", 5))
    o.outlier_check_window = int(f.get("outlierCheckWindow", 5))
    o.outlier_voxel_thres = f.get("outlierVoxelThres", 0.01)
    o.outlier_pop_thres = f.get("outlierPopThres", 0.05)
    o.outlier_init_thres = f.get("outlierInitThres", 0.05)
    o.outlier_init_pop_thres = f.get("outlierInitPopThres", 0.20)
    reg = f.get("_reg_index", [])
    lam = f.get("_reg_lambda", [])
    o.n_reg = len(reg)
    for i, (k, l) in enumerate(zip(reg, lam)):
        o.reg_param[i] = k
        o.lambda_[i] = l
    o.reg_type = 1 if str(f.get("regularisationType", "TV")).lower() == "prior" else 0
    if o.reg_type == 0 and str(f.get("dataType", "volumetric")).lower() == "surface":
        o.reg_type = 2
    o.tv_3d = 1 if str(f.get("TVmode", "2D")).upper() == "3D" else 0
    vs = list(f.get("voxelSize", [2, 2, 2])) + [1.0] * 3
    for i in range(3):
        o.voxel_size[i] = float(vs[i])
    o.nthreads = int(f.get("nthreads", os.cpu_count() or 1))
    o.state_f32 = int(bool(f.get("_state_f32", False)))
    return o


def askadam(model: Model, vol: Volume, opts: OrcAdamOpts, want_min=True, want_residual=False,
            want_history=True):
    np_, nm, nv = model.np, model.nm, vol.nvox
    res = OrcAdamResult()
    final = np.zeros((np_, nv))
    mn = np.zeros((np_, nv)) if want_min else None
    fr = np.zeros((nm, nv)) if want_residual else None
    mr = np.zeros((nm, nv)) if want_residual else None
    hist = np.zeros(opts.iteration + 1) if want_history else None
    res.final_theta = _d(final)
    res.min_theta = _d(mn)
    res.final_residual = _d(fr)
    res.min_residual = _d(mr)
    res.loss_history = _d(hist)
    flagged = np.zeros(nv, dtype=np.uint8)
    res.ever_flagged = flagged.ctypes.data_as(C.POINTER(C.c_ubyte))
    rc = lib().orc_askadam(C.byref(model.s), C.byref(vol.s), C.byref(opts), C.byref(res))
    if rc != 0:
        raise RuntimeError(f"orc_askadam failed ({rc})")
    return {"final": final, "min": mn, "final_residual": fr, "min_residual": mr,
            "loss_history": hist, "final_loss": res.final_loss, "final_fid": res.final_fid,
            "final_reg": res.final_reg, "min_loss": res.min_loss, "min_fid": res.min_fid,
            "min_reg": res.min_reg, "final_niter": res.final_niter, "min_niter": res.min_niter,
            "stop_reason": STOP_REASONS[res.stop_reason], "ever_flagged": flagged.astype(bool)}


def model_gradient(model: Model, vol: Volume, opts: OrcAdamOpts, theta):
    theta = _f64(theta)
    g = np.zeros_like(theta)
    resid = np.zeros((model.nm, vol.nvox))
    fid = C.c_double()
    reg = C.c_double()
    L = lib().orc_model_gradient(C.byref(model.s), C.byref(vol.s), C.byref(opts), _d(theta),
                                 _d(g), _d(resid), C.byref(fid), C.byref(reg))
    return L, g, resid, fid.value, reg.value


def mcmc(model: Model, vol: Volume, x0, lb, ub, algorithm="ensemble", iteration=1000,
         thinning=10, burnin=0.1, repetition=1, nwalker=16, step_size=2.0, start_range=0.001,
         ensemble_update="simultaneous", x_step=None, seed=0, want_posterior=False,
         nthreads=None, is_global=None, global_warmup=0):
    """is_global [nvar] (nonzero: one value per walker shared by all voxels)
    selects goodman_weare_wglobal_constant (utils/mcmc.m:385-626)."""
    x0 = _f64(x0)
    nvar, nv = x0.shape
    lb = _f64(lb)
    ub = _f64(ub)
    xs = _f64(x_step if x_step is not None else np.zeros(nvar))
    ig = None if is_global is None else np.ascontiguousarray(is_global, dtype=np.int32)
    o = OrcMcmcOpts(1 if algorithm == "ensemble" else 0, iteration, thinning, burnin, repetition,
                    nwalker, step_size, start_range,
                    1 if ensemble_update == "redblack" else 0, _d(xs), _d(lb), _d(ub), seed,
                    nthreads or os.cpu_count() or 1,
                    None if ig is None else ig.ctypes.data_as(_ip), int(global_warmup))
    ns = lib().orc_mcmc_nsamples(iteration, burnin, thinning)
    W = nwalker if algorithm == "ensemble" else 1
    mean = np.zeros((nvar, nv))
    std = np.zeros((nvar, nv))
    post = np.zeros(nvar * nv * W * ns * repetition, dtype=np.float32) if want_posterior else None
    r = OrcMcmcResult(_d(mean), _d(std), None if post is None else post.ctypes.data_as(_fp), 0, 0, 0)
    st = lib().orc_mcmc(C.byref(model.s), C.byref(vol.s), _d(x0), C.byref(o), C.byref(r))
    if st != 0:
        raise ValueError("global parameters need the ensemble algorithm and at least one local "
                         "and one global parameter")
    out = {"mean": mean, "std": std, "n_accepted": r.n_accepted, "n_proposals": r.n_proposals,
           "ns": r.ns}
    if post is not None:
        # [nvar][rep][ns][W][nv] in C order == MATLAB [Nv, W, Ns, rep] per parameter
        out["posterior"] = post.reshape(nvar, repetition, ns, W, nv)
    return out


def res2out_summaries(samples, lb, ub, nbin=1001):
    """The order and histogram summaries of mcmc.res2out (utils/mcmc.m:806-862)
    restated in numpy for one parameter: samples [nvox, N].  median: mean of
    the two middle values for an even count; iqr: prctile(x, 75) - prctile(x,
    25) with the midpoint rule (numpy's 'hazen'); mode: discretize over
    linspace(lb - 1e-8, ub + 1e-8, nbin) (MATLAB's linspace d1 + ((0:n-1)
    (d2 - d1)) / (n - 1), last element d2; bins closed on the left, the last
    one on both sides, samples outside ignored), most populated bin with the
    lowest index on ties, returned as the bin centre (NaN if no sample is
    inside).  Returns float32 arrays [nvox]."""
    x = np.asarray(samples, dtype=np.float64)
    med = np.median(x, axis=1)
    q = np.percentile(x, [25, 75], axis=1, method="hazen")
    iqr = q[1] - q[0]
    d1, d2 = float(lb) - 1e-8, float(ub) + 1e-8
    n1 = nbin - 1
    edges = d1 + (np.arange(nbin, dtype=np.float64) * (d2 - d1)) / n1
    edges[-1] = d2
    mode = np.full(x.shape[0], np.nan)
    for v in range(x.shape[0]):
        xv = x[v]
        inside = (xv >= d1) & (xv <= d2)
        if not inside.any():
            continue
        b = np.searchsorted(edges, xv[inside], side="right") - 1
        b = np.minimum(b, n1 - 1)       # x == d2 falls in the last bin
        cnt = np.bincount(b, minlength=n1)
        k = int(np.argmax(cnt))         # first maximum: the lowest bin
        mode[v] = (edges[k] + edges[k + 1]) / 2
    return med.astype(np.float32), iqr.astype(np.float32), mode.astype(np.float32)
