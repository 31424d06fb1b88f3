"""Host-side mirror of GACELLE's ``mcmc`` class (utils/mcmc.m) running the
samplers of the built-in models on the B200 engine.

``mcmc().optimisation(data, mask, weights, pars0, fitting, model, ...)`` keeps
the reference's argument order (utils/mcmc.m:18-80).  The last model
parameter is the Gaussian noise sigma, as in the reference's contracts.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, utils
from ._lib import GacelleError, GX_EINVAL
from .askadam_solver import _model_of

POSTERIOR_LIMIT_BYTES = 1 << 30  # default cap for returning out['posterior']


def check_set_default_basic(fitting: dict | None) -> dict:
    """mcmc.check_set_default_basic (utils/mcmc.m:633-679)."""
    g = dict(fitting or {})
    d = g.setdefault
    d("iteration", 2e5)
    d("thinning", 20)
    d("metric", ["mean", "std"])
    d("burnin", 0.1)
    d("repetition", 1)
    d("outputFilename", [])
    d("algorithm", "MH")
    d("StepSize", 2)
    d("Nwalker", 50)
    d("ub", [])
    d("lb", [])
    d("startRange", 0.001)
    d("Ensembleupdate", "simultaneous")
    d("globalWarmup", 0)
    if isinstance(g["metric"], str):
        g["metric"] = [g["metric"]]
    if "mode" in [m.lower() for m in g["metric"]]:
        d("Nbin", 1001)
    d("autoMemManage", True)
    if str(g["algorithm"]).lower() == "gw":
        g["algorithm"] = "ensemble"
    return g


def get_number_burnin(fitting) -> int:
    """mcmc.get_number_burnin (utils/mcmc.m:788-794)."""
    b = fitting["burnin"]
    return int(np.floor(fitting["iteration"] * b)) if b < 1 else int(b)


def number_of_samples(fitting) -> int:
    """Ns = numel(Nburnin+1:thinning:iteration)."""
    nb = get_number_burnin(fitting)
    it = int(fitting["iteration"])
    return 0 if nb + 1 > it else (it - nb - 1) // int(fitting["thinning"]) + 1


class mcmc:
    """MCMC solvers (utils/mcmc.m) on the B200 engine."""

    def __init__(self, context=None):
        self.ctx = context
        self.last_timing = None
        self.last_stats = None

    check_set_default_basic = staticmethod(check_set_default_basic)
    get_number_burnin = staticmethod(get_number_burnin)

    @staticmethod
    def save_mcmc_output(outputFilename, out):
        """utils/mcmc.m:702-718: save ``out`` to a MAT-file when a file name
        is given."""
        return utils.save_output(outputFilename, out)

    def optimisation(self, data, mask, weights, pars0, fitting, FWDfunc, *varargin, extradata=None):
        """mcmc.optimisation (utils/mcmc.m:18-80)."""
        model = _model_of(FWDfunc)
        fitting = check_set_default_basic(fitting)
        mask = np.asarray(mask)
        idx = utils.mask_index(mask)
        y = utils.to_GD(data, mask, idx).astype(np.float32)
        nm, nv = y.shape
        names = list(fitting.get("modelParams") or model.modelParams)
        if names[-1] != "noise":
            raise GacelleError(GX_EINVAL, "the last MCMC parameter must be 'noise'")
        sizes = model.nparam_nmeas()
        if sizes[0] + 1 != len(names) or sizes[1] != nm:
            raise GacelleError(GX_EINVAL, "modelParams / data size do not match the model")
        # a start field with one value while another has one per voxel marks a
        # global parameter: the ensemble sampler becomes
        # goodman_weare_wglobal_constant (mcmc.m:52-74, check_global_constant :775-785);
        # Metropolis-Hastings broadcasts the value as the reference's struct2array does
        sizes_glob = [np.size(pars0[p]) for p in names]
        is_global = None
        if fitting["algorithm"].lower() == "ensemble" and any(s == 1 for s in sizes_glob) \
                and any(s > 1 for s in sizes_glob):
            is_global = [1 if s == 1 else 0 for s in sizes_glob]
        x0 = np.stack([utils.param_to_GD(pars0[p], mask, idx, nv) for p in names]).astype(np.float32)
        w = None
        if weights is not None and np.size(weights) > 0:
            w = utils.to_GD(weights, mask, idx).astype(np.float32)
            if np.all(w == 1):
                w = None
        ex = dict(extradata or {})
        for a in varargin:
            if isinstance(a, dict) and "b1" in a:
                ex.update(a)
        b1 = utils.param_to_GD(ex["b1"], mask, idx, nv).astype(np.float32) if "b1" in ex else None
        metrics = [m.lower() for m in fitting["metric"]]
        ns = number_of_samples(fitting)
        W = int(fitting["Nwalker"]) if fitting["algorithm"].lower() == "ensemble" else 1
        post_bytes = 4 * len(names) * nv * W * ns * int(fitting["repetition"])
        want_post = fitting.get("returnPosterior", post_bytes <= POSTERIOR_LIMIT_BYTES)
        res = self._run(model, y, w, x0, b1, names, fitting, want_post, is_global,
                        stats=[m for m in ("median", "iqr", "mode") if m in metrics])
        return self.res2out(res, fitting, mask, names)

    def _run(self, model, y, w, x0, b1, names, fitting, want_post, is_global=None, stats=()):
        """stats: any of 'median', 'iqr', 'mode', computed on the device."""
        ctx = self.ctx or _lib.Context.default()
        nvar = len(names)
        nm, nv = y.shape
        alg = fitting["algorithm"].lower()
        W = int(fitting["Nwalker"]) if alg == "ensemble" else 1
        ns = number_of_samples(fitting)
        rep = int(fitting["repetition"])
        lb = np.ascontiguousarray(np.asarray(fitting["lb"], dtype=np.float64).ravel()[:nvar])
        ub = np.ascontiguousarray(np.asarray(fitting["ub"], dtype=np.float64).ravel()[:nvar])
        xs = np.ascontiguousarray(np.asarray(fitting.get("xStepSize", np.zeros(nvar)), dtype=np.float64).ravel()[:nvar])
        o = _lib.GxMcmcOpts()
        o.algorithm = 1 if alg == "ensemble" else 0
        o.iteration = int(fitting["iteration"])
        o.thinning = int(fitting["thinning"])
        o.burnin = float(fitting["burnin"])
        o.repetition = rep
        o.nwalker = W
        o.step_size = float(fitting["StepSize"])
        o.start_range = float(fitting["startRange"])
        o.ensemble_update = 1 if str(fitting["Ensembleupdate"]).lower() == "redblack" else 0
        o.x_step = xs.ctypes.data_as(_lib._dp)
        o.lb = lb.ctypes.data_as(_lib._dp)
        o.ub = ub.ctypes.data_as(_lib._dp)
        o.seed = int(fitting.get("seed", model.seed))
        o.block_size = int(fitting.get("blockSize", 0))
        o.nbin = int(fitting.get("Nbin", 1001))
        keep = [y, x0]
        if is_global is not None:
            ig = np.ascontiguousarray(is_global, dtype=np.int32)
            keep.append(ig)
            o.is_global = ig.ctypes.data_as(_lib._i32p)
            o.global_warmup = int(fitting.get("globalWarmup", 0))
        vol = _lib.GxVolume()
        vol.dims[0], vol.dims[1], vol.dims[2] = nv, 1, 1
        vol.nvox = nv
        vol.data = y.ctypes.data_as(_lib._fp)
        if w is not None:
            w = np.ascontiguousarray(w, np.float32)
            keep.append(w)
            vol.weights = w.ctypes.data_as(_lib._fp)
        vol.theta0 = x0.ctypes.data_as(_lib._fp)
        if b1 is not None:
            b1 = np.ascontiguousarray(b1, np.float32)
            keep.append(b1)
            vol.b1 = b1.ctypes.data_as(_lib._fp)
        mean = np.zeros((nvar, nv), np.float32)
        std = np.zeros((nvar, nv), np.float32)
        post = np.zeros((nvar, rep, ns, W, nv), np.float32) if want_post else None
        r = _lib.GxMcmcResult()
        r.mean = mean.ctypes.data_as(_lib._fp)
        r.std = std.ctypes.data_as(_lib._fp)
        if post is not None:
            r.posterior = post.ctypes.data_as(_lib._fp)
        summaries = {}
        for m in stats:
            summaries[m] = np.zeros((nvar, nv), np.float32)
            setattr(r, m, summaries[m].ctypes.data_as(_lib._fp))
        _lib.check(_lib.lib().gx_mcmc(ctx.ptr, C.byref(model._gx_model().s), _lib.MEM_HOST, C.byref(vol), 1,
                                      C.byref(o), C.byref(r)))
        self.last_timing = ctx.timing()
        self.last_stats = {"n_accepted": r.n_accepted, "n_proposals": r.n_proposals, "ns": r.ns,
                           "n_global_accepted": r.n_global_accepted, "n_global_proposals": r.n_global_proposals}
        return {"mean": mean, "std": std, "posterior": post, "W": W, "ns": ns, "rep": rep, **summaries,
                "is_global": list(is_global) if is_global is not None else [0] * nvar}

    @staticmethod
    def res2out(res, fitting, mask, names):
        """mcmc.res2out (utils/mcmc.m:806-862)."""
        shape = np.shape(mask)
        out = {}
        post = res["posterior"]
        nv = res["mean"].shape[1]
        isg = res.get("is_global") or [0] * len(names)
        if post is not None:
            # [Nv, Nwalker, Ns, rep] per parameter (MH: [Nv, Ns, rep]); a global
            # parameter keeps a leading dimension of 1 (array2struct_wglobal)
            out["posterior"] = {}
            for k, p in enumerate(names):
                a = np.transpose(post[k], (3, 2, 1, 0))  # [nv, W, ns, rep]
                if isg[k]:
                    a = a[:1]
                out["posterior"][p] = a[:, 0] if res["W"] == 1 else a
        for m in [m.lower() for m in fitting["metric"]]:
            out[m] = {}
            for k, p in enumerate(names):
                if m in ("mean", "std", "median", "iqr", "mode") and m in res:
                    v = res[m][k]   # computed on the device
                else:
                    raise GacelleError(GX_EINVAL, f"unknown metric {m}")
                if isg[k]:
                    # one value for all voxels: a scalar, as reshape_ND2image passes it
                    out[m][p] = float(np.asarray(v).ravel()[0])
                    continue
                out[m][p] = utils.reshape_GD2ND(np.asarray(v, dtype=np.float32), mask).reshape(shape, order="F")
        return out

    # direct-solver entry points of the reference (utils/mcmc.m:82, :192)
    def metropolis_hastings(self, y, x0, weights, fitting, FWDfunc, *varargin):
        f = dict(fitting)
        f["algorithm"] = "MH"
        return self._direct(y, x0, weights, f, FWDfunc, varargin)

    def goodman_weare(self, y, x0, weights, fitting, FWDfunc, *varargin):
        f = dict(fitting)
        f["algorithm"] = "ensemble"
        return self._direct(y, x0, weights, f, FWDfunc, varargin)

    def goodman_weare_wglobal_constant(self, y, x0, weights, fitting, FWDfunc, *varargin):
        """Direct entry of the global-parameter sampler (utils/mcmc.m:385): the
        fields of x0 with one value are the global parameters."""
        f = dict(fitting)
        f["algorithm"] = "ensemble"
        return self._direct(y, x0, weights, f, FWDfunc, varargin)

    def _direct(self, y, x0, weights, fitting, FWDfunc, varargin):
        """Returns xPosterior as {param: [Nv, Nwalker, Ns, rep]}."""
        y = np.asarray(y)
        mask = np.ones((1, y.shape[1]), dtype=bool)
        f = check_set_default_basic(fitting)
        f["returnPosterior"] = True
        f["metric"] = []
        out = self.optimisation(y, mask, weights, x0, f, FWDfunc, *varargin)
        return out["posterior"]
