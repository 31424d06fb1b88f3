"""Host-side mirror of GACELLE's ``askadam`` class (utils/askadam.m) that
dispatches the optimisation of a built-in model to the B200 engine.

``askadam().optimisation(data, mask, weights, pars0, fitting, model, *extra)``
keeps the reference's argument order and meaning (utils/askadam.m:121-135);
``model`` is a built-in model object (or its bound ``FWD``) because the engine
carries hand-written adjoints for the built-in forward models only.  Any other
callable raises ``GACELLE:b200:unsupported``.
"""
from __future__ import annotations

import copy
import math

import numpy as np

from . import _lib
from ._lib import GacelleError, GX_EUNSUPPORTED, GX_EINVAL
from . import utils


def check_set_default_basic(fitting: dict | None) -> dict:
    """askadam.check_set_default_basic (utils/askadam.m:735-878)."""
    f = dict(fitting or {})
    g = dict(f)
    g["defaultRegularisation"] = True
    d = g.setdefault
    d("optimiser", "adam")
    d("initialLearnRate", 0.001)
    d("decayRate", 0.0)
    d("enableComplex", True)
    d("randomness", 0.0)
    d("parameterTransform", "sigmoid")
    opt = g["optimiser"].lower()
    if opt == "adam":
        d("adamupdateGradDecay", 0.9)
        d("adamupdateSqGradDecay", 0.999)
        d("adamupdateEpsilon", 1e-8)
    elif opt == "sgdm":
        d("sgdmupdateMomentum", 0.9)
    elif opt == "rmsprop":
        d("rmspropupdateSqGradDecay", 0.9)
        d("rmspropupdateEpsilon", 1e-8)
    d("lossFunction", "L1")
    d("tol", 1e-3)
    d("iteration", 1e4)
    d("convergenceValue", 1e-6)
    d("patience", 5)
    d("patienceConvergence", g["patience"])
    if "Nepoch" in f:
        g["iteration"] = f["Nepoch"]
        g.pop("Nepoch")
    d("convergenceModel", "ema")
    d("convergenceWindow", 20)
    d("emaDecay", 0.95)
    d("robustConvergence", False)
    d("outlierThresholdMethod", "behaviour")
    d("outlierWeight", 0.1)
    d("weightUpdateInterval", 5)
    d("outlierCheckWindow", 5)
    d("outlierMinFlagDuration", 5)
    d("outlierVoxelThres", 0.01)
    d("outlierPopThres", 0.05)
    d("outlierInitThres", 0.05)
    d("outlierInitPopThres", 0.20)
    d("convergenceStepTol", 1e-6)
    d("convergenceGradTol", 1e-6)
    d("patienceStep", g["patience"])
    d("patienceGrad", g["patience"])
    d("lambda", [0])
    d("TVmode", "2D")
    d("regmap", [])
    d("voxelSize", [2, 2, 2])
    if not isinstance(g["lambda"], (list, tuple)):
        g["lambda"] = list(np.atleast_1d(g["lambda"]))
    d("isOptimiseMemory", True)
    d("autoMemManage", True)
    d("segmentOverlap", 0)
    d("NSegmentUser", [])
    d("outputFilename", [])
    d("ub", [])
    d("lb", [])
    d("debug", False)
    d("isDisplay", 0)
    d("isMaskedOut", True)
    d("isSampleConsistency", False)
    d("isClipGradient", 0)
    d("maxGradientThres", 1)
    return g


def _regulariser_of(userfunc):
    """The regulariser of a two-function ``userFcn`` cell (askadam.model_gradient,
    utils/askadam.m:58-71): only gpuNEXI.prior_distribution_normal is
    accelerated; None for the default spatial TV."""
    if isinstance(userfunc, (list, tuple)) and len(userfunc) > 1:
        name = getattr(userfunc[1], "__name__", "")
        if name == "prior_distribution_normal":
            return "prior"
        if name == "surface_total_variation":
            return "surface"
        raise GacelleError(GX_EUNSUPPORTED, "custom regularisation functions other than "
                                            "prior_distribution_normal and surface_total_variation are not "
                                            "accelerated")
    return None


def _model_of(userfunc):
    """The built-in model object behind ``userfunc`` (object or bound FWD)."""
    if isinstance(userfunc, (list, tuple)):
        _regulariser_of(userfunc)
        userfunc = userfunc[0]
    obj = getattr(userfunc, "__self__", userfunc)
    if not hasattr(obj, "_gx_model"):
        raise GacelleError(GX_EUNSUPPORTED, "only the built-in models (gpuR2starMapping, "
                                            "gpuJointR1R2starMapping, gpuNEXI) are accelerated")
    return obj


def _patience(x):
    x = float(x)
    return x if math.isfinite(x) else float("inf")


def build_opts(fitting: dict, model_params, lb, ub, path="fused"):
    """Flatten a defaulted ``fitting`` dict into gx_askadam_opts."""
    f = fitting
    o = _lib.GxAskadamOpts()
    o.iteration = int(f["iteration"])
    o.initial_learn_rate = float(f["initialLearnRate"])
    o.decay_rate = float(f["decayRate"])
    opt = f["optimiser"].lower()
    if opt not in _lib.OPTIMISER:
        raise GacelleError(GX_EINVAL, f"unknown optimiser {opt}")
    o.optimiser = _lib.OPTIMISER[opt]
    o.beta1 = float(f.get("adamupdateGradDecay", 0.9))
    o.beta2 = float(f.get("adamupdateSqGradDecay", 0.999))
    o.epsilon = float(f.get("adamupdateEpsilon", 1e-8))
    o.momentum = float(f.get("sgdmupdateMomentum", 0.9))
    o.rms_decay = float(f.get("rmspropupdateSqGradDecay", 0.9))
    o.rms_epsilon = float(f.get("rmspropupdateEpsilon", 1e-8))
    loss = f["lossFunction"].lower()
    if loss not in _lib.LOSS:
        raise GacelleError(GX_EINVAL, f"unknown lossFunction {loss}")
    o.loss = _lib.LOSS[loss]
    o.mse_scale = float(f.get("mseScale", 0.5))
    o.huber_delta = float(f.get("huberTransitionPoint", 1.0))
    o.sigma = float(f.get("noiseSigma", 0.0))
    o.transform = _lib.TRANSFORM[f["parameterTransform"]]
    o.randomness = float(f["randomness"])
    o.seed = int(f.get("seed", 0))
    lb = np.ascontiguousarray(lb, dtype=np.float64)
    ub = np.ascontiguousarray(ub, dtype=np.float64)
    o._keep = (lb, ub)
    o.lb = lb.ctypes.data_as(_lib._dp)
    o.ub = ub.ctypes.data_as(_lib._dp)
    o.tol = float(f["tol"])
    o.convergence_value = float(f["convergenceValue"])
    o.convergence_window = int(f["convergenceWindow"])
    o.patience_convergence = _patience(f["patienceConvergence"])
    o.convergence_model = _lib.CONV_MODEL[f["convergenceModel"]]
    o.ema_decay = float(f["emaDecay"])
    o.step_tol = float(f["convergenceStepTol"])
    o.grad_tol = float(f["convergenceGradTol"])
    o.patience_step = _patience(f["patienceStep"])
    o.patience_grad = _patience(f["patienceGrad"])
    lam = [float(x) for x in np.atleast_1d(f["lambda"])]
    regmap = f.get("regmap") or []
    if isinstance(regmap, str):
        regmap = [regmap]
    if lam and lam[0] > 0:
        if len(regmap) < len(lam):
            raise GacelleError(GX_EINVAL, "fitting.regmap needs one entry per lambda")
        o.n_reg = len(lam)
        for i, (name, l) in enumerate(zip(regmap, lam)):
            if name not in model_params:
                raise GacelleError(GX_EINVAL, f"regmap {name} is not a model parameter")
            o.reg_param[i] = list(model_params).index(name)
            o.lambda_[i] = l
    if str(f.get("regularisationType", "TV")).lower() == "prior":
        o.reg_type = _lib.REG_PRIOR
    elif str(f.get("dataType", "volumetric")).lower() == "surface":
        o.reg_type = _lib.REG_SURFACE_TV
    else:
        o.reg_type = _lib.REG_TV
    o.tv_3d = 1 if str(f["TVmode"]).upper() == "3D" else 0
    vs = [float(x) for x in np.atleast_1d(f["voxelSize"])] + [1.0, 1.0, 1.0]
    for i in range(3):
        o.voxel_size[i] = vs[i]
    o.path = _lib.PATH[path]
    o.chunk = int(f.get("chunk", 0))
    o.block_size = int(f.get("blockSize", 0))
    o.robust_convergence = 1 if f.get("robustConvergence") else 0
    o.outlier_weight = float(f.get("outlierWeight", 0.1))
    o.weight_update_interval = int(f.get("weightUpdateInterval", 5))
    o.outlier_check_window = int(f.get("outlierCheckWindow", 5))
    o.outlier_min_flag_duration = int(f.get("outlierMinFlagDuration", 5))
    o.outlier_voxel_thres = float(f.get("outlierVoxelThres", 0.01))
    o.outlier_pop_thres = float(f.get("outlierPopThres", 0.05))
    o.outlier_init_thres = float(f.get("outlierInitThres", 0.05))
    o.outlier_init_pop_thres = float(f.get("outlierInitPopThres", 0.20))
    return o


class askadam:
    """askAdam solver (utils/askadam.m) on the B200 engine."""

    epsilon = 1e-8

    def __init__(self, context=None, path: str = "fused"):
        self.ctx = context
        self.path = path
        self.last_timing = None

    check_set_default_basic = staticmethod(check_set_default_basic)

    def optimisation(self, data, mask, weights, parameters, fitting, userfuncCell, *varargin,
                     extradata=None):
        """askadam.optimisation (utils/askadam.m:121-365)."""
        model = _model_of(userfuncCell)
        fitting = check_set_default_basic(fitting)
        prior = surface = None
        reg_kind = _regulariser_of(userfuncCell)
        if reg_kind == "prior":
            # userInput = {{model inputs}, {mask, lambda, regmap, mu, sigma}} (NEXI/gpuNEXI.m:411-415)
            _, lam, regmap, mu, sd = varargin[0][1]
            fitting = dict(fitting, regularisationType="prior", regmap=list(np.atleast_1d(regmap)))
            fitting["lambda"] = list(np.atleast_1d(lam))
            prior = (mu, sd)
            varargin = ()
        elif reg_kind == "surface":
            # userInput = {{model inputs}, {mask, neighbours, lambda, regmap, edgeLength}} (NEXI/gpuNEXI.m:430-432)
            _, nbrs, lam, regmap, elen = varargin[0][1]
            fitting = dict(fitting, regularisationType="TV", dataType="surface", regmap=list(np.atleast_1d(regmap)))
            fitting["lambda"] = list(np.atleast_1d(lam))
            surface = (nbrs, elen)
            varargin = ()
        mask = np.asarray(mask)
        d3 = utils.dims3(mask)
        idx = utils.mask_index(mask)
        y = utils.to_GD(data, mask, idx).astype(np.float32)
        nm, nv = y.shape
        model_params = list(fitting.get("modelParams") or model.modelParams)
        np_ = len(model_params)
        gxm = model._gx_model()
        ksz = model.nparam_nmeas()
        if ksz[0] != np_:
            raise GacelleError(GX_EINVAL, f"fitting.modelParams has {np_} entries; the model fits {ksz[0]}")
        if ksz[1] != nm:
            raise GacelleError(GX_EINVAL, f"data has {nm} measurements; the model produces {ksz[1]}")
        lb = np.asarray(fitting["lb"], dtype=np.float64).ravel()[:np_]
        ub = np.asarray(fitting["ub"], dtype=np.float64).ravel()[:np_]
        if lb.size != np_ or ub.size != np_:
            raise GacelleError(GX_EINVAL, "fitting.lb/ub need one entry per model parameter")
        w = None
        if weights is not None and np.size(weights) > 0:
            w = utils.to_GD(weights, mask, idx).astype(np.float32)
        theta0 = None
        if parameters:
            theta0 = np.stack([utils.param_to_GD(parameters[p], mask, idx, nv) for p in model_params]).astype(np.float32)
        ex = dict(extradata or {})
        for a in varargin:
            if isinstance(a, dict):
                ex.update(a)
        b1 = utils.param_to_GD(ex["b1"], mask, idx, nv).astype(np.float32) if "b1" in ex else None
        sig = utils.param_to_GD(ex["sigma"], mask, idx, nv).astype(np.float32) if "sigma" in ex else None
        gidx = idx.astype(np.int32)
        opts = build_opts(fitting, model_params, lb, ub, self.path)
        pr = self._prior_maps(prior, fitting, mask, idx, nv) if prior is not None and opts.n_reg > 0 else None
        sf = self._surface_tables(surface, mask, idx) if surface is not None and opts.n_reg > 0 else None
        res = self._run(gxm, y, w, theta0, b1, sig, gidx, d3, opts, nm, np_, pr, sf)
        return self._to_out(res, model_params, mask, fitting, nm, nv)

    @staticmethod
    def _prior_maps(prior, fitting, mask, idx, nv):
        """mu / SD rows of the regularised parameters at the mask's voxels, and
        the regulariser's loss from the grid points outside the mask, where the
        reference's parameter image is 0 (NEXI/gpuNEXI.m:1296-1303)."""
        mu, sd = prior
        regmap = list(fitting["regmap"])
        lam = [float(x) for x in np.atleast_1d(fitting["lambda"])]
        mus, sds, off = [], [], 0.0
        outside = np.asarray(mask).ravel(order="F") == 0
        for name, l in zip(regmap, lam):
            m = np.asarray(mu[name], dtype=np.float32)
            s = np.asarray(sd[name], dtype=np.float32)
            mus.append(utils.param_to_GD(m, mask, idx, nv))
            sds.append(utils.param_to_GD(s, mask, idx, nv))
            # a scalar broadcasts over the grid; a [1, Nvox] row has no grid
            m, s = (np.full(outside.size, x.ravel()[0], np.float32) if x.size == 1 else x for x in (m, s))
            if m.size == outside.size and s.size == outside.size and outside.any():
                with np.errstate(divide="ignore", invalid="ignore"):
                    z = (np.float32(0) - m.ravel(order="F")[outside]) / s.ravel(order="F")[outside]
                off += l / nv * float(np.sum(np.abs(z[np.isfinite(z)]), dtype=np.float64))
        return np.stack(mus).astype(np.float32), np.stack(sds).astype(np.float32), off

    @staticmethod
    def _surface_tables(surface, mask, idx):
        """Neighbour grid indices and edge lengths, [maxNeighbours][Nvox], of
        the masked vertices from the reference's [1, Nvertex, Nhemi,
        maxNeighbours] arrays of 1-based per-hemisphere vertex indices
        (utils.get_surface_neighbours; NEXI/gpuNEXI.m:1224-1229 makes them
        global with a hemisphere offset)."""
        nbrs, elen = surface
        nbrs = np.asarray(nbrs)
        elen = np.asarray(elen, dtype=np.float32)
        d3 = utils.dims3(mask)
        nvert = d3[1]
        maxnb = nbrs.shape[3] if nbrs.ndim == 4 else 1
        nb = nbrs.reshape((-1, maxnb), order="F").astype(np.int64)
        hemi = np.arange(nb.shape[0]) // (d3[0] * nvert)
        glob = (nb - 1) + (hemi * nvert)[:, None]
        ln = elen.reshape((-1, maxnb), order="F")
        return (np.ascontiguousarray(glob[idx].T, dtype=np.int32), np.ascontiguousarray(ln[idx].T))

    def _run(self, gxm, y, w, theta0, b1, sig, gidx, d3, opts, nm, np_, prior=None, surface=None):
        ctx = self.ctx or _lib.Context.default()
        nv = y.shape[1]
        keep = []

        def fp(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32)
            keep.append(a)
            return a.ctypes.data_as(_lib._fp)

        vol = _lib.GxVolume()
        for i in range(3):
            vol.dims[i] = d3[i]
        vol.nvox = nv
        g = np.ascontiguousarray(gidx, dtype=np.int32)
        keep.append(g)
        vol.grid_index = g.ctypes.data_as(_lib._i32p)
        vol.data = fp(y)
        vol.weights = fp(w)
        vol.theta0 = fp(theta0)
        vol.b1 = fp(b1)
        vol.sigma = fp(sig)
        if prior is not None:
            vol.prior_mu = fp(prior[0])
            vol.prior_sd = fp(prior[1])
            vol.prior_offset = float(prior[2])
        if surface is not None:
            nbt = np.ascontiguousarray(surface[0], dtype=np.int32)
            keep.append(nbt)
            vol.max_neighbours = nbt.shape[0]
            vol.neighbours = nbt.ctypes.data_as(_lib._i32p)
            vol.edge_length = fp(surface[1])
        out = {"final_theta": np.zeros((np_, nv), np.float32), "min_theta": np.zeros((np_, nv), np.float32),
               "final_residual": np.zeros((nm, nv), np.float32), "min_residual": np.zeros((nm, nv), np.float32),
               "final_resloss": np.zeros(nv, np.float32), "min_resloss": np.zeros(nv, np.float32),
               "loss_history": np.zeros(opts.iteration + 1, np.float64)}
        r = _lib.GxAskadamResult()
        for k, a in out.items():
            setattr(r, k, a.ctypes.data_as(_lib._dp if a.dtype == np.float64 else _lib._fp))
        st = _lib.lib().gx_askadam(ctx.ptr, _lib.C.byref(gxm.s), _lib.MEM_HOST, _lib.C.byref(vol), 1,
                                   _lib.C.byref(opts), _lib.C.byref(r))
        self.last_timing = ctx.timing()
        for f in ("final_loss", "final_loss_fidelity", "final_loss_reg", "min_loss", "min_loss_fidelity",
                  "min_loss_reg", "final_niteration", "min_niteration", "stop_reason"):
            out[f] = getattr(r, f)
        try:
            _lib.check(st)
        except _lib.GacelleError as e:
            # a non-finite loss still returns the fit's (partial) result
            if st == _lib.GX_ENUMERIC:
                e.partial = out
            raise
        return out

    @staticmethod
    def _to_out(res, model_params, mask, fitting, nm, nv):
        """Output structure of utils/askadam.m:327-362."""
        out = {"final": {}, "min": {}}
        shape = np.shape(mask)
        for k, p in enumerate(model_params):
            for which in ("final", "min"):
                out[which][p] = utils.reshape_GD2ND(res[f"{which}_theta"][k], mask).reshape(shape, order="F")
        for which in ("final", "min"):
            o = out[which]
            o["loss"] = res[f"{which}_loss"]
            o["loss_fidelity"] = res[f"{which}_loss_fidelity"]
            o["loss_reg"] = res[f"{which}_loss_reg"]
            o["resloss"] = utils.reshape_GD2ND(res[f"{which}_resloss"], mask).reshape(shape, order="F")
            o["residual"] = res[f"{which}_residual"]
            o["Niteration"] = res[f"{which}_niteration"]
        out["final"]["memoryUsage"] = 0.0
        out["final"]["stopReason"] = _lib.STOP_REASONS.get(res["stop_reason"], "none")
        out["lossHistory"] = res["loss_history"]
        return out

    @staticmethod
    def save_askadam_output(output_filename, out):
        """utils/askadam.m:993-1009: save ``out`` to a MAT-file when a file
        name is given."""
        return utils.save_output(output_filename, out)

    # ----- static tools of the reference (utils/askadam.m:1063-1183) -----
    @staticmethod
    def unscale_parameters(parameters, lb, ub, modelParams, parameterTransform="linear"):
        out = dict(parameters)
        for k, p in enumerate(modelParams):
            z = np.asarray(parameters[p], dtype=np.float64)
            if parameterTransform == "sigmoid":
                out[p] = lb[k] + (ub[k] - lb[k]) / (1 + np.exp(-z))
            else:
                out[p] = z * (ub[k] - lb[k]) + lb[k]
        return out

    @staticmethod
    def rescale_parameters(parameters, lb, ub, modelParams, parameterTransform="linear"):
        out = dict(parameters)
        for k, p in enumerate(modelParams):
            t = np.asarray(parameters[p], dtype=np.float64)
            if parameterTransform == "sigmoid":
                eb = 1e-4 * (ub[k] - lb[k])
                n = (np.clip(t, lb[k] + eb, ub[k] - eb) - lb[k]) / (ub[k] - lb[k])
                out[p] = np.log(n / (1 - n))
            else:
                out[p] = (t - lb[k]) / (ub[k] - lb[k])
        return out

    @staticmethod
    def set_boundary(parameters, ub, lb):
        return {p: np.minimum(np.maximum(v, lb[k]), ub[k]) for k, (p, v) in enumerate(parameters.items())}

    @staticmethod
    def update_learn_rate(initialLearnRate, decayRate, epoch):
        return initialLearnRate / (1 + decayRate * (epoch - 1))
