"""Host-side mirrors of GACELLE's built-in model classes whose fits run on the
B200 engine: gpuR2starMapping (R2star/gpuR2starMapping.m),
gpuJointR1R2starMapping (R1R2s/gpuJointR1R2starMapping.m), gpuNEXI
(NEXI/gpuNEXI.m; volumetric and surface data, TV or prior-distribution
regularisation) and gpuNEXIrice (NEXI/gpuNEXIrice.m).

Each class keeps the reference's parameter contract (modelParams, lb, ub,
startPoint, step, index-aligned), ``updateProperty``, ``fit`` and ``FWD``.
``fit`` dispatches to :class:`gacelle_b200.askadam_solver.askadam` or
:class:`gacelle_b200.mcmc_solver.mcmc` exactly where the reference calls
``askadam().optimisation`` / ``mcmc().optimisation``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, utils
from . import dwi as dwi_util
from ._lib import GacelleError, GX_EINVAL, GX_EUNSUPPORTED


def _segmented(fitting, fit, data, mask, extradata=None, pars0=None):
    """fit(data, mask, extradata, pars0) whole, or in fitting.NSegmentUser
    slabs with fitting.segmentOverlap halo slices (segments.fit_segmented)."""
    from . import segments
    nseg = fitting.get("NSegmentUser")
    nseg = int(np.atleast_1d(nseg)[0]) if nseg is not None and np.size(nseg) else 1
    if nseg <= 1:
        return fit(data, mask, extradata, pars0)
    return segments.fit_segmented(fit, data, mask, nseg, int(fitting.get("segmentOverlap") or 0), extradata, pars0)


def _rescale_m0(out, fitting, scale):
    """Undo the data scaling on M0 (R2star/gpuR2starMapping.m:163-177): final
    and min maps for askadam; every metric map and the posterior for mcmc."""
    keys = ["final", "min"] if fitting.get("solver", "askadam") != "mcmc" else \
        list(np.atleast_1d(fitting.get("metric", ["mean", "std"]))) + ["posterior"]
    for k in keys:
        if isinstance(out.get(k), dict) and "M0" in out[k]:
            out[k]["M0"] = out[k]["M0"] * scale


def _float_data(a):
    """float32 / float64 arrays as they are; anything else as float64."""
    a = np.asarray(a)
    return a if a.dtype in (np.float32, np.float64) else a.astype(np.float64)


def _save(fitting, out):
    """The end of every model's estimate(): askadam.save_askadam_output or
    mcmc.save_mcmc_output of fitting.outputFilename (e.g.
    NEXI/gpuNEXI.m:243-249)."""
    utils.save_output(fitting.get("outputFilename"), out)


class _GxModelHandle:
    """A gx_model struct plus the arrays it points into."""

    def __init__(self, kind, te=None, fa_deg=None, tr=0.0, bval=None, delta=None, lmax=0, nx=14):
        self._arrays = []

        def arr(a):
            if a is None:
                return None, 0
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
            self._arrays.append(a)
            return a.ctypes.data_as(_lib._dp), a.size

        te_p, nte = arr(te)
        fa_p, nfa = arr(fa_deg)
        b_p, nb = arr(bval)
        d_p, _ = arr(delta)
        self.s = _lib.GxModel(kind, lmax, nx, nte, te_p, nfa, fa_p, float(tr), nb, b_p, d_p)

    def sizes(self):
        npar = C.c_int32()
        nmeas = C.c_int32()
        _lib.check(_lib.lib().gx_model_sizes(C.byref(self.s), C.byref(npar), C.byref(nmeas)))
        return npar.value, nmeas.value


class _ModelBase:
    modelParams: list
    ub: list
    lb: list
    startPoint: list
    step: list
    epsilon = 1e-8
    seed = 48463

    def __init__(self):
        # per-instance copies of the contract so updateProperty never leaks
        self.modelParams = list(type(self).modelParams)
        self.ub = list(type(self).ub)
        self.lb = list(type(self).lb)
        self.startPoint = list(type(self).startPoint)
        self.step = list(type(self).step)
        self.context = None

    def _strip(self, name):
        if name in self.modelParams:
            i = self.modelParams.index(name)
            for attr in ("modelParams", "lb", "ub", "startPoint", "step"):
                getattr(self, attr).pop(i)

    def updateProperty(self, fitting):
        """Drop 'noise' unless the solver is mcmc (e.g. R2star/gpuR2starMapping.m:78-91)."""
        if str(fitting.get("solver", "askadam")).lower() != "mcmc":
            self._strip("noise")
        return self

    def nparam_nmeas(self):
        return self._gx_model().sizes()

    def _forward(self, theta: np.ndarray, b1=None) -> np.ndarray:
        """theta [np][N] -> signal [nm][N] on the engine (gx_forward)."""
        ctx = self.context or _lib.Context.default()
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        n = theta.shape[1]
        npar, nm = self.nparam_nmeas()
        if theta.shape[0] < npar:
            raise GacelleError(GX_EINVAL, f"FWD needs {npar} parameters")
        theta = np.ascontiguousarray(theta[:npar])
        out = np.zeros((nm, n), np.float32)
        b1p = None
        if b1 is not None:
            b1 = np.ascontiguousarray(b1, dtype=np.float32)
            b1p = b1.ctypes.data
        _lib.check(_lib.lib().gx_forward(ctx.ptr, C.byref(self._gx_model().s), _lib.MEM_HOST,
                                         theta.ctypes.data, b1p, n, out.ctypes.data))
        return out

    def _fwd_struct(self, pars: dict, names, b1=None):
        """FWD on a parameter struct: [1,N] rows -> [nm, N]; N-D maps -> [..., nm]."""
        first = np.asarray(pars[names[0]])
        shape = first.shape
        cols = [np.broadcast_to(np.asarray(pars[p], dtype=np.float64), shape).reshape(-1, order="F") for p in names]
        b1v = None if b1 is None else np.broadcast_to(np.asarray(b1, dtype=np.float64), shape).reshape(-1, order="F")
        s = self._forward(np.stack(cols), b1v)
        if first.ndim <= 2 and (first.ndim < 2 or first.shape[0] == 1):
            return s
        return s.T.reshape(shape + (s.shape[0],), order="F")

    def _solve(self, data, mask, w, pars0, fitting, extradata=None):
        from .askadam_solver import askadam
        from .mcmc_solver import mcmc
        if fitting["solver"] == "askadam":
            return askadam(self.context, fitting.get("path", "fused")).optimisation(
                data, mask, w, pars0, fitting, self, extradata=extradata)
        fitting = dict(fitting)
        fitting["xStepSize"] = list(self.step)
        return mcmc(self.context).optimisation(data, mask, w, pars0, fitting, self, extradata=extradata)


class gpuR2starMapping(_ModelBase):
    """Mono-exponential R2* mapping (R2star/gpuR2starMapping.m)."""

    modelParams = ["M0", "R2star", "noise"]
    ub = [2, 200, 0.1]
    lb = [0, 0.1, 0.001]
    startPoint = [1, 30, 0.05]
    step = [0.01, 1, 0.005]

    def __init__(self, te):
        super().__init__()
        self.te = np.asarray(te, dtype=np.float64).ravel()

    def _gx_model(self):
        return _GxModelHandle(_lib.MODEL_R2S, te=self.te)

    def FWD(self, pars, solver=None, fitting=None):
        """R2star/gpuR2starMapping.m:321-363."""
        return self._fwd_struct(pars, ["M0", "R2star"])

    @staticmethod
    def check_set_default(fitting):
        """R2star/gpuR2starMapping.m:463-486."""
        from .askadam_solver import check_set_default_basic as adam_def
        from .mcmc_solver import check_set_default_basic as mcmc_def
        f = dict(fitting or {})
        f.setdefault("solver", "askadam")
        g = mcmc_def(f) if f["solver"].lower() == "mcmc" else adam_def(f)
        g.setdefault("weightMethod", "1stecho")
        g.setdefault("isWeighted", False)
        g.setdefault("weightPower", 2)
        g.setdefault("start", "prior")
        return g

    @staticmethod
    def compute_optimisation_weights(data, fitting):
        """R2star/gpuR2starMapping.m:507-530."""
        data = np.abs(np.asarray(data, dtype=np.float64))
        if fitting["isWeighted"]:
            if fitting["weightMethod"].lower() == "norm":
                w = np.sqrt(data)
            else:
                p = fitting["weightPower"]
                w = data ** p / data[..., :1] ** p
        else:
            w = np.ones_like(data)
        return np.clip(w, 0, 1)

    @staticmethod
    def R2star_trapezoidal(img, te):
        """Closed-form R2* start (R2star/gpuR2starMapping.m:436-459)."""
        img = np.abs(np.asarray(img, dtype=np.float64))
        te = np.asarray(te, dtype=np.float64)
        temp = 0.0
        for k in range(img.shape[-1] - 1):
            temp = temp + 0.5 * (img[..., k] + img[..., k + 1]) * (te[k + 1] - te[k])
        with np.errstate(divide="ignore", invalid="ignore"):
            t2s = temp / (img[..., 0] - img[..., -1])
            return 1.0 / t2s

    def determine_x0(self, y, mask, fitting):
        """R2star/gpuR2starMapping.m:257-290."""
        d3 = utils.dims3(mask)
        start = fitting["start"]
        if isinstance(start, str):
            if start.lower() == "prior":
                x0 = self.estimate_prior(y)
            else:
                x0 = utils.initialise_x0(d3, self.modelParams, self.startPoint)
        else:
            x0 = utils.initialise_x0(d3, self.modelParams, np.ravel(start))
        return {p: np.clip(v, fitting["lb"][k], fitting["ub"][k]) for k, (p, v) in enumerate(x0.items())}

    def estimate_prior(self, data):
        """R2star/gpuR2starMapping.m:293-316 (invalid R2* voxels are set to the
        R2star lower bound)."""
        data = np.asarray(data)
        if data.ndim < 4:
            data = data.reshape(data.shape + (1,) * (4 - data.ndim)) if data.ndim != 2 else data.T[:, None, None, :]
        r2 = self.R2star_trapezoidal(data, self.te)
        bad = ~np.isfinite(r2) | (r2 < self.lb[1])
        r2 = np.where(bad, self.lb[1], np.minimum(r2, self.ub[1]))
        return {"M0": np.abs(data[..., 0]).astype(np.float32), "R2star": r2.astype(np.float32)}

    def prepare_data(self, img, mask):
        """98th-percentile scaling of the first echo (R2star/gpuR2starMapping.m:398-414)."""
        mask = np.asarray(mask) > 0
        tmp = np.abs(np.asarray(img)[..., 0])
        scale = float(np.percentile(tmp[mask], 98, method="hazen"))
        img = np.asarray(img) / scale
        img, bad = utils.set_nan_inf_zero(img)
        mask = mask & ~np.any(bad.reshape(mask.shape + (-1,)), axis=-1)
        return img, mask, scale

    def fit(self, data, mask=None, fitting=None):
        """R2star/gpuR2starMapping.m:182-252."""
        data = np.asarray(data)
        if mask is None:
            mask = np.ones(utils.dims3(data), dtype=bool)
        fitting = self.check_set_default(fitting)
        self.updateProperty(fitting)
        fitting["modelParams"] = list(self.modelParams)
        if not len(fitting["ub"]):
            fitting["ub"] = self.ub[: len(self.modelParams)]
        if not len(fitting["lb"]):
            fitting["lb"] = self.lb[: len(self.modelParams)]
        pars0 = self.determine_x0(data, mask, fitting)
        w = self.compute_optimisation_weights(data, fitting)
        w = None if np.all(w == 1) else w
        return self._solve(data, mask, w, pars0, fitting)

    def estimate(self, data, mask, fitting=None):
        """R2star/gpuR2starMapping.m:94-179: scaled data, fit (in
        fitting.NSegmentUser slabs with segmentOverlap halo slices when asked;
        the engine needs no memory-driven split), M0 scaled back."""
        fitting = self.check_set_default(fitting)
        data, mask, scale = self.prepare_data(data, mask)
        out = _segmented(fitting, lambda d, m, e, p: self.fit(d.astype(np.float32), m, fitting), data, mask)
        out["mask"] = mask
        _rescale_m0(out, fitting, scale)
        _save(fitting, out)
        return out


class despot1:
    """DESPOT1 T1 / M0 from variable-flip-angle spoiled GRE
    (MCRMWI/private/despot1.m:28-160, the 'regression' solver used by the
    joint R1-R2* model).  Per voxel, with a = b1 FA: S / sin(a) = E1 S / tan(a)
    + M0 (1 - E1), E1 = exp(-TR/T1); the two coefficients are the least-squares
    solution over the flip angles, T1 = -TR / log(E1), M0 = b / (1 - E1)
    (real parts, as the reference takes them when E1 <= 0)."""

    def __init__(self, tr, fa):
        self.tr = float(tr)
        self.fa = np.asarray(fa, dtype=np.float64).ravel()

    def fit(self, S, b1=1.0):
        """One or many voxels: S [..., nFA] -> (m0, t1), FP64."""
        S = np.asarray(S, dtype=np.float64)
        if S.shape[-1] < 2:
            raise GacelleError(GX_EINVAL, "DESPOT1: only one point to fit")
        if S.shape[-1] != self.fa.size:
            raise GacelleError(GX_EINVAL, "DESPOT1: size of signal is not equal to size of flip angle")
        a = np.deg2rad(self.fa * np.asarray(b1, dtype=np.float64)[..., None])
        y = S / np.sin(a)
        x = S / np.tan(a)
        # normal equations of [x 1] [E1 b]' = y, solved in closed form
        n = S.shape[-1]
        sx, sy = x.sum(-1), y.sum(-1)
        sxx, sxy = (x * x).sum(-1), (x * y).sum(-1)
        det = n * sxx - sx * sx
        with np.errstate(divide="ignore", invalid="ignore"):
            e1 = (n * sxy - sx * sy) / det
            bb = (sxx * sy - sx * sxy) / det
            t1 = -self.tr / np.log(e1.astype(np.complex128))
            m0 = bb / (1 - np.exp(-self.tr / t1))
        return np.real(m0), np.real(t1)

    def estimate(self, img, mask=None, b1=None):
        """img [x,y,z,nFA] -> (t1, m0, mask_fitted): voxels whose signals sum
        to zero get 0; physically infeasible fits (T1 <= 0, M0 < 0, non-finite)
        are zeroed and left out of mask_fitted."""
        img = np.abs(np.asarray(img, dtype=np.float64))
        d3 = img.shape[:3]
        mask = np.ones(d3, dtype=bool) if mask is None else np.asarray(mask).reshape(d3) > 0
        b1 = np.ones(d3) if b1 is None else np.asarray(b1, dtype=np.float64).reshape(d3)
        t1 = np.zeros(d3)
        m0 = np.zeros(d3)
        sel = mask & (img.sum(-1) != 0)
        m0[sel], t1[sel] = self.fit(img[sel], b1[sel])
        ok = (t1 > 0) & np.isfinite(t1) & (m0 >= 0) & np.isfinite(m0) & mask
        return np.where(ok, t1, 0.0), np.where(ok, m0, 0.0), ok


class gpuJointR1R2starMapping(_ModelBase):
    """Joint R1-R2* mapping from vFA multi-echo GRE (R1R2s/gpuJointR1R2starMapping.m)."""

    modelParams = ["M0", "R1", "R2star", "noise"]
    ub = [2, 10, 200, 0.1]
    lb = [0, 0.1, 0.1, 0.001]
    startPoint = [1, 1, 30, 0.05]
    step = [0.01, 0.01, 1, 0.005]

    def __init__(self, te, tr, fa):
        super().__init__()
        self.te = np.asarray(te, dtype=np.float64).ravel()
        self.tr = float(tr)
        self.fa = np.asarray(fa, dtype=np.float64).ravel()

    def _gx_model(self):
        return _GxModelHandle(_lib.MODEL_R1R2S, te=self.te, fa_deg=self.fa, tr=self.tr)

    def _with_b1(self, extraData):
        """extraData with ``b1`` for the engine.  The reference takes the
        flip angles as extraData.trueFlipAngle [..., 1, Nfa] in radians when
        given, else b1 x the nominal angles (R1R2s/gpuJointR1R2starMapping.m:
        387-391).  The engine scales the nominal angles by one b1 per voxel,
        so trueFlipAngle becomes b1 = trueFlipAngle / nominal when that ratio
        is the same for every flip angle (to 1e-6); otherwise it is rejected."""
        if extraData is None or "trueFlipAngle" not in extraData:
            return extraData
        tfa = np.asarray(extraData["trueFlipAngle"], dtype=np.float64)
        nfa = self.fa.size
        if tfa.shape[-1] != nfa:
            raise GacelleError(GX_EINVAL, f"extraData.trueFlipAngle needs {nfa} flip angles along its last axis")
        ratio = tfa / np.deg2rad(self.fa)
        b1 = ratio[..., :1]
        if np.any(np.abs(ratio - b1) > 1e-6 * np.maximum(np.abs(b1), 1e-30)):
            raise GacelleError(GX_EUNSUPPORTED, "extraData.trueFlipAngle with a flip-angle-dependent scale: the "
                                                "engine takes one b1 per voxel")
        b1 = b1[..., 0]
        while b1.ndim > 3 and b1.shape[-1] == 1:   # the singleton TE axis of [x,y,z,1,Nfa]
            b1 = b1[..., 0]
        ex = dict(extraData)
        del ex["trueFlipAngle"]
        ex["b1"] = b1
        return ex

    def FWD(self, pars, extraData=None, solver=None, fitting=None):
        """R1R2s/gpuJointR1R2starMapping.m:375-422 (measurements TE fastest, then FA)."""
        b1 = None
        extraData = self._with_b1(extraData)
        if extraData is not None and "b1" in extraData:
            b1 = extraData["b1"]
        return self._fwd_struct(pars, ["M0", "R1", "R2star"], b1)

    @staticmethod
    def check_set_default(fitting):
        from .askadam_solver import check_set_default_basic as adam_def
        from .mcmc_solver import check_set_default_basic as mcmc_def
        f = dict(fitting or {})
        f.setdefault("solver", "askadam")
        g = mcmc_def(f) if f["solver"].lower() == "mcmc" else adam_def(f)
        g.setdefault("isWeighted", False)
        g.setdefault("start", "default")
        return g

    def fit(self, data, mask=None, fitting=None, extraData=None):
        """R1R2s/gpuJointR1R2starMapping.m:196-288.  data [x,y,z,TE,FA]."""
        data = np.asarray(data)
        if mask is None:
            mask = np.ones(utils.dims3(data), dtype=bool)
        extraData = self._with_b1(extraData)
        fitting = self.check_set_default(fitting)
        self.updateProperty(fitting)
        fitting["modelParams"] = list(self.modelParams)
        if not len(fitting["ub"]):
            fitting["ub"] = self.ub[: len(self.modelParams)]
        if not len(fitting["lb"]):
            fitting["lb"] = self.lb[: len(self.modelParams)]
        d3 = utils.dims3(mask)
        if isinstance(fitting["start"], str) and fitting["start"].lower() == "prior":
            pars0 = self.estimate_prior(data, mask, extraData)
        else:  # numeric starts are ignored, as determine_x0 does (R1R2s/...:315-317)
            pars0 = utils.initialise_x0(d3, self.modelParams, self.startPoint)
        pars0 = {p: np.clip(v, fitting["lb"][k], fitting["ub"][k]).astype(np.float32)
                 for k, (p, v) in enumerate(pars0.items())}
        if data.ndim == 5:  # [x,y,z,TE,FA] -> [x,y,z,TE*FA] with TE fastest
            data = data.reshape(data.shape[:3] + (-1,), order="F")
        return self._solve(data, mask, None, pars0, fitting, extradata=extraData)

    def _b1(self, extraData, d3):
        extraData = self._with_b1(extraData)
        if extraData is not None and "b1" in extraData and extraData["b1"] is not None:
            return np.asarray(extraData["b1"], dtype=np.float64).reshape(d3)
        return np.ones(d3)

    def estimate_prior(self, data, mask, extraData=None):
        """R1R2s/gpuJointR1R2starMapping.m:327-368: R2* from the trapezoid
        closed form on the flip-angle mean, T1 and M0 from DESPOT1 on the first
        echo, each clamped to the bounds (non-finite values to the lower
        bound), and R2* set to R1/2 where it falls below R1."""
        data = np.asarray(data, dtype=np.float64)
        d3 = utils.dims3(mask)
        data = data.reshape(d3 + (self.te.size, self.fa.size), order="F")
        lb, ub = self.lb, self.ub

        def clamp(v, k):
            v = np.where(np.isfinite(v), v, lb[k])
            return np.minimum(np.maximum(v, lb[k]), ub[k])

        r2 = clamp(gpuR2starMapping.R2star_trapezoidal(np.abs(data).mean(axis=4), self.te), 2)
        t1, m0, _ = despot1(self.tr, self.fa).estimate(np.abs(data[:, :, :, 0, :]), mask, self._b1(extraData, d3))
        with np.errstate(divide="ignore"):
            r1 = 1.0 / t1
        m0, r1 = clamp(m0, 0), clamp(r1, 1)
        r2 = np.where(r1 > r2, r1 / 2, r2)
        pars0 = utils.initialise_x0(d3, self.modelParams, self.startPoint)  # noise keeps its start point
        pars0.update({"M0": m0.astype(np.float32), "R1": r1.astype(np.float32), "R2star": r2.astype(np.float32)})
        return pars0

    def prepare_data(self, img, mask, extraData=None):
        """R1R2s/gpuJointR1R2starMapping.m:474-492: the data divided by the
        98th percentile of the DESPOT1 M0 over the fitted voxels (first echo),
        then non-finite values zeroed and left out of the mask."""
        img = np.asarray(img, dtype=np.float64)
        mask = np.asarray(mask) > 0
        d3 = utils.dims3(mask)
        img5 = img.reshape(d3 + (self.te.size, self.fa.size), order="F")
        _, m0, ok = despot1(self.tr, self.fa).estimate(np.abs(img5[:, :, :, 0, :]), mask, self._b1(extraData, d3))
        scale = float(np.percentile(m0[ok], 98, method="hazen"))
        img = img / scale
        img, bad = utils.set_nan_inf_zero(img)
        mask = mask & ~np.any(bad.reshape(d3 + (-1,), order="F"), axis=-1)
        return img, mask, scale

    def estimate(self, data, mask, fitting=None, extraData=None):
        """R1R2s/gpuJointR1R2starMapping.m:120-194: scaled data, fit (in
        fitting.NSegmentUser slabs when asked, extraData cut with them), M0
        scaled back."""
        fitting = self.check_set_default(fitting)
        data, mask, scale = self.prepare_data(data, mask, extraData)
        out = _segmented(fitting, lambda d, m, e, p: self.fit(d.astype(np.float32), m, fitting, e), data, mask,
                         extraData)
        out["mask"] = mask
        _rescale_m0(out, fitting, scale)
        _save(fitting, out)
        return out


class gpuNEXI(_ModelBase):
    """Neurite exchange imaging, narrow-pulse Karger model (NEXI/gpuNEXI.m)."""

    modelParams = ["fa", "Da", "De", "ra", "p2", "noise"]
    ub = [1, 3, 3, 1, 1, 0.1]
    lb = [np.finfo(float).eps, np.finfo(float).eps, np.finfo(float).eps, 1 / 250, np.finfo(float).eps, 0.01]
    startPoint = [0.4, 2, 1, 0.05, 0.2, 0.005]
    step = [0.05, 0.15, 0.15, 0.005, 0.05, 0.005]

    def __init__(self, b, Delta, Nav=None, nx=14):
        """Shells sorted by DWIutility.unique_shell_keepb0 (NEXI/gpuNEXI.m:70-104):
        b = 0 discarded; unique Delta ascending, then unique b ascending.
        ``nx`` is the powder-average trapezoid size (14 in the reference)."""
        super().__init__()
        bs, _, ds, _ = dwi_util.DWIutility.unique_shell_keepb0(b, None, Delta, None, True)
        self.b = np.array(bs, dtype=np.float32).astype(np.float64)
        self.Delta = np.array(ds, dtype=np.float32).astype(np.float64)
        self.Nav = np.ones(len(self.b)) if Nav is None else np.asarray(Nav, dtype=np.float64).ravel()
        self.nx = int(nx)
        self.lmax = 0

    def _gx_model(self):
        return _GxModelHandle(_lib.MODEL_NEXI, bval=self.b, delta=self.Delta, lmax=self.lmax, nx=self.nx)

    def updateProperty(self, fitting):
        """NEXI/gpuNEXI.m:107-133."""
        super().updateProperty(fitting)
        if int(fitting.get("lmax", 0)) == 0:
            self._strip("p2")
        self.lmax = int(fitting.get("lmax", 0))
        return self

    def FWD(self, pars, lmax=0, solver=None):
        """NEXI/gpuNEXI.m:902-930."""
        self.lmax = int(lmax)
        names = ["fa", "Da", "De", "ra"] + (["p2"] if self.lmax == 2 else [])
        return self._fwd_struct(pars, names)

    @staticmethod
    def check_set_default(fitting):
        """NEXI/gpuNEXI.m:1101-1162."""
        from .askadam_solver import check_set_default_basic as adam_def
        from .mcmc_solver import check_set_default_basic as mcmc_def
        f = dict(fitting or {})
        f.setdefault("solver", "askadam")
        if f["solver"].lower() == "mcmc":
            g = mcmc_def(f)
            g["lossFunction"] = "l2"
        else:
            g = adam_def(f)
            g.setdefault("regmap", "fa")
            if "regmap" not in f:
                g["regmap"] = "fa"
            if not isinstance(g["regmap"], (list, tuple)):
                g["regmap"] = [g["regmap"]]
            g.setdefault("regularisationType", "TV")
            if g["regularisationType"].lower() not in ("tv", "prior"):
                raise GacelleError(GX_EINVAL, "GACELLE:invalidRegularisationType")
        g.setdefault("lmax", 0)
        g.setdefault("start", "likelihood")
        g.setdefault("dataType", "volumetric")
        return g

    # ---------------------------------------------- likelihood starting points
    TRAIN_INTERVALS = [[0.01, 0.99], [1.5, 3.0], [0.5, 1.5], [1.0, 100.0], [0.01, 0.99]]

    def traindata(self, N_samples=10000, lmax=0, intervals=None, seed=None):
        """traindata (NEXI/gpuNEXI.m:762-811): parameters uniform in the
        intervals (fa, Da, De, exchange time, p2; ra = (1 - fa) / time), in
        batches of 1000, and their NEXI signals (Sl0[, Sl2]) on the engine.
        The reference draws from MATLAB's twister seeded with the model seed;
        here the same seed drives NumPy's PCG64."""
        iv = np.asarray(intervals if intervals is not None else self.TRAIN_INTERVALS, dtype=np.float64)
        batch = 1000
        n = int(np.ceil(N_samples / batch)) * batch
        rng = np.random.default_rng(self.seed if seed is None else seed)
        pars = iv[:, :1] + np.diff(iv, axis=1) * rng.random((iv.shape[0], n))
        pars[3] = 1.0 / pars[3] * (1.0 - pars[0])
        if lmax == 0:
            pars = pars[:4]
        handle = _GxModelHandle(_lib.MODEL_NEXI, bval=self.b, delta=self.Delta, lmax=lmax, nx=self.nx)
        S = self._forward_with(handle, pars)
        out_iv = iv.copy()
        out_iv[3] = (1.0 - iv[0, ::-1]) / iv[3, ::-1]
        if lmax == 2:
            out_iv = out_iv[:4]
        return pars, S, out_iv

    def _forward_with(self, handle, theta):
        ctx = self.context or _lib.Context.default()
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        npar, nm = handle.sizes()
        out = np.zeros((nm, theta.shape[1]), np.float32)
        _lib.check(_lib.lib().gx_forward(ctx.ptr, C.byref(handle.s), _lib.MEM_HOST, theta.ctypes.data, None,
                                         theta.shape[1], out.ctypes.data))
        return out

    def likelihood(self, S0, x_train, S_train, lmax=0):
        """likelihood (NEXI/gpuNEXI.m:813-836) on the engine
        (gx_dictionary_match): the best dictionary parameters per voxel."""
        # kron(Nav(:), 1./(2*(0:2:lmax)+1)) flattened column-major: Sl0 weights, then Sl2 weights
        wt = np.concatenate([self.Nav.ravel() / (2 * l + 1) for l in range(0, lmax + 1, 2)])
        nL = lmax // 2
        S0 = np.ascontiguousarray(np.asarray(S0, dtype=np.float32)[: len(self.b) * (nL + 1)])
        D = np.ascontiguousarray(S_train, dtype=np.float32)
        nm, nv = S0.shape
        best = np.zeros(nv, np.int32)
        sse = np.zeros(nv, np.float32)
        w = None if np.all(wt == 1) else np.ascontiguousarray(wt, np.float32)
        ctx = self.context or _lib.Context.default()
        _lib.check(_lib.lib().gx_dictionary_match(ctx.ptr, _lib.MEM_HOST, S0.ctypes.data, nv, D.ctypes.data,
                                                  D.shape[1], nm, None if w is None else w.ctypes.data,
                                                  best.ctypes.data, sse.ctypes.data))
        return np.asarray(x_train)[:, np.maximum(best, 0)], sse

    def estimate_prior(self, dwi, mask, Nsample=None, lmax=0):
        """estimate_prior (NEXI/gpuNEXI.m:675-760): dictionary starting points
        for every voxel of the mask, then the CSF correction (voxels whose
        low-b apparent diffusivity exceeds 1.5 get fa, ra (and p2) scaled by
        0.01)."""
        Nsample = 10000 if Nsample is None else int(Nsample)
        x_train, S_train, _ = self.traindata(Nsample, lmax)
        dwi = np.asarray(dwi, dtype=np.float64)
        dims = utils.dims3(mask)
        flat = dwi.reshape(-1, dwi.shape[-1], order="F").T           # [nmeas, nvox_all]
        ind = np.flatnonzero(np.asarray(mask).reshape(-1, order="F") > 0)
        npar = x_train.shape[0]  # fa, Da, De, ra [, p2 for lmax 2]
        pars = np.zeros((npar, flat.shape[1]))
        if ind.size:
            pb, _ = self.likelihood(flat[:, ind], x_train, S_train, lmax)
            pars[:, ind] = pb[:npar]
        b = self.b
        idx = b <= max(b.min(), 1.1)
        with np.errstate(divide="ignore", invalid="ignore"):
            y = -np.log(flat[: len(b)][idx])
            D0 = (b[idx] @ y) / (b[idx] @ b[idx])
        D0 = np.maximum(np.where(np.isfinite(D0), D0, 0.0), 0.0)
        csf = D0 > 1.5
        scale = [0.01, 1.0, 1.0, 0.01, 0.01]
        for k in range(npar):
            pars[k, csf] *= scale[k]
        return {p: pars[k].reshape(dims, order="F").astype(np.float32)
                for k, p in enumerate(["fa", "Da", "De", "ra", "p2"][:npar])}

    def compute_optimisation_weights(self, mask, lossFunction, lmax):
        """NEXI/gpuNEXI.m:455-477: w = Nav/(2l+1), sqrt for L1, normalised."""
        ls = list(range(0, lmax + 1, 2))
        w = np.concatenate([self.Nav / (2 * l + 1) for l in ls])
        if str(lossFunction).lower() == "l1":
            w = np.sqrt(w)
        return w / w.max()

    thres_similarity = 0.1
    thres_impossible = 0.1
    thres_bkg = 0.01

    def get_surface_geometry(self, surf_dir, depth=0.5, hemisphere=("lh", "rh")):
        """NEXI/gpuNEXI.m:258-287: utils.get_surface_neighbours, cached on the
        object for the last (surf_dir, depth, hemisphere); returns
        (neighbours, edgeLength)."""
        from . import surface
        depth = 0.5 if depth is None else depth
        hemisphere = [hemisphere] if isinstance(hemisphere, str) else list(hemisphere)
        key = (str(surf_dir), float(depth), tuple(hemisphere))
        cache = getattr(self, "_surface_cache", None)
        if cache is not None and cache[0] == key:
            return cache[1], cache[2]
        nb, _, edge = surface.get_surface_neighbours(surf_dir, depth, hemisphere)
        nb = nb.astype(np.float32)
        edge = edge.astype(np.float32)
        self._surface_cache = (key, nb, edge)
        return nb, edge

    def _prepare_surface(self, data, mask, ex, fitting):
        """The surface branch of NEXI/gpuNEXI.m:482-548: [1, Nvertex, Nhemi]
        data and mask; with TV, the mesh geometry from extradata surf_dir /
        hemisphere / depth into extradata neighbours / dr; segmentation only
        as none or one segment per hemisphere."""
        if mask.shape[0] != 1 or data.shape[0] != 1:
            raise GacelleError(GX_EINVAL, "Surface mode expects data/mask in [1, Nvertex, Nhemi] convention "
                                          f"(singleton 1st dimension), got mask size {list(utils.dims3(mask))}.")
        nhemi = utils.dims3(mask)[2]
        if str(fitting.get("regularisationType", "TV")).lower() == "tv" and np.atleast_1d(fitting["lambda"])[0] > 0:
            if not ex.get("surf_dir"):
                raise GacelleError(GX_EINVAL, "fitting.dataType is 'surface' but extradata.surf_dir was not provided.")
            if not ex.get("hemisphere"):
                raise GacelleError(GX_EINVAL, "fitting.dataType is 'surface' but extradata.hemisphere was not "
                                              "provided.")
            hemi = [ex["hemisphere"]] if isinstance(ex["hemisphere"], str) else list(ex["hemisphere"])
            if len(hemi) != nhemi:
                raise GacelleError(GX_EINVAL, f"extradata.hemisphere has {len(hemi)} entries but mask dim3 (Nhemi) "
                                              f"= {nhemi}; these must match.")
            depth = ex.get("depth") if ex.get("depth") is not None else 0.5
            nb, edge = self.get_surface_geometry(ex["surf_dir"], depth, hemi)
            if nb.shape[2] != nhemi:
                raise GacelleError(GX_EINVAL, f"Computed surface neighbour geometry has {nb.shape[2]} hemisphere(s) "
                                              f"but mask has {nhemi}.")
            ex["neighbours"], ex["dr"] = nb, edge
        nseg = fitting.get("NSegmentUser") or 1
        if nseg not in (1, nhemi):
            raise GacelleError(GX_EINVAL, "Surface segmentation is exact-only and limited to fitting.NSegmentUser "
                                          f"= 1 (no split) or {nhemi} (exact per-hemisphere split); got {nseg}.")
        return ex

    def prepare_dwi_data(self, data, mask, extradata, lmax=0, fitting=None):
        """NEXI/gpuNEXI.m:480-633.  Surface data ([1, Nvertex, Nhemi]) get
        their mesh geometry for TV and no mask rules.  A full acquisition
        (more volumes than shells x (lmax/2+1)) becomes rotationally
        invariant signals through
        DWIutility.compute_rotationally_invariant_signal with the little
        delta left empty and one TE.  The mask then loses voxels whose S_0
        exceeds 1 + 0.1 in magnitude on any shell, whose first-shell S_0 is
        below 0.01, whose S_0 decay correlates below 0.1 with the median
        decay of the voxels that passed the two tests (a flat decay counts as
        0), or that hold NaN/Inf (set to 0 in the returned data)."""
        data = _float_data(data)  # single stays single, as in the reference
        mask = np.asarray(mask) > 0
        ex = dict(extradata or {})
        surface = fitting is not None and str(fitting.get("dataType", "volumetric")).lower() == "surface"
        if surface:
            ex = self._prepare_surface(data, mask, ex, fitting)
        nsl = lmax // 2 + 1
        if data.shape[-1] / nsl > len(self.b):
            for k in ("bval", "bvec", "BDELTA"):
                if k not in ex:
                    raise GacelleError(GX_EINVAL, f"full DWI input needs extradata['{k}']")
            data = dwi_util.DWIutility().compute_rotationally_invariant_signal(
                data, ex["bval"], ex["bvec"], None, ex["BDELTA"], None, lmax)[0]
        elif data.shape[-1] < len(self.b) * nsl:
            raise GacelleError(GX_EINVAL, f"Input has {data.shape[-1]} volumes but model expects "
                                          f"{len(self.b) * nsl}. Check lmax or input data.")
        if surface:
            return data, mask, ex
        ns = len(self.b)
        sl0 = data[..., :ns]
        with np.errstate(invalid="ignore"):
            valid = ~np.any(np.abs(sl0) > 1 + self.thres_impossible, axis=-1)
            valid &= ~(sl0[..., 0] < self.thres_bkg)
        idx = utils.mask_index(valid)
        d2 = utils.reshape_ND2GD(sl0, idx)
        incoherent = np.zeros(valid.shape, dtype=bool)
        if d2.shape[1] > 0:
            with np.errstate(invalid="ignore", divide="ignore"):
                tmpl = np.nanmedian(d2, axis=1)
                tsd = np.nanstd(tmpl, ddof=1) if np.sum(np.isfinite(tmpl)) > 1 else 0.0
                tmpl = (tmpl - np.nanmean(tmpl)) / tsd
                sd = d2.std(axis=0, ddof=1) if ns > 1 else np.zeros(d2.shape[1])
                xc = tmpl - tmpl.mean()
                yc = d2 - d2.mean(axis=0)
                r = (xc @ yc) / np.sqrt((xc @ xc) * np.sum(yc * yc, axis=0))
            r = np.where(sd < np.finfo(float).eps, 0.0, r)
            rc = np.zeros(valid.size)
            rc[idx] = r
            incoherent = rc.reshape(valid.shape, order="F") < self.thres_similarity
        valid &= ~incoherent
        data, bad = utils.set_nan_inf_zero(data)
        valid &= mask & ~bad.any(axis=-1)
        return data, valid, ex

    def estimate(self, dwi, mask, extradata=None, fitting=None, pars0=None):
        """NEXI/gpuNEXI.m:148-252: data preparation, then fit (in
        fitting.NSegmentUser slabs / hemispheres when asked, extradata and
        pars0 cut with them)."""
        fitting = self.check_set_default(fitting)
        dwi, mask, ex = self.prepare_dwi_data(dwi, mask, extradata, int(fitting["lmax"]), fitting)
        out = _segmented(fitting, lambda d, m, e, p: self.fit(d.astype(np.float32), m, fitting, p, e), dwi, mask,
                         ex, pars0)
        out["mask"] = mask
        _save(fitting, out)
        return out

    def fit(self, dwi, mask=None, fitting=None, pars0=None, extradata=None):
        """NEXI/gpuNEXI.m:290-450 (volumetric data)."""
        dwi = np.asarray(dwi)
        if mask is None:
            mask = np.ones(utils.dims3(dwi), dtype=bool)
        fitting = self.check_set_default(fitting)
        self.updateProperty(fitting)
        fitting["modelParams"] = list(self.modelParams)
        if not len(fitting["ub"]):
            fitting["ub"] = self.ub[: len(self.modelParams)]
        if not len(fitting["lb"]):
            fitting["lb"] = self.lb[: len(self.modelParams)]
        surface = str(fitting.get("dataType", "volumetric")).lower() == "surface"
        prior = fitting["solver"] == "askadam" and str(fitting.get("regularisationType", "TV")).lower() == "prior" \
            and np.atleast_1d(fitting["lambda"])[0] > 0
        surface_tv = fitting["solver"] == "askadam" and surface and not prior \
            and np.atleast_1d(fitting["lambda"])[0] > 0
        if surface_tv and (not extradata or "neighbours" not in extradata or "dr" not in extradata):
            raise GacelleError(GX_EINVAL, "fitting.dataType is 'surface' and fitting.lambda > 0, but "
                                          "extradata.neighbours/extradata.dr were not provided to fit(). This is "
                                          "normally populated by estimate() - if calling fit() directly, supply "
                                          "extradata.neighbours and extradata.dr yourself.")
        if prior:
            # NEXI/gpuNEXI.m:382-410: mu / sigma structs with a field per regmap name
            ex = extradata or {}
            if not isinstance(ex.get("mu"), dict) or not isinstance(ex.get("sigma"), dict):
                raise GacelleError(GX_EINVAL, "fitting.regularisationType is 'prior' and fitting.lambda > 0, but "
                                              "extradata.mu/extradata.sigma were not provided to fit().")
            miss_mu = [r for r in fitting["regmap"] if r not in ex["mu"]]
            miss_sd = [r for r in fitting["regmap"] if r not in ex["sigma"]]
            if miss_mu or miss_sd:
                raise GacelleError(GX_EINVAL, "extradata.mu/extradata.sigma must have a field for every name in "
                                              f"fitting.regmap. Missing from mu: {{{', '.join(miss_mu)}}}. "
                                              f"Missing from sigma: {{{', '.join(miss_sd)}}}.")
        wv = self.compute_optimisation_weights(mask, fitting["lossFunction"], fitting["lmax"])
        if pars0 is None:
            start = fitting["start"]
            if isinstance(start, str) and start.lower() == "likelihood":
                # determine_x0 (NEXI/gpuNEXI.m:632-662): dictionary starting points
                pars0 = self.estimate_prior(dwi, mask, None, int(fitting["lmax"]))
                if "noise" in self.modelParams:
                    pars0["noise"] = np.full(utils.dims3(mask), self.startPoint[-1], np.float32)
            else:
                pars0 = utils.initialise_x0(utils.dims3(mask), self.modelParams, self.startPoint)
        pars0 = {p: np.clip(np.asarray(pars0[p], dtype=np.float32), fitting["lb"][k], fitting["ub"][k])
                 for k, p in enumerate(self.modelParams)}
        w = None
        if not np.all(wv == 1):
            w = np.broadcast_to(wv, utils.dims3(mask) + (wv.size,)).copy()
        if surface_tv:
            from .askadam_solver import askadam
            userFcn = [self.FWD, self.surface_total_variation]
            userInput = [[fitting["lmax"], fitting["solver"]],
                         [mask, extradata["neighbours"], fitting["lambda"], fitting["regmap"], extradata["dr"]]]
            return askadam(self.context, fitting.get("path", "fused")).optimisation(
                dwi, mask, w, pars0, fitting, userFcn, userInput)
        if prior:
            from .askadam_solver import askadam
            ex = extradata or {}
            userFcn = [self.FWD, self.prior_distribution_normal]
            userInput = [[fitting["lmax"], fitting["solver"]],
                         [mask, fitting["lambda"], fitting["regmap"], ex["mu"], ex["sigma"]]]
            return askadam(self.context, fitting.get("path", "fused")).optimisation(
                dwi, mask, w, pars0, fitting, userFcn, userInput)
        return self._solve(dwi, mask, w, pars0, fitting, extradata=extradata)

    @staticmethod
    def surface_total_variation(parameters, mask, neighbours, lambda_, regmap, edgeLength):
        """gpuNEXI.surface_total_variation (NEXI/gpuNEXI.m:1165-1254): sum_r
        lambda_r / Nmask * sum |theta(v) - theta(nb)| / edgeLength over every
        neighbour slot of every masked vertex, theta being the parameter image
        [1, Nvertex, Nhemi] (0 off the mask) and non-finite quotients dropped.
        As a userFcn entry it selects the engine's surface TV; called directly
        it evaluates the loss of [1, Nvox] parameter rows on the host."""
        lam = [float(x) for x in np.atleast_1d(lambda_)]
        if not lam or lam[0] <= 0:
            return 0.0
        mask = np.asarray(mask)
        d3 = utils.dims3(mask)
        nmask = int(np.count_nonzero(mask))
        nb = np.asarray(neighbours)
        maxnb = nb.shape[3]
        glob = (nb.reshape((-1, maxnb), order="F").astype(np.int64) - 1
                + (np.arange(d3[0] * d3[1] * d3[2]) // (d3[0] * d3[1]) * d3[1])[:, None])
        ln = np.asarray(edgeLength, dtype=np.float32).reshape((-1, maxnb), order="F")
        sel = mask.ravel(order="F") > 0
        loss = 0.0
        for name, l in zip(np.atleast_1d(regmap), lam):
            th = utils.reshape_GD2ND(np.asarray(parameters[name], dtype=np.float32).reshape(1, -1), mask)
            th = np.asarray(th, dtype=np.float32).ravel(order="F")
            with np.errstate(divide="ignore", invalid="ignore"):
                q = (th[:, None] - th[glob]) / ln
            q = q[sel]
            loss += float(np.sum(np.abs(q[np.isfinite(q)]), dtype=np.float64)) / nmask * l
        return loss

    @staticmethod
    def prior_distribution_normal(parameters, mask, lambda_, regmap, mu, sigma):
        """gpuNEXI.prior_distribution_normal (NEXI/gpuNEXI.m:1256-1307): the
        regularisation loss sum_r lambda_r / Nmask * sum |(theta_r - mu_r) /
        sigma_r| over the grid's finite z-scores, theta_r being the parameter
        image (0 outside the mask).  As a userFcn entry it selects the
        engine's prior regulariser; called directly it evaluates the loss of
        [1, Nvox] parameter rows on the host."""
        lam = [float(x) for x in np.atleast_1d(lambda_)]
        if not lam or lam[0] <= 0:
            return 0.0
        mask = np.asarray(mask)
        nmask = int(np.count_nonzero(mask))
        loss = 0.0
        for name, l in zip(np.atleast_1d(regmap), lam):
            th = utils.reshape_GD2ND(np.asarray(parameters[name], dtype=np.float32).reshape(1, -1), mask)
            th = th.reshape(mask.shape, order="F")
            with np.errstate(divide="ignore", invalid="ignore"):
                z = (th - np.asarray(mu[name], dtype=np.float32)) / np.asarray(sigma[name], dtype=np.float32)
            loss += float(np.sum(np.abs(z[np.isfinite(z)]), dtype=np.float64)) / nmask * l
        return loss


class gpuNEXIrice(gpuNEXI):
    """NEXI with the Rician noise floor in the forward model
    (NEXI/gpuNEXIrice.m): the lmax-0 NEXI signal passed through the Rician
    mean for each voxel's noise sigma (normalised by the b0 signal), fitted
    with askAdam."""

    eps = float(np.finfo(float).eps)
    modelParams = ["fa", "Da", "De", "ra", "p2"]
    ub = [1 - eps, 3, 3, 1, 1]
    lb = [eps, eps, eps, 1 / 250, eps]
    startPoint = [0.4, 2, 1, 0.05, 0.2]
    step = [0.05, 0.15, 0.15, 0.005, 0.05]

    def __init__(self, b, Delta, Nav=None, nx=14):
        """NEXI/gpuNEXIrice.m:31-72: b and Delta are kept in the given order."""
        _ModelBase.__init__(self)
        self.b = np.asarray(b, dtype=np.float64).ravel()
        self.Delta = np.asarray(Delta, dtype=np.float64).ravel()
        self.Nav = np.ones(len(self.b)) if Nav is None else np.asarray(Nav, dtype=np.float64).ravel()
        self.nx = int(nx)
        self.lmax = 0

    def _gx_model(self):
        return _GxModelHandle(_lib.MODEL_NEXI_RICE, bval=self.b, delta=self.Delta, lmax=0, nx=self.nx)

    def updateProperty(self, fitting):
        """NEXI/gpuNEXIrice.m:74-84 (no noise parameter)."""
        if int(fitting.get("lmax", 0)) == 0:
            self._strip("p2")
        else:
            raise GacelleError(GX_EUNSUPPORTED, "gpuNEXIrice.FWD computes the lmax-0 signal only")
        return self

    def FWD(self, pars, extraData=None, solver=None):
        """NEXI/gpuNEXIrice.m:635-662; extraData['sigma'] is the noise map."""
        if extraData is None or "sigma" not in extraData:
            raise GacelleError(GX_EINVAL, "gpuNEXIrice.FWD needs extraData['sigma']")
        return self._fwd_struct(pars, ["fa", "Da", "De", "ra"], b1=extraData["sigma"])

    @staticmethod
    def check_set_default(fitting):
        """NEXI/gpuNEXIrice.m:759-772."""
        from .askadam_solver import check_set_default_basic as adam_def
        f = dict(fitting or {})
        g = adam_def(f)
        g["solver"] = "askadam"
        if "regmap" not in f:
            g["regmap"] = "fa"
        if not isinstance(g["regmap"], (list, tuple)):
            g["regmap"] = [g["regmap"]]
        g.setdefault("lmax", 0)
        g.setdefault("start", "likelihood")
        return g

    def prepare_dwi_data(self, dwi, mask, extradata, lmax=0):
        """NEXI/gpuNEXIrice.m:344-405 for rotationally invariant input: sigma
        normalised by the mean b0 signal and floored at epsilon; voxels with
        NaN/Inf, a signal above 1.01, sigma > 1 (SNR < 1) or a signal whose
        correlation with the mean signal shape is below 0.1 leave the mask."""
        dwi = _float_data(dwi)  # single stays single, as in the reference
        mask = np.asarray(mask) > 0
        ex = dict(extradata)
        bval = np.asarray(ex.get("bval", np.ones(dwi.shape[-1])), dtype=np.float64).ravel()
        b0 = bval == 0
        dwi_b0 = np.mean(dwi[..., b0], axis=-1) if b0.any() else np.ones(mask.shape)
        with np.errstate(divide="ignore", invalid="ignore"):
            sigma = np.asarray(ex["sigma"], dtype=np.float64) / dwi_b0
        sigma[~np.isfinite(sigma)] = 0.0
        ex["sigma"] = np.maximum(sigma, self.epsilon)
        if dwi.shape[-1] / (lmax / 2 + 1) > len(self.b):
            # full acquisition: per-(little delta, big delta) invariants, each
            # group normalised by its own b = 0 mean (DWIutility.get_Sl_all)
            for k in ("bval", "bvec", "ldelta", "BDELTA"):
                if k not in ex:
                    raise GacelleError(GX_EINVAL, f"full DWI input needs extradata['{k}']")
            ld = np.asarray(ex["ldelta"], dtype=np.float64).ravel()
            if ld.size == 1:
                ex["ldelta"] = np.full(bval.size, float(ld[0]))
            dwi, _ = dwi_util.DWIutility().get_Sl_all(dwi, bval, ex["bvec"], ex["ldelta"], ex["BDELTA"], lmax)
        elif dwi.shape[-1] < len(self.b):
            raise GacelleError(GX_EINVAL, "There are more b-shells in the class object than available in the "
                                          "input data. Please check your input data.")
        bad = ~np.isfinite(dwi)
        dwi = np.where(bad, 0.0, dwi)
        valid = mask & (dwi.max(axis=-1) <= 1.01) & ~bad.any(axis=-1) & ~(ex["sigma"] > 1)
        idx = utils.mask_index(valid)
        d2 = utils.reshape_ND2GD(dwi, idx)
        if d2.shape[1] > 1:
            tmpl = np.nanmean(d2, axis=1)
            tmpl = (tmpl - tmpl.mean()) / tmpl.std(ddof=1)
            z = (d2 - d2.mean(axis=0)) / d2.std(axis=0, ddof=1)
            r = (tmpl @ z) / (len(tmpl) - 1)
            keep = np.ones(valid.shape, dtype=bool).reshape(-1, order="F")
            keep[idx] = ~(r < 0.1)
            valid &= keep.reshape(valid.shape, order="F")
        return dwi, valid, ex

    def estimate_prior(self, dwi, mask, Nsample=None, sigma=None):
        """estimate_prior (NEXI/gpuNEXIrice.m:449-531): as gpuNEXI's, with the
        dictionary signals passed through the Rician mean at the scalar sigma
        (determine_x0 uses the median of the sigma map in the mask).  The
        engine's forward also applies min(s, 1), which only touches entries
        above 1, a range the data mask excludes."""
        Nsample = 10000 if Nsample is None else int(Nsample)
        x_train, _, _ = self.traindata(Nsample, 0)
        handle = _GxModelHandle(_lib.MODEL_NEXI_RICE, bval=self.b, delta=self.Delta, lmax=0, nx=self.nx)
        ctx = self.context or _lib.Context.default()
        th = np.ascontiguousarray(x_train, dtype=np.float32)
        sig = np.full(th.shape[1], float(sigma), np.float32)
        S_train = np.zeros((len(self.b), th.shape[1]), np.float32)
        _lib.check(_lib.lib().gx_forward(ctx.ptr, C.byref(handle.s), _lib.MEM_HOST, th.ctypes.data,
                                         sig.ctypes.data, th.shape[1], S_train.ctypes.data))
        dims = utils.dims3(mask)
        idx = utils.mask_index(mask)
        y = utils.reshape_ND2GD(np.asarray(dwi, dtype=np.float64), idx)
        pb, _ = self.likelihood(y, x_train, S_train, 0)
        b = self.b
        sel = b <= max(b.min(), 1.1)
        with np.errstate(divide="ignore", invalid="ignore"):
            D0 = (b[sel] @ -np.log(y[: len(b)][sel])) / (b[sel] @ b[sel])
        D0 = np.maximum(np.where(np.isfinite(D0), D0, 0.0), 1e-8)
        csf = D0 > 1.5
        for k, sc in enumerate([0.01, 1.0, 1.0, 0.01]):
            pb[k, csf] *= sc
        return {p: utils.reshape_GD2ND(pb[k].astype(np.float32), mask).reshape(dims, order="F")
                for k, p in enumerate(["fa", "Da", "De", "ra"])}

    def fit(self, dwi, mask=None, fitting=None, extraData=None, pars0=None):
        """NEXI/gpuNEXIrice.m:203-316 (argument order of the reference)."""
        if extraData is None or "sigma" not in extraData:
            raise GacelleError(GX_EINVAL, "gpuNEXIrice.fit needs extraData['sigma']")
        fitting = self.check_set_default(fitting)
        # the reference calls askadam with its FWD alone (NEXI/gpuNEXIrice.m:303):
        # volumetric data and the default spatial TV, whatever else is set
        fitting["regularisationType"] = "TV"
        fitting["dataType"] = "volumetric"
        if mask is None:
            mask = np.ones(utils.dims3(np.asarray(dwi)), dtype=bool)
        start = fitting.get("start")
        if pars0 is None and isinstance(start, str) and start.lower() == "likelihood":
            # determine_x0 (NEXI/gpuNEXIrice.m:410-447): the median sigma in the mask
            sig = np.asarray(extraData["sigma"], dtype=np.float64)
            sigma = float(np.median(np.broadcast_to(sig, utils.dims3(mask))[np.asarray(mask) > 0]))
            pars0 = self.estimate_prior(dwi, mask, None, sigma)
        return gpuNEXI.fit(self, dwi, mask, fitting, pars0, extradata=extraData)

    def estimate(self, dwi, mask, extraData, fitting=None, pars0=None):
        """NEXI/gpuNEXIrice.m:104-199: data preparation, then fit (the engine
        fits the whole volume in one call, no segmentation)."""
        fitting = self.check_set_default(fitting)
        dwi, mask, ex = self.prepare_dwi_data(dwi, mask, extraData, int(fitting["lmax"]))
        out = self.fit(dwi, mask, fitting, ex, pars0)
        out["mask"] = mask
        _save(fitting, out)
        return out
