"""Shared helpers for the parity tests: run the same problem through the
engine's C-ABI and through the FP64 oracle."""
from __future__ import annotations

import numpy as np

import oracle
from gacelle_b200 import _lib, askadam_solver as gx_askadam
from gacelle_b200.models import _GxModelHandle

R2S_BOUNDS = ([0.0, 0.1], [2.0, 200.0])
R1R2S_BOUNDS = ([0.0, 0.1, 0.1], [2.0, 10.0, 200.0])
NEXI_BOUNDS = ([2.220446049250313e-16] * 3 + [1 / 250], [1.0, 3.0, 3.0, 1.0])
NEXI2_BOUNDS = ([2.220446049250313e-16] * 3 + [1 / 250, 2.220446049250313e-16], [1.0, 3.0, 3.0, 1.0, 1.0])


def rel_rmse(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-300))


def models(kind, **kw):
    """(engine model handle, oracle model) for one protocol."""
    if kind == "r2s":
        te = kw.get("te", np.arange(2.0, 40.6, 3.5) * 1e-3)
        return _GxModelHandle(_lib.MODEL_R2S, te=te), oracle.r2s(te)
    if kind == "r1r2s":
        te = kw.get("te", np.linspace(2, 40, 12) * 1e-3)
        fa = kw.get("fa", [5.0, 20.0])
        tr = kw.get("tr", 0.03)
        return _GxModelHandle(_lib.MODEL_R1R2S, te=te, fa_deg=fa, tr=tr), oracle.r1r2s(te, fa, tr)
    if kind in ("nexi", "nexi2"):
        b = kw.get("b", np.tile([1.0, 2.5, 4.0, 6.0, 8.0, 10.0], 4))
        d = kw.get("delta", np.repeat([20.0, 27.0, 35.0, 49.0], 6))
        lmax = 2 if kind == "nexi2" else 0
        nx = kw.get("nx", 14)
        return (_GxModelHandle(_lib.MODEL_NEXI, bval=b, delta=d, lmax=lmax, nx=nx),
                oracle.nexi(b, d, lmax=lmax, nx=nx))
    if kind == "nexi_rice":
        b = kw.get("b", np.tile([1.0, 2.5, 4.0, 6.0, 8.0, 10.0], 4))
        d = kw.get("delta", np.repeat([20.0, 27.0, 35.0, 49.0], 6))
        return (_GxModelHandle(_lib.MODEL_NEXI_RICE, bval=b, delta=d, lmax=0, nx=14),
                oracle.nexi_rice(b, d, nx=14))
    raise ValueError(kind)


def bounds(kind):
    return {"r2s": R2S_BOUNDS, "r1r2s": R1R2S_BOUNDS, "nexi": NEXI_BOUNDS, "nexi2": NEXI2_BOUNDS,
            "nexi_rice": NEXI_BOUNDS}[kind]


def random_theta(kind, n, rng):
    if kind == "r2s":
        return np.vstack([rng.uniform(0.5, 1.5, n), rng.uniform(10, 60, n)])
    if kind == "r1r2s":
        return np.vstack([rng.uniform(0.5, 2, n), rng.uniform(0.4, 1.5, n), rng.uniform(10, 60, n)])
    th = np.vstack([rng.uniform(0.1, 0.9, n), rng.uniform(1, 3, n), rng.uniform(0.5, 1.5, n),
                    rng.uniform(0.01, 0.3, n)])
    if kind == "nexi2":
        th = np.vstack([th, rng.uniform(0.05, 0.5, n)])
    return th


def fitting(**over):
    f = gx_askadam.check_set_default_basic(dict({
        "iteration": 200, "initialLearnRate": 0.01, "lossFunction": "mse", "tol": 0.0,
        "convergenceValue": 1e-6, "patienceConvergence": float("inf"), "convergenceStepTol": 0.0,
        "convergenceGradTol": 0.0}, **over))
    return f


def _oracle_opts(kind, f):
    lb, ub = bounds(kind)
    o = oracle.adam_opts(lb, ub, f)
    return o


def reg_fields(f, names):
    """Fill the oracle's regmap indices from a fitting dict."""
    lam = [float(x) for x in np.atleast_1d(f["lambda"])]
    reg = f.get("regmap") or []
    if isinstance(reg, str):
        reg = [reg]
    if lam and lam[0] > 0:
        f["_reg_index"] = [names.index(r) for r in reg[:len(lam)]]
        f["_reg_lambda"] = lam
    return f


def run_engine(kind, y, theta0, f, names, path="fused", dims=None, gidx=None, b1=None, sigma=None,
               weights=None, context=None, prior=None, surface=None, **model_kw):
    gxm, _ = models(kind, **model_kw)
    lb, ub = bounds(kind)
    opts = gx_askadam.build_opts(f, names, lb, ub, path)
    y = np.ascontiguousarray(y, np.float32)
    nm, nv = y.shape
    d3 = dims if dims is not None else (nv, 1, 1)
    g = gidx if gidx is not None else np.arange(nv, dtype=np.int32)
    solver = gx_askadam.askadam(context, path)
    res = solver._run(gxm, y, weights, theta0, b1, sigma, g, d3, opts, nm, len(names), prior, surface)
    res["timing"] = solver.last_timing
    return res


def run_oracle(kind, y, theta0, f, names, dims=None, gidx=None, b1=None, sigma=None, weights=None,
               norm_nvox=0.0, prior=None, surface=None, **model_kw):
    """prior: (mu [n_reg][nvox], sd [n_reg][nvox], offset) of the prior regulariser;
    surface: (neighbours, edge lengths), [maxNeighbours][nvox], of the surface TV."""
    _, om = models(kind, **model_kw)
    f = reg_fields(dict(f), names)
    o = _oracle_opts(kind, f)
    nv = y.shape[1]
    vol = oracle.Volume(np.asarray(y, np.float64), dims=dims or (nv, 1, 1),
                        grid_index=gidx if gidx is not None else np.arange(nv, dtype=np.int32),
                        weights=None if weights is None else np.asarray(weights, np.float64),
                        theta0=None if theta0 is None else np.asarray(theta0, np.float64),
                        b1=None if b1 is None else np.asarray(b1, np.float64),
                        sigma=None if sigma is None else np.asarray(sigma, np.float64),
                        norm_nvox=norm_nvox,
                        prior_mu=None if prior is None else np.asarray(prior[0], np.float64),
                        prior_sd=None if prior is None else np.asarray(prior[1], np.float64),
                        prior_offset=0.0 if prior is None else float(prior[2]),
                        neighbours=None if surface is None else surface[0],
                        edge_length=None if surface is None else np.asarray(surface[1], np.float64))
    return oracle.askadam(om, vol, o, want_residual=True)


NAMES = {"r2s": ["M0", "R2star"], "r1r2s": ["M0", "R1", "R2star"], "nexi": ["fa", "Da", "De", "ra"],
         "nexi2": ["fa", "Da", "De", "ra", "p2"], "nexi_rice": ["fa", "Da", "De", "ra"]}
