"""MCMC parity on the GPU (C-ABI vs FP64 oracle).

Both sides draw every random number from the same Philox4x32-10 streams
(keyed by voxel, walker, step and repetition), so the FP32 device chains and
the FP64 oracle chains follow the same path until an acceptance test falls
within rounding of its threshold.  Checks:
- sample paths agree for most kept samples (random-stream layout parity);
- posterior mean and std differ from the oracle's by no more than two oracle
  runs with different seeds differ from each other (Monte-Carlo error).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from gacelle_b200 import _lib

from helpers import models

pytestmark = pytest.mark.gpu


def _engine_mcmc(ctx, gxm, y, x0, lb, ub, algorithm="ensemble", iteration=1000, thinning=10, burnin=0.1,
                 repetition=1, nwalker=16, step_size=2.0, start_range=0.001, update="simultaneous",
                 x_step=None, seed=7, posterior=True, weights=None, is_global=None, global_warmup=0, _hook=None):
    nvar, nv = x0.shape
    y = np.ascontiguousarray(y, np.float32)
    x0 = np.ascontiguousarray(x0, np.float32)
    lb = np.ascontiguousarray(lb, np.float64)
    ub = np.ascontiguousarray(ub, np.float64)
    xs = np.ascontiguousarray(x_step if x_step is not None else np.zeros(nvar), np.float64)
    o = _lib.GxMcmcOpts(1 if algorithm == "ensemble" else 0, iteration, thinning, burnin, repetition,
                        nwalker, step_size, start_range, 1 if update == "redblack" else 0,
                        xs.ctypes.data_as(_lib._dp), lb.ctypes.data_as(_lib._dp), ub.ctypes.data_as(_lib._dp),
                        seed, 0)
    ig = None
    if is_global is not None:
        ig = np.ascontiguousarray(is_global, np.int32)
        o.is_global = ig.ctypes.data_as(_lib._i32p)
        o.global_warmup = global_warmup
    ns = oracle.lib().orc_mcmc_nsamples(iteration, burnin, thinning)
    W = nwalker if algorithm == "ensemble" else 1
    vol = _lib.GxVolume()
    vol.dims[0], vol.dims[1], vol.dims[2] = nv, 1, 1
    vol.nvox = nv
    vol.data = y.ctypes.data_as(_lib._fp)
    vol.theta0 = x0.ctypes.data_as(_lib._fp)
    if weights is not None:
        w = np.ascontiguousarray(weights, np.float32)
        vol.weights = w.ctypes.data_as(_lib._fp)
    mean = np.zeros((nvar, nv), np.float32)
    std = np.zeros((nvar, nv), np.float32)
    post = np.zeros((nvar, repetition, ns, W, nv), np.float32) if posterior else None
    r = _lib.GxMcmcResult()
    r.mean = mean.ctypes.data_as(_lib._fp)
    r.std = std.ctypes.data_as(_lib._fp)
    if post is not None:
        r.posterior = post.ctypes.data_as(_lib._fp)
    if _hook is not None:
        _hook(r, o)
    _lib.check(_lib.lib().gx_mcmc(ctx.ptr, C.byref(gxm.s), _lib.MEM_HOST, C.byref(vol), 1, C.byref(o), C.byref(r)))
    return {"mean": mean, "std": std, "posterior": post, "n_accepted": r.n_accepted,
            "n_proposals": r.n_proposals, "ns": r.ns, "n_global_accepted": r.n_global_accepted,
            "n_global_proposals": r.n_global_proposals}


def _r2s_problem(nv, seed, sigma=0.02):
    rng = np.random.default_rng(seed)
    gxm, om = models("r2s")
    th = np.vstack([rng.uniform(0.5, 1.5, nv), rng.uniform(10, 60, nv)])
    s = oracle.forward(om, th)
    y = (s + sigma * rng.standard_normal(s.shape)).astype(np.float32)
    x0 = np.vstack([th, np.full(nv, sigma)]).astype(np.float32)
    lb = [0.0, 0.1, sigma]
    ub = [2.0, 200.0, sigma]
    return gxm, om, y, x0, lb, ub


def _moments_agree(eng, orc, orc_b, nparam):
    """Engine-vs-oracle differences of the posterior mean and std, per voxel,
    must not exceed the Monte-Carlo spread between two oracle runs that differ
    only in seed (the engine shares the first oracle's random streams, so its
    differences come from FP32 rounding and are normally far smaller)."""
    for k in range(nparam):
        for q in ("mean", "std"):
            d2 = np.mean((eng[q][k] - orc[q][k]) ** 2)
            r2 = np.mean((orc_b[q][k] - orc[q][k]) ** 2)
            # ratio of mean squares over the voxels; 2.5 is well above the
            # sampling spread of such a ratio for two equal-variance sets
            assert d2 <= 2.5 * r2 + 1e-20, (k, q, d2, r2)


@pytest.mark.parametrize("algorithm,update", [("ensemble", "simultaneous"), ("ensemble", "redblack"),
                                              ("mh", "simultaneous")])
def test_random_streams_match_oracle(ctx, algorithm, update):
    """Same Philox streams: over the first steps the device and oracle chains
    take the same moves (walker starts, stretch factors, partners, accepts)."""
    gxm, om, y, x0, lb, ub = _r2s_problem(128, 10)
    kw = dict(iteration=12, thinning=1, burnin=0.0, nwalker=16, seed=4, algorithm=algorithm)
    xs = [0.01, 1.0, 0.0]
    eng = _engine_mcmc(ctx, gxm, y, x0, lb, ub, update=update, x_step=xs, **kw)
    orc = oracle.mcmc(om, oracle.Volume(y.astype(np.float64)), x0.astype(np.float64), lb, ub,
                      ensemble_update=update, x_step=np.array(xs), want_posterior=True, **kw)
    assert eng["ns"] == orc["ns"] == 12
    pe, po = eng["posterior"][:2], orc["posterior"][:2]
    same = np.abs(pe - po) <= 1e-4 * np.abs(po) + 1e-7
    assert same.mean() > 0.97, same.mean()
    assert abs(eng["n_accepted"] - orc["n_accepted"]) <= 0.01 * orc["n_proposals"]


@pytest.mark.parametrize("update", ["simultaneous", "redblack"])
def test_gw_matches_oracle(ctx, update):
    gxm, om, y, x0, lb, ub = _r2s_problem(64, 11)
    kw = dict(iteration=1500, thinning=5, burnin=0.3, nwalker=16, seed=99)
    eng = _engine_mcmc(ctx, gxm, y, x0, lb, ub, update=update, **kw)
    orc = oracle.mcmc(om, oracle.Volume(y.astype(np.float64)), x0.astype(np.float64), lb, ub,
                      algorithm="ensemble", ensemble_update=update, want_posterior=True, **kw)
    orc_b = oracle.mcmc(om, oracle.Volume(y.astype(np.float64)), x0.astype(np.float64), lb, ub,
                        algorithm="ensemble", ensemble_update=update, **dict(kw, seed=kw["seed"] + 1))
    assert eng["ns"] == orc["ns"]
    assert eng["n_proposals"] == orc["n_proposals"]
    _moments_agree(eng, orc, orc_b, 2)
    acc_e = eng["n_accepted"] / eng["n_proposals"]
    acc_o = orc["n_accepted"] / orc["n_proposals"]
    assert abs(acc_e - acc_o) < 0.02


def test_mh_matches_oracle(ctx):
    gxm, om, y, x0, lb, ub = _r2s_problem(256, 12)
    xs = [0.01, 1.0, 0.0]
    kw = dict(iteration=4000, thinning=4, burnin=0.25, seed=5)
    eng = _engine_mcmc(ctx, gxm, y, x0, lb, ub, algorithm="mh", x_step=xs, **kw)
    orc = oracle.mcmc(om, oracle.Volume(y.astype(np.float64)), x0.astype(np.float64), lb, ub, algorithm="mh",
                      x_step=np.array(xs), want_posterior=True, **kw)
    orc_b = oracle.mcmc(om, oracle.Volume(y.astype(np.float64)), x0.astype(np.float64), lb, ub, algorithm="mh",
                        x_step=np.array(xs), **dict(kw, seed=kw["seed"] + 1))
    _moments_agree(eng, orc, orc_b, 2)


def test_gw_nexi_moments(ctx):
    rng = np.random.default_rng(13)
    gxm, om = models("nexi")
    nv = 96
    th = np.vstack([rng.uniform(0.3, 0.7, nv), rng.uniform(1.5, 2.5, nv), rng.uniform(0.7, 1.2, nv),
                    rng.uniform(0.02, 0.1, nv)])
    s = oracle.forward(om, th)
    y = (s + 0.02 * rng.standard_normal(s.shape)).astype(np.float32)
    x0 = np.vstack([th, np.full(nv, 0.02)]).astype(np.float32)
    lb = [2.2e-16, 2.2e-16, 2.2e-16, 1 / 250, 0.02]
    ub = [1.0, 3.0, 3.0, 1.0, 0.02]
    kw = dict(iteration=800, thinning=4, burnin=0.25, nwalker=32, seed=3)
    eng = _engine_mcmc(ctx, gxm, y, x0, lb, ub, **kw)
    orc = oracle.mcmc(om, oracle.Volume(y.astype(np.float64)), x0.astype(np.float64), lb, ub, want_posterior=True,
                      **kw)
    orc_b = oracle.mcmc(om, oracle.Volume(y.astype(np.float64)), x0.astype(np.float64), lb, ub,
                        **dict(kw, seed=kw["seed"] + 1))
    _moments_agree(eng, orc, orc_b, 4)


# ------------------------------------------- goodman_weare_wglobal_constant ----
def _shared_r2s_problem(nv, seed, sigma=0.05):
    """Voxels with their own M0 sharing R2* = 35 /s and the noise sigma."""
    rng = np.random.default_rng(seed)
    gxm, om = models("r2s")
    m0 = rng.uniform(0.8, 1.2, nv)
    th = np.vstack([m0, np.full(nv, 35.0)])
    s = oracle.forward(om, th)
    y = (s + sigma * rng.standard_normal(s.shape)).astype(np.float32)
    x0 = np.vstack([m0, np.full(nv, 30.0), np.full(nv, sigma)]).astype(np.float32)
    return gxm, om, y, x0, [0.0, 0.1, 0.02], [2.0, 200.0, 0.12]


@pytest.mark.parametrize("update", ["simultaneous", "redblack"])
def test_gw_global_random_streams_match_oracle(ctx, update):
    """Global-parameter sampler (utils/mcmc.m:385-626): the device and the FP64
    oracle draw the local moves, the global partners, stretch factors and
    accept tests from the same streams, so the first steps coincide (locals
    per voxel and walker, globals per walker), warm-up included."""
    gxm, om, y, x0, lb, ub = _shared_r2s_problem(64, 30)
    kw = dict(iteration=12, thinning=1, burnin=0.0, nwalker=16, seed=8, start_range=0.05)
    eng = _engine_mcmc(ctx, gxm, y, x0, lb, ub, update=update, is_global=[0, 1, 1], global_warmup=3, **kw)
    orc = oracle.mcmc(om, oracle.Volume(y.astype(np.float64)), x0.astype(np.float64), lb, ub,
                      algorithm="ensemble", ensemble_update=update, want_posterior=True,
                      is_global=[0, 1, 1], global_warmup=3, **kw)
    pe, po = eng["posterior"], orc["posterior"]
    same = np.abs(pe - po) <= 1e-4 * np.abs(po) + 1e-7
    assert same.mean() > 0.97, same.mean()
    # a global parameter has one value per walker: the same for every voxel
    assert np.ptp(pe[1], axis=-1).max() == 0 and np.ptp(pe[2], axis=-1).max() == 0
    assert eng["n_global_proposals"] == 16 * (12 + 3)
    assert abs(eng["n_accepted"] - orc["n_accepted"]) <= 0.01 * orc["n_proposals"]


@pytest.mark.parametrize("update", ["simultaneous", "redblack"])
def test_gw_global_posterior_known_answer(ctx, update):
    """Through the C-ABI: four voxels with their own M0 sharing R2* and sigma;
    the posterior mean/std of the shared parameters match quadrature of the
    exact marginal posterior (flat priors on the bounds)."""
    import test_oracle
    om, y = test_oracle._gw_global_problem()
    gxm, _ = models("r2s")
    nv = y.shape[1]
    x0 = np.vstack([np.ones(nv), np.full(nv, 30.0), np.full(nv, 0.05)])
    lb, ub = [0.0, 0.1, 0.02], [2.0, 200.0, 0.12]
    eng = _engine_mcmc(ctx, gxm, y, x0, lb, ub, iteration=8000, thinning=2, burnin=0.2, nwalker=32, seed=5,
                       update=update, start_range=0.05, is_global=[0, 1, 1], global_warmup=20, posterior=False)
    mean, std = test_oracle._global_posterior_grid(y)
    for k, q in ((1, 0), (2, 1)):
        assert np.ptp(eng["mean"][k]) == 0 and np.ptp(eng["std"][k]) == 0
        assert abs(eng["mean"][k][0] - mean[q]) < 0.1 * std[q], (k, eng["mean"][k][0], mean[q], std[q])
        assert eng["std"][k][0] == pytest.approx(std[q], rel=0.06)


def test_gw_global_through_mirror_returns_scalars(ctx):
    """mcmc().optimisation with a scalar start field (the reference's cue for
    a global parameter): the statistics of a global come back as scalars and
    its posterior has a leading dimension of 1."""
    from gacelle_b200 import gpuR2starMapping, mcmc_solver
    gxm, om, y, x0, lb, ub = _shared_r2s_problem(50, 31)
    te = np.arange(2.0, 40.6, 3.5) * 1e-3
    model = gpuR2starMapping(te)
    mask = np.ones((50, 1, 1), dtype=bool)
    data = y.T.reshape(50, 1, 1, 12)
    pars0 = {"M0": x0[0].reshape(50, 1, 1), "R2star": 30.0, "noise": 0.05}
    fit = {"algorithm": "GW", "iteration": 400, "thinning": 2, "burnin": 0.25, "Nwalker": 16,
           "lb": lb, "ub": ub, "modelParams": ["M0", "R2star", "noise"], "metric": ["mean", "std", "median"],
           "startRange": 0.05, "globalWarmup": 5, "seed": 3}
    out = mcmc_solver.mcmc(ctx).optimisation(data, mask, None, pars0, fit, model)
    assert isinstance(out["mean"]["R2star"], float) and isinstance(out["median"]["noise"], float)
    assert out["mean"]["M0"].shape == (50, 1, 1)
    assert out["posterior"]["R2star"].shape[0] == 1 and out["posterior"]["M0"].shape[0] == 50
    assert 25.0 < out["mean"]["R2star"] < 45.0


# --------------------------------------------------------- res2out summaries on the device
def _engine_summaries(ctx, gxm, y, x0, lb, ub, nbin=1001, posterior=True, **kw):
    """_engine_mcmc plus the device's median / iqr / mode."""
    nvar, nv = x0.shape
    out = {}
    arrays = {m: np.zeros((nvar, nv), np.float32) for m in ("median", "iqr", "mode")}

    def hook(r, o):
        for m, a in arrays.items():
            setattr(r, m, a.ctypes.data_as(_lib._fp))
        o.nbin = nbin
    res = _engine_mcmc(ctx, gxm, y, x0, lb, ub, posterior=posterior, _hook=hook, **kw)
    out.update(res)
    out.update(arrays)
    return out


@pytest.mark.parametrize("case", ["gw_even", "gw_odd_redblack", "mh", "unfilled_slots", "beyond_smem"])
def test_posterior_median_iqr_mode_on_device(ctx, case):
    """median / iqr / mode computed on the device from the kept samples equal
    the res2out restatement (utils/mcmc.m:806-862) applied to the returned
    posterior: the sampler's N = W x ns x rep samples per voxel and parameter,
    with an even and an odd count, Metropolis-Hastings (W = 1), slots that no
    step fills (zeros, counted), a pinned parameter (all samples equal) and a
    sample count too large for shared memory (read from HBM each pass)."""
    gxm, om, y, x0, lb, ub = _r2s_problem(48 if case != "beyond_smem" else 6, 20)
    kw = {"gw_even": dict(iteration=600, thinning=2, burnin=0.25, nwalker=16, seed=3),
          "gw_odd_redblack": dict(iteration=601, thinning=4, burnin=0.2, nwalker=15, seed=4, update="redblack"),
          "mh": dict(iteration=3001, thinning=3, burnin=0.1, seed=5, algorithm="mh", x_step=[0.01, 1.0, 0.0]),
          "unfilled_slots": dict(iteration=5, thinning=10, burnin=0.0, nwalker=16, seed=6),
          "beyond_smem": dict(iteration=1000, thinning=1, burnin=0.0, nwalker=64, seed=7)}[case]
    eng = _engine_summaries(ctx, gxm, y, x0, lb, ub, nbin=501, **kw)
    post = eng["posterior"]
    nvar, nv = x0.shape
    if case == "unfilled_slots":
        assert eng["ns"] == 1 and np.all(post == 0)   # numel(1:10:5) = 1 slot, no step fills it
    if case == "beyond_smem":
        assert post.shape[1] * post.shape[2] * post.shape[3] == 64000
    for k in range(nvar):
        samples = post[k].reshape(-1, nv).T
        med, iqr, mode = oracle.res2out_summaries(samples, lb[k], ub[k], nbin=501)
        np.testing.assert_array_equal(eng["median"][k], med, err_msg=f"median {k}")
        np.testing.assert_allclose(eng["iqr"][k], iqr, rtol=1e-6, atol=1e-7, err_msg=f"iqr {k}")
        np.testing.assert_array_equal(eng["mode"][k], mode, err_msg=f"mode {k}")
    # the pinned noise parameter: every sample equal
    if case != "unfilled_slots":
        assert np.all(eng["iqr"][2] == 0) and np.all(eng["median"][2] == np.float32(lb[2]))
    if case in ("mh", "gw_odd_redblack"):
        assert (post.shape[1] * post.shape[2] * post.shape[3]) % 2 == 1


def test_posterior_summaries_without_returning_the_posterior(ctx):
    """The summaries need no posterior output: the same run with and without
    the posterior returned gives identical median / iqr / mode; and the host
    mirror's optimisation() returns them as images."""
    gxm, om, y, x0, lb, ub = _r2s_problem(32, 21)
    kw = dict(iteration=400, thinning=2, burnin=0.2, nwalker=16, seed=9)
    a = _engine_summaries(ctx, gxm, y, x0, lb, ub, posterior=True, **kw)
    b = _engine_summaries(ctx, gxm, y, x0, lb, ub, posterior=False, **kw)
    for m in ("median", "iqr", "mode"):
        np.testing.assert_array_equal(a[m], b[m])
    from gacelle_b200 import gpuR2starMapping, mcmc_solver
    te = np.arange(2.0, 40.6, 3.5) * 1e-3
    mask = np.ones((32, 1, 1), dtype=bool)
    data = y.T.reshape(32, 1, 1, 12)
    pars0 = {"M0": x0[0].reshape(32, 1, 1), "R2star": x0[1].reshape(32, 1, 1), "noise": x0[2].reshape(32, 1, 1)}
    fit = {"algorithm": "GW", "iteration": 400, "thinning": 2, "burnin": 0.2, "Nwalker": 16, "lb": lb, "ub": ub,
           "modelParams": ["M0", "R2star", "noise"], "metric": ["mean", "median", "iqr", "mode"], "seed": 9,
           "returnPosterior": False}
    out = mcmc_solver.mcmc(ctx).optimisation(data, mask, None, pars0, fit, gpuR2starMapping(te))
    assert "posterior" not in out
    np.testing.assert_array_equal(out["median"]["R2star"].ravel(), a["median"][1])
    np.testing.assert_array_equal(out["mode"]["M0"].ravel(), a["mode"][0])
    np.testing.assert_array_equal(out["iqr"]["R2star"].ravel(), a["iqr"][1])
