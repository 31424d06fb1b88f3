"""Parity of the benchmark configurations and of the askAdam branches that
the per-feature tests leave out, on the GPU through the C-ABI, against the
FP64 oracle on the same FP32-rounded inputs.

- The headline workload itself (128x128x64 ellipsoid, 629,432 voxels, 12
  echoes, MSE, lambda 1e-3 3-D TV on R2*, Adam lr 0.01, seed 1002), on the
  exact kernel variant the benchmark times (persistent, voxel pairs,
  measurements as pair quads from L2), for 400 epochs: the fused and the
  op-by-op (plain) paths each within twice the FP32-state band that the FP64
  oracle shows against its own FP32-state twin at this size
  (utils/askadam.m:121-365, utils/spatial_total_variation.m:24-66).
- NEXI lmax 0 with the Rician likelihood loss and a 100-node powder average
  on the 500k-voxel workload: the engine fits all 500k voxels, the oracle a
  voxel subset with the full run's loss normalisation (voxels are
  independent once the normalisation is fixed): 1e-4 relative RMSE.
- Goodman-Weare on NEXI with the 24-shell protocol, 14 nodes, 64 walkers,
  stretch 2 and sigma pinned at 0.02, on a voxel subset of the 200k-voxel
  phantom: same Philox streams (sample paths) and posterior moments within
  the oracle's seed spread (utils/mcmc.m:192-383).
- Weighted losses with gpuNEXI's optimisation weights (NEXI/gpuNEXI.m:455-477;
  L1 is the reference's default loss, utils/askadam.m:785).
- SGDM and RMSProp (utils/askadam.m:680-688), random initialisation
  (randomness > 0, and no start point; utils/askadam.m:368-412).
"""
import numpy as np
import pytest

import oracle
from gacelle_b200 import _lib

from helpers import NAMES, bounds, fitting, models, random_theta, rel_rmse, run_engine, run_oracle

pytestmark = pytest.mark.gpu


# ----------------------------------------------------------------- headline workload
def test_benchmark_workload_fused_and_plain_within_fp32_band(ctx):
    from gacelle_b200 import phantoms
    P = phantoms.r2s_tv_volume(1002, (128, 128, 64))
    y, th0, idx = P["y"], P["th0"], P["idx"]
    assert P["nvox"] == 629432
    kw = dict(dims=P["mask"].shape, gidx=idx)
    f = fitting(iteration=400, initialLearnRate=0.01,
                **{"lambda": [1e-3], "regmap": ["R2star"], "TVmode": "3D", "voxelSize": [2, 2, 2]})
    fused = run_engine("r2s", y, th0, f, NAMES["r2s"], context=ctx, **kw)
    assert fused["timing"]["tv_path"] == _lib.TV_PERSISTENT | _lib.TV_PAIRS | _lib.TV_DATA_QUADS
    plain = run_engine("r2s", y, th0, f, NAMES["r2s"], path="plain", context=ctx, **kw)
    orc = run_oracle("r2s", y, th0, f, NAMES["r2s"], **kw)
    o32 = run_oracle("r2s", y, th0, dict(f, _state_f32=True), NAMES["r2s"], **kw)
    for k in range(2):
        band = rel_rmse(o32["final"][k], orc["final"][k])
        for name, r in (("fused", fused), ("plain", plain)):
            err = rel_rmse(r["final_theta"][k], orc["final"][k])
            assert err <= 2 * band + 1e-5, (name, k, err, band)
    lband = abs(o32["final_loss"] - orc["final_loss"])
    for r in (fused, plain):
        assert abs(r["final_loss"] - orc["final_loss"]) <= 2 * lband + 1e-6 * orc["final_loss"]


# --------------------------------------------------------------------- NEXI Rician, Nx 100
def test_nexi_rician_nx100_workload_matches_oracle_on_a_voxel_subset(ctx):
    import ctypes as C
    nv, nx, sig = 500_000, 100, 0.02
    rng = np.random.default_rng(1004)
    fa = rng.uniform(0.1, 0.9, nv)
    tex = rng.uniform(2.0, 50.0, nv)
    ra = (1 - fa) / tex
    while (ra < 1 / 250).any():
        bad = ra < 1 / 250
        tex[bad] = rng.uniform(2.0, 50.0, bad.sum())
        ra = (1 - fa) / tex
    th = np.ascontiguousarray(np.vstack([fa, rng.uniform(1, 3, nv), rng.uniform(0.5, 1.5, nv), ra]), np.float32)
    gxm, _ = models("nexi", nx=nx)
    S = np.zeros((24, nv), np.float32)
    _lib.check(_lib.lib().gx_forward(ctx.ptr, C.byref(gxm.s), _lib.MEM_HOST, th.ctypes.data, None, nv,
                                     S.ctypes.data))
    y = np.ascontiguousarray(np.sqrt((S + sig * rng.standard_normal(S.shape)) ** 2 +
                                     (sig * rng.standard_normal(S.shape)) ** 2), np.float32)
    lb, ub = bounds("nexi")
    th0 = np.tile(np.array([[0.4], [2.0], [1.0], [0.05]], np.float32), (1, nv))
    # tol -inf: the Rician log-likelihood loss can be negative, and the
    # reference's loss-tolerance stop (loss < tol) would end the fit when the
    # mean over all voxels crosses tol, an epoch a voxel subset cannot reproduce
    f = fitting(iteration=100, initialLearnRate=0.01, lossFunction="rician", noiseSigma=sig, tol=-np.inf)
    eng = run_engine("nexi", y, th0, f, NAMES["nexi"], context=ctx, nx=nx)
    assert eng["final_niteration"] == 100
    rng = np.random.default_rng(4)
    sub = np.sort(rng.choice(nv, 1500, replace=False))
    orc = run_oracle("nexi", y[:, sub], th0[:, sub], f, NAMES["nexi"], norm_nvox=float(nv), nx=nx)
    for k in range(4):
        err = rel_rmse(eng["final_theta"][k, sub], orc["final"][k])
        assert err <= 1e-4, (k, err)
    # the fit moved the parameters: the check is not of the start point
    assert rel_rmse(eng["final_theta"][0, sub], th0[0, sub]) > 0.05


# ------------------------------------------------------------------- Goodman-Weare NEXI
def test_gw_nexi_workload_protocol_on_a_voxel_subset(ctx):
    from test_gpu_mcmc import _engine_mcmc, _moments_agree
    from gacelle_b200 import phantoms
    nv_full, nv, sig = 200_000, 48, 0.02
    y, gt = phantoms.nexi_volume(nv_full, 1005, sigma=sig, rician=False, nx=14)
    y = np.ascontiguousarray(y[:, :nv])
    gxm, om = models("nexi", nx=14)
    x0 = np.vstack([gt["fa"][:nv], gt["Da"][:nv], gt["De"][:nv], gt["ra"][:nv], np.full(nv, sig)])
    lb = list(bounds("nexi")[0]) + [sig]
    ub = list(bounds("nexi")[1]) + [sig]
    ov = oracle.Volume(y.astype(np.float64))
    # sample paths: the first steps take the same moves
    kw = dict(iteration=10, thinning=1, burnin=0.0, nwalker=64, step_size=2.0, seed=1005)
    eng = _engine_mcmc(ctx, gxm, y, x0, lb, ub, **kw)
    orc = oracle.mcmc(om, ov, x0.astype(np.float64), lb, ub, want_posterior=True, **kw)
    pe, po = eng["posterior"][:4], orc["posterior"][:4]
    same = np.abs(pe - po) <= 1e-4 * np.abs(po) + 1e-7
    assert same.mean() > 0.97, same.mean()
    # posterior moments within the Monte-Carlo spread of two oracle seeds
    kw = dict(iteration=500, thinning=10, burnin=0.2, nwalker=64, step_size=2.0, seed=1005)
    eng = _engine_mcmc(ctx, gxm, y, x0, lb, ub, posterior=False, **kw)
    orc = oracle.mcmc(om, ov, x0.astype(np.float64), lb, ub, **kw)
    orc_b = oracle.mcmc(om, ov, x0.astype(np.float64), lb, ub, **dict(kw, seed=kw["seed"] + 1))
    assert eng["n_proposals"] == orc["n_proposals"] == 500 * 64 * nv
    _moments_agree(eng, orc, orc_b, 4)
    # the pinned noise parameter stays pinned
    assert np.all(eng["mean"][4] == np.float32(sig)) and np.all(eng["std"][4] <= 1e-6)


# ------------------------------------------------------------------ weighted losses (NEXI)
def _nexi_weights(loss, n, nav):
    from gacelle_b200.models import gpuNEXI
    b, d = np.tile([1.0, 2.5, 4.0, 6.0, 8.0, 10.0], 4), np.repeat([20.0, 27.0, 35.0, 49.0], 6)
    m = gpuNEXI(b, d, nav)
    w = m.compute_optimisation_weights(None, loss, 0)
    assert w.shape == (24,) and np.ptp(w) > 0
    return np.ascontiguousarray(np.tile(w[:, None], (1, n)), np.float32)


@pytest.mark.parametrize("loss", ["l1", "l2", "huber"])
@pytest.mark.parametrize("path", ["fused", "plain"])
def test_weighted_loss_with_nexi_weights_matches_oracle(ctx, loss, path):
    """gpuNEXI weights w = Nav / (2l + 1), square-rooted for L1, normalised by
    the maximum (per-shell direction counts that differ).  L2 and Huber are
    smooth: 1e-4 relative RMSE.  L1's sign subgradient amplifies single
    roundings: within twice the FP32-state band of the FP64 oracle."""
    rng = np.random.default_rng(40)
    n = 512
    gxm, om = models("nexi")
    th = random_theta("nexi", n, rng)
    s = oracle.forward(om, th)
    y = (s + 0.02 * rng.standard_normal(s.shape)).astype(np.float32)
    nav = rng.integers(6, 64, 24).astype(np.float64)
    w = _nexi_weights(loss, n, nav)
    lb, ub = bounds("nexi")
    th0 = np.tile(((np.array(lb) + np.array(ub)) / 2)[:, None], (1, n)).astype(np.float32)
    f = fitting(iteration=300, initialLearnRate=0.01, lossFunction=loss)
    eng = run_engine("nexi", y, th0, f, NAMES["nexi"], path=path, weights=w, context=ctx)
    orc = run_oracle("nexi", y, th0, f, NAMES["nexi"], weights=w)
    # the weights change the loss gradient (Adam's normalised steps can make
    # the parameters themselves move alike early in the fit)
    o = oracle.adam_opts(*bounds("nexi"), f)
    _, gw, _, _, _ = oracle.model_gradient(om, oracle.Volume(y.astype(np.float64), weights=w.astype(np.float64)),
                                           o, th0.astype(np.float64))
    _, gu, _, _, _ = oracle.model_gradient(om, oracle.Volume(y.astype(np.float64)), o, th0.astype(np.float64))
    assert rel_rmse(gw, gu) > 1e-2
    if loss == "l1":
        # the band of an FP32 run: the FP64 oracle with its state rounded to
        # FP32 each epoch, and with the measurements perturbed at the FP32
        # forward model's relative precision (2e-6; the 14-node trapezoid of
        # fast exponentials is held to 2e-5 by test_forward_matches_oracle):
        # the sign subgradient flips for residuals inside that precision, which
        # the state rounding alone does not provoke
        o32 = run_oracle("nexi", y, th0, dict(f, _state_f32=True), NAMES["nexi"], weights=w)
        yp = (y.astype(np.float64) * (1 + 2e-6 * np.random.default_rng(43).standard_normal(y.shape)))
        opert = run_oracle("nexi", yp, th0, f, NAMES["nexi"], weights=w)
        for k in range(4):
            band = max(rel_rmse(o32["final"][k], orc["final"][k]), rel_rmse(opert["final"][k], orc["final"][k]))
            assert rel_rmse(eng["final_theta"][k], orc["final"][k]) <= 2 * band + 1e-4, (k, band)
        return
    for k in range(4):
        assert rel_rmse(eng["final_theta"][k], orc["final"][k]) <= 1e-4, k
        assert rel_rmse(eng["min_theta"][k], orc["min"][k]) <= 1e-4, k
    assert abs(eng["final_loss"] - orc["final_loss"]) <= 1e-4 * abs(orc["final_loss"])


# --------------------------------------------------------------------------- optimisers
@pytest.mark.parametrize("optimiser", ["sgdm", "rmsprop"])
@pytest.mark.parametrize("kind", ["r2s", "nexi"])
@pytest.mark.parametrize("path", ["fused", "plain"])
def test_sgdm_and_rmsprop_match_oracle(ctx, optimiser, kind, path):
    rng = np.random.default_rng(41)
    n = 512
    gxm, om = models(kind)
    th = random_theta(kind, n, rng)
    s = oracle.forward(om, th)
    y = (s + 0.01 * rng.standard_normal(s.shape)).astype(np.float32)
    lb, ub = bounds(kind)
    th0 = np.tile(((np.array(lb) + np.array(ub)) / 2)[:, None], (1, n)).astype(np.float32)
    if kind == "r2s":
        th0[:] = np.array([[1.0], [30.0]])
    # SGDM steps are lr x gradient (not normalised like Adam's): a rate that moves the fit
    lr = {"sgdm": 50.0 if kind == "r2s" else 20.0, "rmsprop": 0.01}[optimiser]
    f = fitting(iteration=300, initialLearnRate=lr, optimiser=optimiser)
    eng = run_engine(kind, y, th0, f, NAMES[kind], path=path, context=ctx)
    orc = run_oracle(kind, y, th0, f, NAMES[kind])
    adam = run_oracle(kind, y, th0, fitting(iteration=300, initialLearnRate=0.01), NAMES[kind])
    assert rel_rmse(orc["final"][0], adam["final"][0]) > 1e-3  # a different optimiser, a different fit
    assert rel_rmse(orc["final"][0], th0[0]) > 1e-3            # and it moved
    if optimiser == "rmsprop":
        # RMSProp's step lr g / sqrt(E[g^2]) has no momentum: near the optimum it
        # is sign-like and the parameters oscillate with amplitude ~lr, so single
        # roundings shift the phase; the FP32-state twin of the FP64 oracle
        # measures that band, and the engine must stay within twice it
        o32 = run_oracle(kind, y, th0, dict(f, _state_f32=True), NAMES[kind])
        for k in range(len(NAMES[kind])):
            band = rel_rmse(o32["final"][k], orc["final"][k])
            assert rel_rmse(eng["final_theta"][k], orc["final"][k]) <= 2 * band + 1e-4, (k, band)
        return
    for k in range(len(NAMES[kind])):
        assert rel_rmse(eng["final_theta"][k], orc["final"][k]) <= 1e-4, k
        assert rel_rmse(eng["min_theta"][k], orc["min"][k]) <= 1e-4, k
    assert abs(eng["final_loss"] - orc["final_loss"]) <= 1e-4 * abs(orc["final_loss"])


# ------------------------------------------------------------------ random initialisation
@pytest.mark.parametrize("transform", ["sigmoid", "linear"])
@pytest.mark.parametrize("start", ["perturbed", "none"])
def test_random_initialisation_matches_oracle(ctx, transform, start):
    """initialise_parameter with randomness > 0 (Gaussian in z for the sigmoid
    transform, uniform mixing for the linear one) and without a start point
    (z = randomness x N(0,1), or U(0,1) for linear): the device and the oracle
    draw the same Philox numbers, so the fits agree voxel by voxel."""
    rng = np.random.default_rng(42)
    n = 600
    gxm, om = models("r2s")
    th = random_theta("r2s", n, rng)
    s = oracle.forward(om, th)
    y = (s + 0.01 * rng.standard_normal(s.shape)).astype(np.float32)
    th0 = np.tile(np.array([[1.0], [30.0]], np.float32), (1, n)) if start == "perturbed" else None
    f = fitting(iteration=200, initialLearnRate=0.01, randomness=0.3, parameterTransform=transform, seed=77)
    eng = run_engine("r2s", y, th0, f, NAMES["r2s"], context=ctx)
    orc = run_oracle("r2s", y, th0, f, NAMES["r2s"])
    det = run_oracle("r2s", y, np.tile(np.array([[1.0], [30.0]], np.float32), (1, n)),
                     dict(f, randomness=0.0), NAMES["r2s"])
    assert rel_rmse(orc["final"][1], det["final"][1]) > 1e-3  # the random start changes the fit
    band = 1e-4
    if transform == "linear":
        # the clamp at the bounds and the uniform start put some voxels on a kink
        o32 = run_oracle("r2s", y, th0, dict(f, _state_f32=True), NAMES["r2s"])
        band = max(band, 2 * max(rel_rmse(o32["final"][k], orc["final"][k]) for k in range(2)) + 1e-4)
    for k in range(2):
        assert rel_rmse(eng["final_theta"][k], orc["final"][k]) <= band, (k, band)
