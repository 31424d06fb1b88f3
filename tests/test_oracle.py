"""CPU tests that pin the FP64 oracle.

The reference ships no golden vectors (it is MATLAB-only); the oracle is
pinned by published known answers (Philox KAT), scipy's Bessel functions,
the reference's own source-stated quadrature accuracies, an independent
torch float64 restatement of the model formulas (autograd for the
adjoints), central finite differences, and a known-answer posterior.
"""
import math

import numpy as np
import pytest
import scipy.special as sp
import torch

import oracle
from oracle import torch_ref as T

TE = np.arange(2.0, 40.6, 3.5) * 1e-3
B24 = np.tile([1.0, 2.5, 4.0, 6.0, 8.0, 10.0], 4)
D24 = np.repeat([20.0, 27.0, 35.0, 49.0], 6)


# ---------------------------------------------------------------- Philox ----
@pytest.mark.parametrize("ctr,key,out", [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
])
def test_philox4x32_10_known_answers(ctr, key, out):
    """Known-answer vectors of Philox4x32-10 (Salmon et al., SC'11)."""
    assert oracle.philox(ctr, key) == out


def test_uniform_open_interval_exact_in_fp32():
    for x in (0, 1, 511, 512, 2 ** 31, 2 ** 32 - 1):
        u = oracle.u01(x)
        assert 0.0 < u < 1.0
        assert float(np.float32(u)) == u


# ----------------------------------------------------------------- Bessel ---
def test_bessel_scaled_matches_scipy():
    xs = np.concatenate([np.linspace(0, 40, 401), [55.0, 100.0, 700.0, 2500.0, 1e5]])
    for x in xs:
        assert abs(oracle.i0e(x) - sp.i0e(x)) <= 1e-14 * sp.i0e(x)
        assert abs(oracle.i1e(x) - sp.i1e(x)) <= 1e-14 * max(sp.i1e(x), 1e-300) + 1e-300
    assert oracle.i1e(-3.0) == pytest.approx(-sp.i1e(3.0), rel=1e-14)


def test_reference_bessel_integral_accuracy():
    """utils/gacelle_besseli.m:5 states NRMSE < 0.05% for the 34-node integral."""
    z = np.linspace(0.0, 20.0, 201)
    for nu in (0, 1):
        approx = np.array([oracle.besseli_trapz(nu, zz, 34) for zz in z])
        exact = sp.iv(nu, z)
        nrmse = np.sqrt(np.mean((approx - exact) ** 2)) / np.sqrt(np.mean(exact ** 2))
        assert nrmse < 5e-4


# ------------------------------------------------------------------ models --
def _theta(kind, n, rng):
    if kind == "r2s":
        return np.vstack([rng.uniform(0.5, 1.5, n), rng.uniform(10, 60, n)])
    if kind == "r1r2s":
        return np.vstack([rng.uniform(0.5, 2, n), rng.uniform(0.4, 1.5, n), rng.uniform(10, 60, n)])
    th = np.vstack([rng.uniform(0.1, 0.9, n), rng.uniform(1, 3, n), rng.uniform(0.5, 1.5, n),
                    rng.uniform(0.01, 0.3, n)])
    return np.vstack([th, rng.uniform(0.05, 0.5, n)]) if kind == "nexi2" else th


def _models(kind):
    if kind == "r2s":
        return oracle.r2s(TE), lambda t: T.r2s_fwd(t, TE)
    if kind == "r1r2s":
        te = np.linspace(2, 40, 12) * 1e-3
        return oracle.r1r2s(te, [5.0, 20.0], 0.03), lambda t, b1=None: T.r1r2s_fwd(t, te, [5.0, 20.0], 0.03, b1)
    lmax = 2 if kind == "nexi2" else 0
    return oracle.nexi(B24, D24, lmax=lmax, nx=14), lambda t: T.nexi_fwd(t, B24, D24, lmax, 14)


KINDS = ["r2s", "r1r2s", "nexi", "nexi2"]


@pytest.mark.parametrize("kind", KINDS)
def test_forward_matches_independent_restatement(kind):
    rng = np.random.default_rng(0)
    om, tf = _models(kind)
    th = _theta(kind, 64, rng)
    np.testing.assert_allclose(oracle.forward(om, th), tf(torch.tensor(th)).numpy(), rtol=1e-12, atol=1e-14)


def test_r1r2s_b1_scaling():
    rng = np.random.default_rng(1)
    om, tf = _models("r1r2s")
    th = _theta("r1r2s", 16, rng)
    b1 = rng.uniform(0.7, 1.3, 16)
    np.testing.assert_allclose(oracle.forward(om, th, b1), tf(torch.tensor(th), torch.tensor(b1)).numpy(),
                               rtol=1e-12)


@pytest.mark.parametrize("kind", KINDS)
def test_adjoint_matches_autograd(kind):
    rng = np.random.default_rng(2)
    om, tf = _models(kind)
    for _ in range(5):
        th = _theta(kind, 1, rng)
        sb = rng.normal(size=om.nm)
        t = torch.tensor(th, requires_grad=True)
        (tf(t)[:, 0] * torch.tensor(sb)).sum().backward()
        np.testing.assert_allclose(oracle.vjp_voxel(om, th[:, 0], sb), t.grad.numpy()[:, 0], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("kind", KINDS)
def test_adjoint_matches_central_differences(kind):
    rng = np.random.default_rng(3)
    om, _ = _models(kind)
    th = _theta(kind, 1, rng)[:, 0]
    sb = rng.normal(size=om.nm)
    g = oracle.vjp_voxel(om, th, sb)
    for k in range(len(th)):
        h = 1e-6 * max(abs(th[k]), 1e-3)
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        fd = (sb @ oracle.forward(om, tp[:, None])[:, 0] - sb @ oracle.forward(om, tm[:, None])[:, 0]) / (2 * h)
        assert fd == pytest.approx(g[k], rel=1e-5, abs=1e-9)


def test_nexi_trapezoid_accuracy_claims():
    """NEXI/gpuNEXI.m:950,1019,1062: Nx = 14 gives NRMSE < 0.05% (Sl0) and
    < 0.5% (Sl2) against a converged quadrature."""
    rng = np.random.default_rng(4)
    th = _theta("nexi2", 400, rng)
    coarse = oracle.forward(oracle.nexi(B24, D24, lmax=2, nx=14), th)
    fine = oracle.forward(oracle.nexi(B24, D24, lmax=2, nx=4001), th)
    nrmse = lambda a, b: np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2))  # noqa: E731
    assert nrmse(coarse[:24], fine[:24]) < 5e-4
    assert nrmse(coarse[24:], fine[24:]) < 5e-3


def test_nexi_min_one_and_fa_floor():
    om, _ = _models("nexi")
    th = np.array([[0.0], [2.0], [1.0], [0.05]])  # fa below eps: clamped to 1e-8
    s = oracle.forward(om, th)
    assert np.all(np.isfinite(s)) and np.all(s <= 1.0)
    g = oracle.vjp_voxel(om, th[:, 0], np.ones(24))
    assert g[0] == 0.0  # d max(fa, eps) / d fa = 0 below eps


# ------------------------------------------------------------------ losses --
@pytest.mark.parametrize("loss", ["l1", "l2", "huber", "mse", "gauss", "rician"])
def test_loss_derivative_matches_finite_differences(loss):
    rng = np.random.default_rng(5)
    for _ in range(20):
        s, y = rng.uniform(0.05, 1.5, 2)
        w = rng.uniform(0.2, 1)
        h = 1e-6
        fd = (oracle.loss_value(loss, s + h, y, w, 0.05) - oracle.loss_value(loss, s - h, y, w, 0.05)) / (2 * h)
        assert fd == pytest.approx(oracle.loss_deriv(loss, s, y, w, 0.05), rel=1e-5, abs=1e-6)


@pytest.mark.parametrize("loss", ["l1", "l2", "huber", "mse", "gauss", "rician"])
def test_loss_matches_independent_restatement(loss):
    rng = np.random.default_rng(6)
    s = rng.uniform(0.05, 1.5, 50)
    y = rng.uniform(0.05, 1.5, 50)
    w = rng.uniform(0.2, 1, 50)
    ref = T.loss_elem(loss, torch.tensor(s), torch.tensor(y), torch.tensor(w), sigma=0.05).numpy()
    ours = [oracle.loss_value(loss, a, b, c, 0.05) for a, b, c in zip(s, y, w)]
    np.testing.assert_allclose(ours, ref, rtol=1e-10, atol=1e-10)


def test_rician_nll_is_a_density():
    """exp(-NLL) integrates to one over y (the Rician density)."""
    sigma, S = 0.1, 0.3
    y = np.linspace(1e-6, 2.0, 200001)
    dens = np.exp([-oracle.loss_value("rician", S, yy, 1.0, sigma) for yy in y[::100]])
    assert np.trapezoid(dens, y[::100]) == pytest.approx(1.0, rel=1e-3)


# -------------------------------------------------------------------- TV ----
@pytest.mark.parametrize("tv3d", [False, True])
def test_tv_matches_autograd(tv3d):
    rng = np.random.default_rng(7)
    mask = rng.random((7, 6, 5)) > 0.3
    img = rng.normal(size=mask.shape) * mask
    vs = (2.0, 1.5, 3.0)
    t = torch.tensor(img, requires_grad=True)
    c = T.tv_cost(t, torch.tensor(mask, dtype=torch.float64), tv3d, vs)
    c.backward()
    assert oracle.tv_cost(mask, img, tv3d, vs) == pytest.approx(c.item(), rel=1e-13)
    np.testing.assert_allclose(oracle.tv_grad(mask, img, tv3d, vs) * mask, t.grad.numpy() * mask, atol=1e-13)


# ----------------------------------------------------------- askAdam loop ---
def _torch_askadam(y, th0, lb, ub, iters, lr, lam=0.0, mask=None, idx=None, tv3d=True):
    """Independent restatement of the askadam loop (utils/askadam.m:121-325)
    with torch autograd standing in for dlgradient and MATLAB adamupdate."""
    lb = torch.tensor(lb)[:, None]
    ub = torch.tensor(ub)[:, None]
    t0 = torch.tensor(th0)
    eb = 1e-4 * (ub - lb)
    n = (torch.minimum(torch.maximum(t0, lb + eb), ub - eb) - lb) / (ub - lb)
    z = torch.log(n / (1 - n)).clone().requires_grad_(True)
    m = torch.zeros_like(z)
    v = torch.zeros_like(z)
    yt = torch.tensor(y)
    nm, nv = y.shape
    for e in range(1, iters + 1):
        th = lb + (ub - lb) * torch.sigmoid(z)
        s = T.r2s_fwd(th, TE)
        loss = torch.mean(0.5 * (s - yt) ** 2)
        if lam > 0:
            grid = torch.zeros(mask.size, dtype=torch.float64)
            grid = grid.index_put((torch.tensor(idx),), th[1])
            loss = loss + lam * T.tv_cost(grid.reshape(mask.shape[::-1]).permute(2, 1, 0),
                                          torch.tensor(mask, dtype=torch.float64), tv3d) / nv
        g, = torch.autograd.grad(loss, z)
        if e < iters:
            with torch.no_grad():
                m = 0.9 * m + 0.1 * g
                v = 0.999 * v + 0.001 * g * g
                z -= lr * (m / (1 - 0.9 ** e)) / (torch.sqrt(v / (1 - 0.999 ** e)) + 1e-8)
    return (lb + (ub - lb) * torch.sigmoid(z)).detach().numpy(), loss.item()


def _fitting(**over):
    from gacelle_b200 import askadam_solver as gxa
    f = gxa.check_set_default_basic(dict({"iteration": 30, "initialLearnRate": 0.01, "lossFunction": "mse",
                                          "tol": 0.0, "patienceConvergence": float("inf"),
                                          "convergenceStepTol": 0.0, "convergenceGradTol": 0.0}, **over))
    return f


def test_oracle_askadam_matches_autograd_loop():
    rng = np.random.default_rng(8)
    th = _theta("r2s", 40, rng)
    y = oracle.forward(oracle.r2s(TE), th) + 0.01 * rng.standard_normal((12, 40))
    th0 = np.tile([[1.0], [30.0]], (1, 40))
    lb, ub = [0.0, 0.1], [2.0, 200.0]
    ref, ref_loss = _torch_askadam(y, th0, lb, ub, 30, 0.01)
    f = _fitting()
    r = oracle.askadam(oracle.r2s(TE), oracle.Volume(y, theta0=th0), oracle.adam_opts(lb, ub, f))
    np.testing.assert_allclose(r["final"], ref, rtol=1e-7)  # FP64 rounding through 30 normalised steps
    assert r["final_loss"] == pytest.approx(ref_loss, rel=1e-7)
    assert r["final_niter"] == 30


def test_oracle_askadam_tv_matches_autograd_loop():
    from gacelle_b200 import phantoms, utils
    mask = phantoms.ellipsoid_mask((7, 6, 5), 1.0)
    data, _ = phantoms.r2s_phantom(mask, 9)
    idx = utils.mask_index(mask)
    y = utils.reshape_ND2GD(data, idx).astype(np.float64)
    n = y.shape[1]
    th0 = np.tile([[1.0], [30.0]], (1, n))
    lb, ub = [0.0, 0.1], [2.0, 200.0]
    ref, ref_loss = _torch_askadam(y, th0, lb, ub, 20, 0.01, lam=1e-5, mask=mask, idx=idx)
    f = _fitting(iteration=20, **{"lambda": [1e-5], "regmap": ["R2star"], "TVmode": "3D"})
    f["_reg_index"], f["_reg_lambda"] = [1], [1e-5]
    vol = oracle.Volume(y, dims=mask.shape, grid_index=idx.astype(np.int32), theta0=th0)
    r = oracle.askadam(oracle.r2s(TE), vol, oracle.adam_opts(lb, ub, f))
    np.testing.assert_allclose(r["final"], ref, rtol=1e-7)  # FP64 rounding through 30 normalised steps
    assert r["final_loss"] == pytest.approx(ref_loss, rel=1e-7)


def test_oracle_min_loss_and_no_update_on_last_epoch():
    rng = np.random.default_rng(10)
    th = _theta("r2s", 30, rng)
    y = oracle.forward(oracle.r2s(TE), th)
    th0 = np.tile([[1.0], [30.0]], (1, 30))
    f = _fitting(iteration=1)
    r = oracle.askadam(oracle.r2s(TE), oracle.Volume(y, theta0=th0), oracle.adam_opts([0, 0.1], [2, 200], f))
    # one epoch: evaluation only, no update; the min state is the start
    np.testing.assert_allclose(r["final"], r["min"])
    assert r["min_niter"] == 0 and r["final_niter"] == 1
    assert r["loss_history"][0] == r["loss_history"][1]


def test_oracle_gradient_of_mean_normalisation():
    """loss = mean over Nmeas*Nvox (askadam.m:96): doubling the voxel count with
    copies halves every per-voxel gradient."""
    rng = np.random.default_rng(11)
    th = _theta("r2s", 10, rng)
    y = oracle.forward(oracle.r2s(TE), th) + 0.02
    o = oracle.adam_opts([0, 0.1], [2, 200], _fitting())
    _, g1, _, _, _ = oracle.model_gradient(oracle.r2s(TE), oracle.Volume(y), o, th)
    _, g2, _, _, _ = oracle.model_gradient(oracle.r2s(TE), oracle.Volume(np.hstack([y, y])), o, np.hstack([th, th]))
    np.testing.assert_allclose(g2[:, :10], g1 / 2, rtol=1e-12)


def _prior_problem(nv=50, seed=12):
    """An R2* problem with a prior on both parameters; some SDs are 0 (an
    infinite z-score) and one voxel sits on its mean with SD 0 (NaN): both
    drop out of the regulariser."""
    rng = np.random.default_rng(seed)
    th = _theta("r2s", nv, rng)
    y = oracle.forward(oracle.r2s(TE), th) + 0.01 * rng.standard_normal((12, nv))
    mu = np.vstack([rng.uniform(0.8, 1.2, nv), rng.uniform(20, 40, nv)])
    sd = np.vstack([rng.uniform(0.05, 0.2, nv), rng.uniform(2, 8, nv)])
    sd[0, 3] = 0.0
    sd[1, 7] = 0.0
    th_eval = th * rng.uniform(0.9, 1.1, th.shape)
    th_eval[1, 9] = mu[1, 9]
    sd[1, 9] = 0.0
    return y, th_eval, mu, sd


def test_prior_regulariser_matches_autograd():
    """prior_distribution_normal (NEXI/gpuNEXI.m:1256-1307) in the oracle's
    model_gradient against torch autograd of fidelity + lambda/N sum|z|."""
    y, th, mu, sd = _prior_problem()
    nv = y.shape[1]
    lam = [2e-3, 5e-4]
    f = _fitting(**{"lambda": lam, "regmap": ["M0", "R2star"], "regularisationType": "prior"})
    f["_reg_index"], f["_reg_lambda"] = [0, 1], lam
    o = oracle.adam_opts([0.0, 0.1], [2.0, 200.0], f)
    vol = oracle.Volume(y, prior_mu=mu, prior_sd=sd, prior_offset=0.125)
    L, g, _, fid, reg = oracle.model_gradient(oracle.r2s(TE), vol, o, th)
    t = torch.tensor(th, requires_grad=True)
    loss_fid = torch.mean(0.5 * (T.r2s_fwd(t, TE) - torch.tensor(y)) ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        ok = torch.tensor(np.isfinite((th - mu) / sd))
    # the dropped entries contribute no gradient (autodiff through the 0 SD
    # itself would give 0/0 there)
    sds = torch.tensor(np.where(sd == 0, 1.0, sd))
    z = (t - torch.tensor(mu)) / sds
    loss_reg = sum(lam[r] / nv * torch.sum(torch.abs(z[r][ok[r]])) for r in range(2)) + 0.125
    (loss_fid + loss_reg).backward()
    assert reg == pytest.approx(loss_reg.item(), rel=1e-13)
    assert fid == pytest.approx(loss_fid.item(), rel=1e-12)
    np.testing.assert_allclose(g, t.grad.numpy(), rtol=1e-10, atol=1e-16)
    assert np.isfinite(g).all()


def test_prior_host_loss_and_grid_offset():
    """gpuNEXI.prior_distribution_normal on the host equals the oracle's
    regulariser once the solver's offset for the grid points outside the
    mask (parameter image 0 there) is added."""
    from gacelle_b200 import gpuNEXI, utils
    from gacelle_b200.askadam_solver import askadam
    rng = np.random.default_rng(13)
    shape = (5, 4, 3)
    mask = rng.random(shape) > 0.4
    idx = utils.mask_index(mask)
    nv = idx.size
    fa = rng.uniform(0.2, 0.8, nv)
    mu = {"fa": rng.uniform(0.3, 0.7, shape).astype(np.float32)}
    sd = {"fa": rng.uniform(0.05, 0.2, shape).astype(np.float32)}
    sd["fa"][0, 0, 0] = 0.0
    host = gpuNEXI.prior_distribution_normal({"fa": fa[None, :]}, mask, [0.01], ["fa"], mu, sd)
    fitting = {"lambda": [0.01], "regmap": ["fa"]}
    m_rows, s_rows, off = askadam._prior_maps((mu, sd), fitting, mask, idx, nv)
    f = _fitting(**{"lambda": [0.01], "regmap": ["fa"], "regularisationType": "prior"})
    f["_reg_index"], f["_reg_lambda"] = [0], [0.01]
    om = oracle.nexi(np.array([1.0, 2.0]), np.array([20.0, 20.0]))
    th = np.vstack([fa.astype(np.float32), np.full(nv, 2.0), np.full(nv, 1.0), np.full(nv, 0.1)])
    vol = oracle.Volume(np.zeros((2, nv)), prior_mu=m_rows, prior_sd=s_rows, prior_offset=off)
    _, _, _, _, reg = oracle.model_gradient(om, vol, oracle.adam_opts([0, 0, 0, 0.004], [1, 3, 3, 1], f), th)
    assert off > 0
    assert reg == pytest.approx(host, rel=1e-6)   # float32 z-scores on the host


# ------------------------------------------------------------------ MCMC ----
def test_partner_is_uniform_derangement():
    counts = np.zeros((8, 8))
    for k in range(1, 4001):
        p = oracle.gw_partner(7, k, 0, 8)
        assert np.all(p != np.arange(8)) and sorted(p) == list(range(8))
        counts[np.arange(8), p] += 1
    off = counts[~np.eye(8, dtype=bool)]
    assert off.min() > 0.8 * off.mean() and off.max() < 1.2 * off.mean()


def test_mcmc_sample_count_matches_reference_formula():
    # Ns = numel(Nburnin+1:thinning:iteration)
    for it, b, t in [(5000, 0.2, 10), (100, 0.1, 3), (10, 0.0, 1), (2e5, 0.1, 20), (50, 7, 4)]:
        nb = math.floor(it * b) if b < 1 else int(b)
        assert oracle.lib().orc_mcmc_nsamples(int(it), b, t) == len(range(nb + 1, int(it) + 1, t))


def _posterior_grid(y, lb, ub, free_noise):
    g0 = np.linspace(0.6, 1.4, 161)
    g1 = np.linspace(5, 65, 241)
    g2 = np.linspace(lb[2], ub[2], 101) if free_noise else np.array([lb[2]])
    A, Bm, S = np.meshgrid(g0, g1, g2, indexing="ij")
    s = A[..., None] * np.exp(-TE * Bm[..., None])
    lp = -np.sum((s - y[:, 0]) ** 2, axis=-1) / (2 * S ** 2) - 12 * np.log(S)
    p = np.exp(lp - lp.max())
    p /= p.sum()
    mean = [np.sum(p * A), np.sum(p * Bm)]
    std = [np.sqrt(np.sum(p * (A - mean[0]) ** 2)), np.sqrt(np.sum(p * (Bm - mean[1]) ** 2))]
    return mean, std


def _gw_one_voxel(lb, ub, update, seed=17):
    om = oracle.r2s(TE)
    rng = np.random.default_rng(12)
    y = oracle.forward(om, np.array([[1.0], [35.0]])) + 0.05 * rng.standard_normal((12, 1))
    x0 = np.array([[1.0], [35.0], [0.05]])
    r = oracle.mcmc(om, oracle.Volume(np.repeat(y, 8, axis=1)), np.repeat(x0, 8, axis=1), lb, ub,
                    algorithm="ensemble", iteration=6000, thinning=2, burnin=0.2, nwalker=32, seed=seed,
                    ensemble_update=update, start_range=0.05)
    return r, y


@pytest.mark.parametrize("update", ["simultaneous", "redblack"])
def test_gw_posterior_known_answer(update):
    """One mono-exponential voxel, flat priors on the bounds (noise free in
    [0.02, 0.12]): posterior mean/std of M0 and R2* match 3-D grid quadrature."""
    lb, ub = [0.0, 0.1, 0.02], [2.0, 200.0, 0.12]
    r, y = _gw_one_voxel(lb, ub, update)
    mean, std = _posterior_grid(y, lb, ub, True)
    for k in range(2):
        assert abs(r["mean"][k].mean() - mean[k]) < 0.1 * std[k]
        assert r["std"][k].mean() == pytest.approx(std[k], rel=0.05)


def test_gw_pinned_parameter_keeps_reference_exponent():
    """Reference quirk kept for parity: with a parameter pinned (lb == ub, e.g.
    a fixed noise sigma) the stretch-move factor stays z^(Nvar-1) with Nvar
    counting the pinned parameter (utils/mcmc.m:313), which is not the
    exponent of the 2-D free space; the posterior std comes out inflated."""
    lb, ub = [0.0, 0.1, 0.05], [2.0, 200.0, 0.05]
    r, y = _gw_one_voxel(lb, ub, "simultaneous")
    mean, std = _posterior_grid(y, lb, ub, False)
    assert abs(r["mean"][0].mean() - mean[0]) < 0.2 * std[0]
    assert r["std"][0].mean() > 1.08 * std[0]


def _gw_global_problem(nv=4, seed=21):
    om = oracle.r2s(TE)
    rng = np.random.default_rng(seed)
    m0 = np.linspace(0.8, 1.2, nv)
    y = oracle.forward(om, np.vstack([m0, np.full(nv, 35.0)])) + 0.05 * rng.standard_normal((12, nv))
    return om, y


def _global_posterior_grid(y):
    """Marginal posterior of the shared (R2*, sigma) with each voxel's M0
    integrated out on its own grid; flat priors on the bounds."""
    g0 = np.linspace(0.5, 1.5, 201)
    g1 = np.linspace(15, 55, 161)
    g2 = np.linspace(0.02, 0.12, 101)
    E = np.exp(-TE[None, :] * g1[:, None])                       # [R2, m]
    logI = np.zeros((g1.size, g2.size))
    for u in range(y.shape[1]):
        s = g0[:, None, None] * E[None, :, :]                    # [M0, R2, m]
        sos = np.sum((s - y[None, None, :, u]) ** 2, axis=-1)    # [M0, R2]
        lL = -sos[:, :, None] / (2 * g2[None, None, :] ** 2) - 12 * np.log(g2)[None, None, :]
        mx = lL.max(axis=0)
        logI += mx + np.log(np.exp(lL - mx).sum(axis=0))
    p = np.exp(logI - logI.max())
    p /= p.sum()
    R, S = np.meshgrid(g1, g2, indexing="ij")
    mean = [np.sum(p * R), np.sum(p * S)]
    std = [np.sqrt(np.sum(p * (R - mean[0]) ** 2)), np.sqrt(np.sum(p * (S - mean[1]) ** 2))]
    return mean, std


@pytest.mark.parametrize("update", ["simultaneous", "redblack"])
def test_gw_global_parameters_known_answer(update):
    """goodman_weare_wglobal_constant (utils/mcmc.m:385-626): four voxels with
    their own M0 sharing R2* and the noise sigma (global, one value per walker,
    flat priors, none pinned).  The posterior mean/std of the shared parameters
    match quadrature of the exact marginal; a global parameter's statistics are
    the same for every voxel."""
    om, y = _gw_global_problem()
    nv = y.shape[1]
    lb, ub = [0.0, 0.1, 0.02], [2.0, 200.0, 0.12]
    x0 = np.vstack([np.ones(nv), np.full(nv, 30.0), np.full(nv, 0.05)])
    r = oracle.mcmc(om, oracle.Volume(y), x0, lb, ub, algorithm="ensemble", iteration=8000, thinning=2,
                    burnin=0.2, nwalker=32, seed=5, ensemble_update=update, start_range=0.05,
                    is_global=[0, 1, 1], global_warmup=20)
    mean, std = _global_posterior_grid(y)
    for k, q in ((1, 0), (2, 1)):
        assert np.ptp(r["mean"][k]) == 0 and np.ptp(r["std"][k]) == 0
        assert abs(r["mean"][k][0] - mean[q]) < 0.1 * std[q], (k, r["mean"][k][0], mean[q], std[q])
        assert r["std"][k][0] == pytest.approx(std[q], rel=0.06)


def test_gw_global_needs_local_and_global_parameters():
    om, y = _gw_global_problem(nv=2)
    x0 = np.vstack([np.ones(2), np.full(2, 30.0), np.full(2, 0.05)])
    with pytest.raises(ValueError):
        oracle.mcmc(om, oracle.Volume(y), x0, [0, 0.1, 0.02], [2, 200, 0.12], iteration=10, nwalker=8,
                    is_global=[1, 1, 1])
    with pytest.raises(ValueError):
        oracle.mcmc(om, oracle.Volume(y), x0, [0, 0.1, 0.02], [2, 200, 0.12], algorithm="mh",
                    x_step=[0.01, 1, 0.005], iteration=10, is_global=[0, 1, 0])


# ------------------------------------------------------ NEXI Rician mean ----
def _rice_setup(nv=40, seed=40):
    rng = np.random.default_rng(seed)
    b = np.tile([1.0, 2.5, 4.0, 6.0, 8.0, 10.0], 4)
    d = np.repeat([20.0, 27.0, 35.0, 49.0], 6)
    th = np.vstack([rng.uniform(0.2, 0.8, nv), rng.uniform(1.2, 2.8, nv), rng.uniform(0.6, 1.4, nv),
                    rng.uniform(0.02, 0.3, nv)])
    sigma = rng.uniform(0.02, 0.15, nv)
    return b, d, th, sigma


def test_nexi_rice_forward_matches_exact_rician_mean():
    """gpuNEXIrice.FWD: the Rician mean of the NEXI signal.  With exact Bessel
    functions (scipy) in place of the reference's 34-node trapezoids the mean
    agrees to the reference's stated trapezoid accuracy (NRMSE < 0.05 %,
    utils/gacelle_besseli.m:5), and it never falls below the noise-free
    signal."""
    from scipy.special import i0e, i1e
    b, d, th, sigma = _rice_setup()
    s0 = oracle.forward(oracle.nexi(b, d), th)
    s = oracle.forward(oracle.nexi_rice(b, d), th, b1=sigma)
    x = np.maximum(-s0 ** 2 / (2 * sigma ** 2), -170.0)
    L = (1 - x) * i0e(-x / 2) - x * i1e(-x / 2)
    exact = np.minimum(np.maximum(sigma * np.sqrt(np.pi / 2) * L, s0), 1.0)
    assert np.sqrt(np.mean((s - exact) ** 2)) / np.sqrt(np.mean(exact ** 2)) < 5e-4
    assert np.all(s >= np.minimum(s0, 1.0) - 1e-15)
    assert np.any(s > s0 + 1e-3)   # the Rician floor is active somewhere


def test_nexi_rice_vjp_matches_autograd_and_finite_differences():
    """Adjoint of the discretised model (the derivative MATLAB's autodiff takes
    of gpuNEXIrice.FWD) against torch float64 autograd through the same
    trapezoids, and against central differences."""
    import torch
    from oracle import torch_ref
    b, d, th, sigma = _rice_setup(nv=12, seed=41)
    om = oracle.nexi_rice(b, d)
    rng = np.random.default_rng(42)
    t = torch.tensor(th, dtype=torch.float64, requires_grad=True)
    s_t = torch_ref.nexi_rice_fwd(t, b, d, torch.tensor(sigma))
    np.testing.assert_allclose(s_t.detach().numpy(), oracle.forward(om, th, b1=sigma), rtol=1e-12, atol=1e-14)
    sbar = rng.standard_normal(s_t.shape)
    (s_t * torch.tensor(sbar)).sum().backward()
    g_auto = t.grad.numpy()
    for v in range(th.shape[1]):
        tb = oracle.vjp_voxel(om, th[:, v], sbar[:, v], b1=sigma[v])
        np.testing.assert_allclose(tb, g_auto[:, v], rtol=1e-8, atol=1e-12)
        for k in range(4):
            h = 1e-6 * max(abs(th[k, v]), 1e-3)
            tp, tm = th[:, v].copy(), th[:, v].copy()
            tp[k] += h
            tm[k] -= h
            fd = (oracle.forward(om, tp[:, None], b1=[sigma[v]])[:, 0] -
                  oracle.forward(om, tm[:, None], b1=[sigma[v]])[:, 0]) @ sbar[:, v] / (2 * h)
            assert abs(fd - tb[k]) <= 1e-5 * max(1.0, abs(tb[k])), (v, k, fd, tb[k])


# --------------------------------------------------- robustConvergence ----
def _robust_problem(nv=200, n_out=20, seed=60):
    """Voxels whose data the model fits well (parameters far from the start
    point) and outlier voxels whose data are the start point's signal plus
    large noise: their loss cannot improve, while the population improves."""
    rng = np.random.default_rng(seed)
    om = oracle.r2s(TE)
    th = np.vstack([rng.uniform(0.5, 1.5, nv), rng.uniform(10, 60, nv)])
    y = oracle.forward(om, th) + 0.005 * rng.standard_normal((12, nv))
    out = rng.choice(nv, n_out, replace=False)
    th0 = np.tile([[1.0], [30.0]], (1, nv))
    y[:, out] = oracle.forward(om, th0[:, out]) + 0.3 * rng.standard_normal((12, n_out))
    return om, y.astype(np.float32).astype(np.float64), th0, np.sort(out)


def test_robust_convergence_downweights_exactly_the_stagnant_voxels():
    """update_outlier_mask (utils/askadam.m:448-510): with an L1 loss (weights
    used), voxels flagged as outliers have their gradient scaled by
    outlierWeight, so exactly they leave the unweighted trajectory; the fit is
    voxel-separable, so every other voxel is unchanged.  With mse (weights
    ignored) nothing changes."""
    om, y, th0, out = _robust_problem()
    lb, ub = [0.0, 0.1], [2.0, 200.0]
    for loss, expect in (("l1", True), ("mse", False)):
        f = _fitting(iteration=300, lossFunction=loss)
        a = oracle.askadam(om, oracle.Volume(y, theta0=th0), oracle.adam_opts(lb, ub, f))
        b = oracle.askadam(om, oracle.Volume(y, theta0=th0),
                           oracle.adam_opts(lb, ub, dict(f, robustConvergence=True)))
        changed = np.flatnonzero(np.any(a["final"] != b["final"], axis=0))
        flagged = np.flatnonzero(b["ever_flagged"])
        assert flagged.size >= 5 and np.all(np.isin(flagged, out)), (flagged, out)
        if expect:
            np.testing.assert_array_equal(changed, flagged)
        else:
            assert changed.size == 0


def test_robust_convergence_judges_the_main_population():
    """With robustConvergence the convergence signal is the mean loss of the
    unflagged voxels (askadam.m:530-581): outliers that keep the
    full-population loss moving no longer hold the loop back, and the main
    population's plateau stops the robust run well before the plain run."""
    om, y, th0, out = _robust_problem(n_out=60, seed=61)
    lb, ub = [0.0, 0.1], [2.0, 200.0]
    f = _fitting(iteration=3000, lossFunction="l1", patienceConvergence=5, convergenceValue=1e-6,
                 convergenceModel="linear", initialLearnRate=0.02)
    a = oracle.askadam(om, oracle.Volume(y, theta0=th0), oracle.adam_opts(lb, ub, f))
    b = oracle.askadam(om, oracle.Volume(y, theta0=th0), oracle.adam_opts(lb, ub, dict(f, robustConvergence=True)))
    assert b["ever_flagged"].any() and np.all(np.isin(np.flatnonzero(b["ever_flagged"]), out))
    assert a["stop_reason"] == b["stop_reason"] == "convergence"
    assert b["final_niter"] < 0.6 * a["final_niter"], (b["final_niter"], a["final_niter"])


def test_res2out_summaries_restate_matlab_semantics():
    """Known answers of the res2out restatement: even/odd medians, the
    prctile midpoint rule, the histogram mode with its lowest-bin tie rule and
    samples outside the edges ignored."""
    import oracle
    x = np.array([[4.0, 1.0, 3.0, 2.0], [5.0, 1.0, 2.0, 2.0]])
    med, iqr, mode = oracle.res2out_summaries(x, 0.0, 10.0, nbin=11)
    assert med.tolist() == [2.5, 2.0]
    # n = 4: the 25th percentile sits at position 0.5 (0-based), the 75th at 2.5
    assert iqr[0] == pytest.approx((3.5 - 1.5), abs=1e-6)
    assert iqr[1] == pytest.approx((3.5 - 1.5), abs=1e-6)
    # bins of width 1 (+ 2e-9): row 0 has one sample per bin -> the lowest (x = 1) wins
    assert mode[0] == pytest.approx(1.5, abs=1e-6)
    assert mode[1] == pytest.approx(2.5, abs=1e-6)
    med, iqr, mode = oracle.res2out_summaries(np.array([[1.0, 2.0, 9.0]]), 0.0, 10.0, nbin=11)
    assert med[0] == 2.0
    # n = 3: 25th at position 0.25 -> 1.25; 75th at 1.75 -> 2 + 0.75 * 7 = 7.25
    assert iqr[0] == pytest.approx(7.25 - 1.25, abs=1e-6)
    _, _, mode = oracle.res2out_summaries(np.array([[20.0, 30.0]]), 0.0, 10.0, nbin=11)
    assert np.isnan(mode[0])
