"""DESPOT1 and the joint R1-R2* starting points / data scaling on the host
(MCRMWI/private/despot1.m, R1R2s/gpuJointR1R2starMapping.m:327-368,474-492),
checked on noise-free signals whose T1 and M0 are known."""
import numpy as np
import pytest

from gacelle_b200 import models


def _spgr(m0, t1, fa_deg, tr, b1=1.0):
    a = np.deg2rad(np.asarray(fa_deg) * b1)
    e1 = np.exp(-tr / t1)
    return m0 * np.sin(a) * (1 - e1) / (1 - np.cos(a) * e1)


@pytest.mark.parametrize("fa", [[5.0, 20.0], [3.0, 8.0, 15.0, 30.0]])
def test_despot1_recovers_t1_and_m0(fa):
    rng = np.random.default_rng(3)
    tr = 0.03
    m0 = rng.uniform(0.5, 2.0, (6, 5, 4))
    t1 = rng.uniform(0.4, 2.5, (6, 5, 4))
    b1 = rng.uniform(0.8, 1.2, (6, 5, 4))
    img = _spgr(m0[..., None], t1[..., None], fa, tr, b1[..., None])
    t1e, m0e, ok = models.despot1(tr, fa).estimate(img, None, b1)
    assert ok.all()
    np.testing.assert_allclose(t1e, t1, rtol=1e-9)
    np.testing.assert_allclose(m0e, m0, rtol=1e-9)


def test_despot1_zero_and_infeasible_voxels_are_dropped():
    fa, tr = [5.0, 20.0], 0.03
    img = np.zeros((2, 1, 1, 2))
    img[1, 0, 0] = [0.2, 0.01]   # signal falling too steeply: E1 <= 0, no real T1 > 0
    t1, m0, ok = models.despot1(tr, fa).estimate(img)
    assert not ok.any() and np.all(t1 == 0) and np.all(m0 == 0)


def test_despot1_checks_sizes():
    with pytest.raises(models.GacelleError):
        models.despot1(0.03, [5.0]).fit(np.ones(1))
    with pytest.raises(models.GacelleError):
        models.despot1(0.03, [5.0, 20.0]).fit(np.ones(3))


def test_joint_r1r2s_prior_and_scaling():
    te = np.linspace(2, 40, 12) * 1e-3
    fa, tr = np.array([5.0, 20.0]), 0.03
    rng = np.random.default_rng(4)
    d3 = (5, 4, 3)
    m0 = rng.uniform(500, 2000, d3)
    r1 = rng.uniform(0.5, 1.5, d3)
    r2 = rng.uniform(10, 60, d3)
    r2[0, 0, 0] = 0.3  # below R1/2 is impossible here; force R2* < R1 to test the rule
    mask = np.ones(d3, dtype=bool)
    s = _spgr(m0[..., None, None], 1 / r1[..., None, None], fa, tr) * np.exp(-te[:, None] * r2[..., None, None])
    m = models.gpuJointR1R2starMapping(te, tr, fa)
    img, mask2, scale = m.prepare_data(s, mask)
    assert mask2.all()
    # DESPOT1 on the first echo sees M0 exp(-TE1 R2*)
    np.testing.assert_allclose(scale, np.percentile(m0 * np.exp(-te[0] * r2), 98, method="hazen"), rtol=1e-9)
    np.testing.assert_allclose(img * scale, s)
    p = m.estimate_prior(img, mask2)
    # M0 and R1 from DESPOT1 on the first echo (M0 carries exp(-TE1 R2*)), clamped to the bounds
    m0_first = m0 * np.exp(-te[0] * r2) / scale
    np.testing.assert_allclose(p["M0"], np.clip(m0_first, m.lb[0], m.ub[0]), rtol=1e-5)
    np.testing.assert_allclose(p["R1"], np.clip(r1, m.lb[1], m.ub[1]), rtol=1e-5)
    r2e = p["R2star"]
    assert r2e[0, 0, 0] == pytest.approx(p["R1"][0, 0, 0] / 2, rel=1e-6)
    assert np.all(r2e >= m.lb[2]) and np.all(r2e <= m.ub[2])
    assert np.all(p["noise"] == np.float32(m.startPoint[3]))
