"""Rotationally invariant signals and NEXI data preparation on the host
(utils/DWIutility.m, NEXI/gpuNEXI.m:480-633, NEXI/gpuNEXIrice.m:344-405).

Known answers: a shell signal S(g) = a + g'Ag is band-limited to degree 2,
so with enough directions the least-squares fit is exact and

    S_0 = a + tr(A)/3,   S_2 = sqrt(2 tr(A0^2) / 75),   A0 = A - tr(A)/3 I

(the moments <g_i g_j g_k g_l> over the sphere are
(d_ij d_kl + d_ik d_jl + d_il d_jk)/15), whatever the rotation of A."""
import math

import numpy as np
import pytest
from scipy.special import lpmv, sph_harm_y

from gacelle_b200 import GacelleError, gpuNEXI, gpuNEXIrice
from gacelle_b200.dwi import DWIutility, _legendre_nocs


def _dirs(n, rng):
    g = rng.standard_normal((n, 3))
    return g / np.linalg.norm(g, axis=1, keepdims=True)


def _rot(rng):
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    return q if np.linalg.det(q) > 0 else -q


def _sym(rng, scale=0.3):
    a = rng.standard_normal((3, 3)) * scale
    return (a + a.T) / 2


def _expected(a, A):
    A0 = A - np.trace(A) / 3 * np.eye(3)
    return a + np.trace(A) / 3, math.sqrt(2 * np.trace(A0 @ A0) / 75)


def test_legendre_and_real_sh_match_scipy():
    """The basis: associated Legendre without the Condon-Shortley phase and
    orthonormal real SH with getSH.m's column layout, against scipy."""
    x = np.linspace(-1, 1, 9)
    for n in range(5):
        P = _legendre_nocs(n, x)
        for m in range(n + 1):
            np.testing.assert_allclose(P[m], (-1) ** m * lpmv(m, n, x), rtol=1e-12, atol=1e-12)
    rng = np.random.default_rng(0)
    az = rng.uniform(-np.pi, np.pi, 25)
    inc = np.arccos(rng.uniform(-1, 1, 25))
    Y = DWIutility.getSH(4, np.stack([az, inc], 1))
    col = 0
    for n in range(5):
        for m in range(-n, n + 1):
            c = sph_harm_y(n, abs(m), inc, az)
            ref = c.real if m == 0 else math.sqrt(2) * (-1) ** m * (c.real if m > 0 else c.imag)
            np.testing.assert_allclose(Y[:, col], ref, rtol=1e-12, atol=1e-12)
            col += 1


def test_cart2sph_incl():
    d = DWIutility.cart2sph_incl(np.array([[0, 0, 1.0], [1, 0, 0], [0, 2, 0], [0, 0, 0]]))
    np.testing.assert_allclose(d, [[0, 0], [0, np.pi / 2], [np.pi / 2, np.pi / 2], [0, np.pi / 2]], atol=1e-15)


def test_shrotinv_known_answer_and_rotation_invariance():
    rng = np.random.default_rng(1)
    g = _dirs(30, rng)
    a = rng.uniform(0.3, 0.8, 5)
    As = [_sym(rng) for _ in range(5)]
    S = np.stack([a[k] + np.einsum("ni,ij,nj->n", g, As[k], g) for k in range(5)], axis=1)
    F = DWIutility().SHrotinv(S, g, 2)
    for k in range(5):
        s0, s2 = _expected(a[k], As[k])
        assert F[0, k] == pytest.approx(s0, rel=1e-12)
        assert F[1, k] == pytest.approx(s2, rel=1e-10)
    # the same tensors rotated, sampled on the same directions
    R = _rot(rng)
    Sr = np.stack([a[k] + np.einsum("ni,ij,nj->n", g, R @ As[k] @ R.T, g) for k in range(5)], axis=1)
    np.testing.assert_allclose(DWIutility().SHrotinv(Sr, g, 2), F, rtol=1e-10)
    # lmax 0 is the plain spherical mean of an isotropic shell; antipodes are
    # the same measurement (the doubling keeps the fit even)
    np.testing.assert_allclose(DWIutility().SHrotinv(np.full((7, 2), 0.25), _dirs(7, rng), 0), 0.25, rtol=1e-14)
    np.testing.assert_allclose(DWIutility().SHrotinv(S, -g, 2), F, rtol=1e-12)


def _acquisition(rng, shells, ndir, nb0, M0, coef):
    """Volumes of a full acquisition [x,y,z,vol]: nb0 b=0 volumes at M0, then
    ndir directions per shell with signal M0 (a_b + g'A_b g)."""
    vols, bval, bvec = [], [], []
    for _ in range(nb0):
        vols.append(M0)
        bval.append(0.0)
        bvec.append([0.0, 0.0, 0.0])
    for b in shells:
        g = _dirs(ndir, rng)
        for gi in g:
            a, A = coef(b)
            vols.append(M0 * (a + np.einsum("...ij,i,j->...", A, gi, gi)))
            bval.append(b)
            bvec.append(gi)
    return np.stack(vols, axis=-1), np.array(bval), np.array(bvec).T


def test_compute_rotationally_invariant_signal_single_te():
    """One TE: normalised by the b=0 S_0 and b=0 dropped; layout
    [S0 shells..., S2 shells...] with aligned descriptors
    (utils/DWIutility.m:10-165)."""
    rng = np.random.default_rng(2)
    dims = (3, 2, 2)
    M0 = rng.uniform(0.5, 2.0, dims)
    aa = {1.0: rng.uniform(0.5, 0.7, dims), 2.5: rng.uniform(0.2, 0.4, dims)}
    AA = {b: _sym(rng, 0.1) for b in aa}
    dwi, bval, bvec = _acquisition(rng, [2.5, 1.0], 24, 3, M0, lambda b: (aa[b], AA[b][None, None, None]))
    out, bo, lo, Do, to = DWIutility().compute_rotationally_invariant_signal(dwi, bval, bvec, None, 30.0, None, 2)
    assert out.shape == dims + (4,)
    np.testing.assert_array_equal(bo, [1.0, 2.5, 1.0, 2.5])
    np.testing.assert_array_equal(lo, [1, 1, 1, 1])
    np.testing.assert_array_equal(Do, [30, 30, 30, 30])
    np.testing.assert_array_equal(to, [0, 0, 0, 0])
    for k, b in enumerate([1.0, 2.5]):
        s0, s2 = _expected(0.0, AA[b])
        np.testing.assert_allclose(out[..., k], aa[b] + s0, rtol=1e-12)
        np.testing.assert_allclose(out[..., 2 + k], s2, rtol=1e-9)


def test_compute_rotationally_invariant_signal_multi_te():
    """Several TEs: no normalisation, b=0 kept once per TE in the S_0 block
    only, shells in TE -> little delta -> big delta -> b order."""
    rng = np.random.default_rng(3)
    dims = (2, 2, 1)
    parts, te = [], []
    for t, m0 in ((60.0, 2.0), (80.0, 1.5)):
        d, b, g = _acquisition(rng, [1.0, 2.0], 15, 2, np.full(dims, m0),
                               lambda bb: (np.full(dims, 0.8 / bb), np.zeros((1, 1, 1, 3, 3))))
        parts.append((d, b, g))
        te += [t] * b.size
    dwi = np.concatenate([p[0] for p in parts], axis=-1)
    bval = np.concatenate([p[1] for p in parts])
    bvec = np.concatenate([p[2] for p in parts], axis=1)
    out, bo, lo, Do, to = DWIutility().compute_rotationally_invariant_signal(dwi, bval, bvec, 5.0, 20.0,
                                                                            np.array(te), 2)
    np.testing.assert_array_equal(bo, [0, 1, 2, 0, 1, 2, 1, 2, 1, 2])
    np.testing.assert_array_equal(to, [60, 60, 60, 80, 80, 80, 60, 60, 80, 80])
    np.testing.assert_array_equal(lo, [5] * 10)
    np.testing.assert_allclose(out[..., :6], np.broadcast_to([2.0, 1.6, 0.8, 1.5, 1.2, 0.6], dims + (6,)),
                               rtol=1e-12)
    np.testing.assert_allclose(out[..., 6:], 0.0, atol=1e-12)


def test_get_sl_all_normalises_each_group_by_its_own_b0():
    """get_Sl_all (gpuNEXIrice's path): one normalisation per (little delta,
    big delta) group, groups ordered little delta then big delta."""
    rng = np.random.default_rng(4)
    dims = (2, 1, 1)
    blocks = []
    for D, m0, a in ((40.0, 3.0, 0.5), (20.0, 2.0, 0.7)):
        d, b, g = _acquisition(rng, [1.0, 3.0], 12, 2, np.full(dims, m0),
                               lambda bb, a=a: (np.full(dims, a / bb), np.zeros((1, 1, 1, 3, 3))))
        blocks.append((d, b, g, np.full(b.size, D)))
    dwi = np.concatenate([x[0] for x in blocks], axis=-1)
    bval = np.concatenate([x[1] for x in blocks])
    bvec = np.concatenate([x[2] for x in blocks], axis=1)
    BD = np.concatenate([x[3] for x in blocks])
    out, ball = DWIutility().get_Sl_all(dwi, bval, bvec, np.full(bval.size, 8.0), BD, 0)
    np.testing.assert_array_equal(ball, [1, 3, 1, 3])
    np.testing.assert_allclose(out[0, 0, 0], [0.7, 0.7 / 3, 0.5, 0.5 / 3], rtol=1e-12)


def test_unique_shell_keepb0_orders_and_b0_handling():
    u = DWIutility.unique_shell_keepb0
    b, ld, bd, te = u([0, 0, 1, 2, 0, 0, 1, 2], [10, 10, 10, 10, 20, 20, 20, 20],
                      [20, 20, 20, 20, 40, 40, 40, 40], [80] * 8)
    np.testing.assert_array_equal(b, [0, 1, 2, 1, 2])
    np.testing.assert_array_equal(ld, [10, 10, 10, 20, 20])
    np.testing.assert_array_equal(bd, [20, 20, 20, 40, 40])
    b, _, bd, _ = u([0, 1, 2, 0, 1, 2], None, [20, 20, 20, 40, 40, 40], None, True)
    np.testing.assert_array_equal(b, [1, 2, 1, 2])
    b, _, _, te = u([0, 1, 0, 1], None, None, [60, 60, 80, 80], True)   # several TEs keep b=0
    np.testing.assert_array_equal(b, [0, 1, 0, 1])
    np.testing.assert_array_equal(te, [60, 60, 80, 80])
    b, ld, bd = DWIutility.unique_shell([0, 2, 1, 2, 3], [5, 5, 5, 9, 9], [20, 20, 20, 30, 30])
    np.testing.assert_array_equal(b, [1, 2, 2, 3])
    np.testing.assert_array_equal(ld, [5, 5, 9, 9])


def test_gpunexi_prepare_dwi_data_masks():
    """gpuNEXI.prepare_dwi_data on per-shell input: impossible (|S0| > 1.1),
    background (first shell < 0.01), incoherent (correlation < 0.1 with the
    median decay) and NaN voxels leave the mask; NaN data become 0."""
    m = gpuNEXI([1.0, 2.0, 4.0, 6.0], [20.0] * 4)
    rng = np.random.default_rng(5)
    dims = (4, 3, 1)
    decay = np.array([0.8, 0.6, 0.4, 0.3])
    data = decay * rng.uniform(0.9, 1.1, dims + (1,)) + rng.normal(0, 0.005, dims + (4,))
    data[0, 0, 0] = [1.3, 0.6, 0.4, 0.3]          # impossible
    data[1, 0, 0] = [0.005, 0.004, 0.003, 0.002]  # background
    data[2, 0, 0] = [0.2, 0.4, 0.6, 0.8]          # rising: incoherent
    data[3, 0, 0] = [0.5, 0.5, 0.5, 0.5]          # flat: correlation 0
    data[0, 1, 0, 2] = np.nan                     # NaN
    mask = np.ones(dims, dtype=bool)
    mask[3, 2, 0] = False
    out, valid, _ = m.prepare_dwi_data(data, mask, {}, 0)
    expect = np.ones(dims, dtype=bool)
    for v in [(0, 0, 0), (1, 0, 0), (2, 0, 0), (3, 0, 0), (0, 1, 0), (3, 2, 0)]:
        expect[v] = False
    np.testing.assert_array_equal(valid, expect)
    assert out[0, 1, 0, 2] == 0.0 and np.isfinite(out).all()
    with pytest.raises(GacelleError):
        m.prepare_dwi_data(data[..., :3], mask, {}, 0)


def test_gpunexi_prepare_dwi_data_from_full_acquisition():
    """A full acquisition becomes its invariants: an isotropic shell at value
    v gives S0 = v exactly (in float64), S2 = 0."""
    rng = np.random.default_rng(6)
    dims = (3, 3, 1)
    Sl = np.stack([np.full(dims, v) for v in (0.75, 0.5, 0.3125)], axis=-1)
    shells = {1.0: 0, 2.0: 1, 5.0: 2}
    dwi, bval, bvec = _acquisition(rng, [5.0, 1.0, 2.0], 20, 2, np.full(dims, 2.0),
                                   lambda b: (Sl[..., shells[b]], np.zeros((1, 1, 1, 3, 3))))
    m = gpuNEXI(bval, np.full(bval.size, 30.0))
    assert list(m.b) == [1, 2, 5]
    for lmax in (0, 2):
        out, valid, _ = m.prepare_dwi_data(dwi, np.ones(dims, bool), {"bval": bval, "bvec": bvec,
                                                                      "BDELTA": 30.0}, lmax)
        assert out.shape == dims + (3 * (lmax // 2 + 1),)
        np.testing.assert_allclose(out[..., :3], Sl, rtol=1e-13)
        np.testing.assert_allclose(out[..., 3:], 0.0, atol=1e-13)
        assert np.array_equal(out[..., :3].astype(np.float32), Sl.astype(np.float32))
        assert valid.all()
    with pytest.raises(GacelleError):
        m.prepare_dwi_data(dwi, np.ones(dims, bool), {"bval": bval}, 0)


def test_gpunexirice_prepare_dwi_data_from_full_acquisition():
    """gpuNEXIrice: sigma normalised by the mean of all b=0 volumes, then the
    invariants of each (little delta, big delta) group normalised by the
    group's own b=0 mean."""
    rng = np.random.default_rng(7)
    dims = (2, 2, 1)
    parts = []
    for D, m0, vals in ((20.0, 2.0, (0.75, 0.5)), (40.0, 4.0, (0.625, 0.375))):
        shells = dict(zip((1.0, 2.5), vals))
        d, b, g = _acquisition(rng, [1.0, 2.5], 16, 1, np.full(dims, m0),
                               lambda bb, s=shells: (np.full(dims, s[bb]), np.zeros((1, 1, 1, 3, 3))))
        parts.append((d, b, g, np.full(b.size, D)))
    dwi = np.concatenate([p[0] for p in parts], axis=-1)
    bval = np.concatenate([p[1] for p in parts])
    bvec = np.concatenate([p[2] for p in parts], axis=1)
    BD = np.concatenate([p[3] for p in parts])
    m = gpuNEXIrice([1.0, 2.5, 1.0, 2.5], [20.0, 20.0, 40.0, 40.0])
    out, valid, ex = m.prepare_dwi_data(dwi, np.ones(dims, bool),
                                        {"bval": bval, "bvec": bvec, "ldelta": 10.0, "BDELTA": BD,
                                         "sigma": np.full(dims, 0.15)}, 0)
    np.testing.assert_allclose(out[0, 0, 0], [0.75, 0.5, 0.625, 0.375], rtol=1e-13)
    np.testing.assert_allclose(ex["sigma"], 0.15 / 3.0, rtol=1e-14)   # mean b0 = (2 + 4) / 2
    assert ex["ldelta"].shape == bval.shape and valid.all()
