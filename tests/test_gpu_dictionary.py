"""Dictionary starting points (gpuNEXI.likelihood, NEXI/gpuNEXI.m:813-836)
through the C-ABI against the FP64 oracle.

Both sides receive the same FP32 signals and dictionary; the engine
accumulates in FP64 in the expanded form, the oracle evaluates the reference's
direct form in FP64, so the chosen entries agree except where two entries tie
to within ~1e-12 of the score."""
import numpy as np
import pytest

import oracle
from gacelle_b200 import _lib

from helpers import models

pytestmark = pytest.mark.gpu


def _engine(ctx, S0, D, wt=None):
    S0 = np.ascontiguousarray(S0, np.float32)
    D = np.ascontiguousarray(D, np.float32)
    nm, nv = S0.shape
    best = np.zeros(nv, np.int32)
    sse = np.zeros(nv, np.float32)
    w = None if wt is None else np.ascontiguousarray(wt, np.float32)
    _lib.check(_lib.lib().gx_dictionary_match(ctx.ptr, _lib.MEM_HOST, S0.ctypes.data, nv, D.ctypes.data,
                                              D.shape[1], nm, None if w is None else w.ctypes.data,
                                              best.ctypes.data, sse.ctypes.data))
    return best, sse


def _nexi_dictionary(n, lmax, seed):
    rng = np.random.default_rng(seed)
    om = models("nexi2" if lmax == 2 else "nexi")[1]
    th = np.vstack([rng.uniform(0.01, 0.99, n), rng.uniform(1.5, 3, n), rng.uniform(0.5, 1.5, n),
                    rng.uniform(0.01, 0.5, n)] + ([rng.uniform(0.01, 0.99, n)] if lmax == 2 else []))
    return th, oracle.forward(om, th)


def _check_against_oracle(ctx, S0, D, wt):
    be, se = _engine(ctx, S0, D, wt)
    bo, so = oracle.dictionary_match(S0.astype(np.float32), D.astype(np.float32),
                                     None if wt is None else wt.astype(np.float32))
    diff = np.flatnonzero(be != bo)
    if diff.size:
        # near-ties only: the oracle scores the engine's choice as (almost) its best
        d = D.astype(np.float32).astype(np.float64)
        for i in diff:
            s0 = S0[:, i].astype(np.float64)
            def score(j):
                c = s0 @ d[:, j] / (d[:, j] @ d[:, j])
                r = s0 - c * d[:, j]
                return np.sum((1.0 if wt is None else wt.astype(np.float32).astype(np.float64)) * r * r)
            assert abs(score(be[i]) - score(bo[i])) <= 1e-12 * max(score(bo[i]), 1e-300) + 1e-18, i
    assert diff.size <= max(1, S0.shape[1] // 1000)
    np.testing.assert_allclose(se, so, rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("lmax,weighted,nv,nd", [(0, False, 2000, 3000), (0, True, 1999, 3001),
                                                 (2, True, 777, 1234), (2, False, 130, 65)])
def test_dictionary_match_matches_oracle(ctx, lmax, weighted, nv, nd):
    _, D = _nexi_dictionary(nd, lmax, 80 + lmax)
    th, S = _nexi_dictionary(nv, lmax, 90 + lmax)
    rng = np.random.default_rng(91)
    S0 = S * rng.uniform(0.5, 1.5, nv) + 0.01 * rng.standard_normal(S.shape)
    wt = None
    if weighted:
        nb = D.shape[0] // (lmax // 2 + 1)
        nav = rng.integers(6, 30, nb).astype(np.float64)
        wt = np.concatenate([nav / (2 * l + 1) for l in range(0, lmax + 1, 2)])
    _check_against_oracle(ctx, S0, D, wt)


def test_dictionary_match_recovers_scaled_entries(ctx):
    """A voxel signal equal to a scaled dictionary entry matches that entry
    exactly (score 0); all-zero entries never win; with only zero entries no
    entry scores."""
    _, D = _nexi_dictionary(500, 0, 82)
    pick = np.array([3, 77, 499, 250, 0])
    S0 = D[:, pick] * np.array([0.7, 1.0, 1.3, 0.9, 1.1])
    D2 = np.hstack([np.zeros((D.shape[0], 3)), D])
    be, se = _engine(ctx, S0, D2)
    np.testing.assert_array_equal(be, pick + 3)
    assert np.all(se <= 1e-10)
    be, _ = _engine(ctx, S0, np.zeros((D.shape[0], 4)))
    np.testing.assert_array_equal(be, -1)


def test_gpuNEXI_likelihood_start(ctx):
    """gpuNEXI.estimate_prior (NEXI/gpuNEXI.m:675-760) on the engine: voxels
    whose signals are scaled dictionary signals start at exactly the
    dictionary parameters; fit(start='likelihood') runs from them."""
    from gacelle_b200 import gpuNEXI
    b = np.tile([1.0, 2.5, 4.0, 6.0, 8.0, 10.0], 4)
    d = np.repeat([20.0, 27.0, 35.0, 49.0], 6)
    m = gpuNEXI(b, d)
    m.context = ctx
    x_train, S_train, _ = m.traindata(2000, 0)
    pick = np.arange(0, 2000, 97)
    dwi = (S_train[:, pick] * 0.9).T.reshape(len(pick), 1, 1, -1)
    mask = np.ones((len(pick), 1, 1), dtype=bool)
    pars = m.estimate_prior(dwi, mask, 2000, 0)
    # CSF correction (gpuNEXI.m:731-745): low-b apparent diffusivity above 1.5
    s_low = dwi.reshape(len(pick), -1)[:, m.b <= max(m.b.min(), 1.1)]
    bl = m.b[m.b <= max(m.b.min(), 1.1)]
    csf = (-np.log(s_low) @ bl) / (bl @ bl) > 1.5
    for k, p in enumerate(["fa", "Da", "De", "ra"]):
        expect = x_train[k, pick] * np.where(csf, [0.01, 1, 1, 0.01][k], 1.0)
        np.testing.assert_allclose(pars[p].ravel(), expect.astype(np.float32), rtol=1e-6)
    out = m.fit(dwi.astype(np.float32), mask, {"iteration": 20, "lossFunction": "mse"})
    assert out["final"]["fa"].shape == (len(pick), 1, 1)
