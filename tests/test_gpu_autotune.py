"""The project's autotuner (block_size = 0): the fused askAdam kernel's launch
block and the MCMC kernels' block shape are chosen by timed trials on the
first call of a key and cached for the process.  A tuned call reports the
chosen shape and that the trials ran; the next call of the same key reuses it
without trials; and the result equals the call with that block size given
explicitly (the per-voxel / per-walker arithmetic does not depend on the
launch shape).  GACELLE_B200_AUTOTUNE=0 keeps the default shape.
"""
import numpy as np
import pytest

import oracle
from gacelle_b200 import _lib

from helpers import NAMES, bounds, fitting, models, random_theta, run_engine

pytestmark = pytest.mark.gpu


def _nexi2_problem(n, seed):
    rng = np.random.default_rng(seed)
    gxm, om = models("nexi2")
    th = random_theta("nexi2", n, rng)
    s = oracle.forward(om, th)
    y = (s + 0.01 * rng.standard_normal(s.shape)).astype(np.float32)
    lb, ub = bounds("nexi2")
    th0 = np.tile(((np.array(lb) + np.array(ub)) / 2)[:, None], (1, n)).astype(np.float32)
    return y, th0


def test_fused_block_is_tuned_once_and_reused(ctx, monkeypatch):
    monkeypatch.delenv("GACELLE_B200_AUTOTUNE", raising=False)
    y, th0 = _nexi2_problem(20000, 60)   # a key no other test uses: lmax 2, RMSProp, Huber
    f = fitting(iteration=40, initialLearnRate=0.01, optimiser="rmsprop", lossFunction="huber")
    a = run_engine("nexi2", y, th0, f, NAMES["nexi2"], context=ctx)
    ta = a["timing"]
    assert ta["autotuned"] == 1 and ta["block_size"] in (32, 64, 128, 256, 512), ta
    b = run_engine("nexi2", y, th0, f, NAMES["nexi2"], context=ctx)
    assert b["timing"]["autotuned"] == 0 and b["timing"]["block_size"] == ta["block_size"]
    c = run_engine("nexi2", y, th0, dict(f, blockSize=ta["block_size"]), NAMES["nexi2"], context=ctx)
    assert c["timing"]["autotuned"] == 0 and c["timing"]["block_size"] == ta["block_size"]
    for r in (b, c):
        np.testing.assert_array_equal(r["final_theta"], a["final_theta"])
        np.testing.assert_array_equal(r["min_theta"], a["min_theta"])
    # every other block gives the same parameters too
    other = 64 if ta["block_size"] != 64 else 256
    d = run_engine("nexi2", y, th0, dict(f, blockSize=other), NAMES["nexi2"], context=ctx)
    np.testing.assert_array_equal(d["final_theta"], a["final_theta"])


def test_autotune_off_keeps_the_default_block(ctx, monkeypatch):
    monkeypatch.setenv("GACELLE_B200_AUTOTUNE", "0")
    y, th0 = _nexi2_problem(3000, 61)
    f = fitting(iteration=20, initialLearnRate=0.01, optimiser="sgdm", lossFunction="l2")
    r = run_engine("nexi2", y, th0, f, NAMES["nexi2"], context=ctx)
    assert r["timing"]["autotuned"] == 0 and r["timing"]["block_size"] == 128


@pytest.mark.parametrize("algorithm,update", [("ensemble", "redblack"), ("mh", "simultaneous")])
def test_mcmc_block_is_tuned_once_and_reused(ctx, monkeypatch, algorithm, update):
    from test_gpu_mcmc import _engine_mcmc
    monkeypatch.delenv("GACELLE_B200_AUTOTUNE", raising=False)
    rng = np.random.default_rng(62)
    gxm, om = models("r1r2s")
    nv = 1500
    th = random_theta("r1r2s", nv, rng)
    y = (oracle.forward(om, th) + 0.01 * rng.standard_normal((24, nv))).astype(np.float32)
    x0 = np.vstack([th, np.full(nv, 0.01)]).astype(np.float32)
    lb, ub = [0.0, 0.1, 0.1, 0.01], [2.0, 10.0, 200.0, 0.01]
    kw = dict(iteration=60, thinning=2, burnin=0.2, nwalker=24, seed=5, algorithm=algorithm, update=update,
              x_step=[0.01, 0.05, 1.0, 0.0])

    def run(block):
        def hook(r, o):
            o.block_size = block
        out = _engine_mcmc(ctx, gxm, y, x0, lb, ub, _hook=hook, **kw)
        out["timing"] = ctx.timing()
        return out
    a = run(0)
    assert a["timing"]["autotuned"] == 1, a["timing"]
    blk = a["timing"]["block_size"]
    if algorithm == "ensemble":
        assert blk % 12 == 0            # whole voxels of W / 2 threads (red-black)
    b = run(0)
    assert b["timing"]["autotuned"] == 0 and b["timing"]["block_size"] == blk
    c = run(blk)
    for r in (b, c):
        np.testing.assert_array_equal(r["posterior"], a["posterior"])
        np.testing.assert_array_equal(r["mean"], a["mean"])
        assert r["n_accepted"] == a["n_accepted"]
