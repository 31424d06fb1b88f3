"""Failure paths of the engine on the GPU, provoked without faulting the GPU.

The reference reports failures through MATLAB error identifiers
(``error('GACELLE:...')``) and catches out-of-memory around its fits
(utils/utils.m:698-706).  The engine's counterparts are the gx_status codes,
mirrored as ``GACELLE:b200:<status>``:

- GX_ECANCELLED: a host cancel flag, set before or during a call;
- GX_ETIMEOUT: the persistent TV kernel's bounded waits.  The context's test
  hooks shorten the bound (about 1 ms) and make the grid barrier wait for one
  arrival more than the grid makes, so the wait runs out: every CTA returns,
  the call reports the timeout and the context stays usable;
- GX_ENUMERIC: a non-finite loss (a NaN measurement), with the partial result;
- GX_ENOMEM: a device workspace request refused by the test hooks, at every
  request of a call in turn; afterwards the context is usable and gives the
  undisturbed result.
"""
import ctypes as C
import threading
import time

import numpy as np
import pytest

from gacelle_b200 import _lib

from helpers import NAMES, fitting, models, random_theta, rel_rmse, run_engine

pytestmark = pytest.mark.gpu


def _hooks(ctx, fail_alloc_at=0, wait_limit_cycles=0, barrier_extra_arrivals=0):
    h = _lib.GxTestHooks(fail_alloc_at, wait_limit_cycles, barrier_extra_arrivals)
    _lib.check(_lib.lib().gx_context_set_test_hooks(ctx.ptr, C.byref(h)))


def _clear(ctx):
    _lib.check(_lib.lib().gx_context_set_test_hooks(ctx.ptr, None))


def _r2s_voxels(n, seed):
    import oracle
    rng = np.random.default_rng(seed)
    _, om = models("r2s")
    th = random_theta("r2s", n, rng)
    y = (oracle.forward(om, th) + 0.01 * rng.standard_normal((12, n))).astype(np.float32)
    th0 = np.tile(np.array([[1.0], [30.0]], np.float32), (1, n))
    return y, th0


def _tv_volume(shape=(24, 24, 16), seed=3):
    from gacelle_b200 import phantoms, utils
    mask = phantoms.ellipsoid_mask(shape, 1.0)
    data, _ = phantoms.r2s_phantom(mask, seed)
    idx = utils.mask_index(mask)
    y = utils.reshape_ND2GD(data, idx)
    th0 = np.tile(np.array([[1.0], [30.0]], np.float32), (1, y.shape[1]))
    return y, th0, dict(dims=mask.shape, gidx=idx.astype(np.int32))


def _tv_fitting(iters=200):
    return fitting(iteration=iters, **{"lambda": [1e-4], "regmap": ["R2star"], "TVmode": "3D"})


@pytest.fixture
def own_ctx():
    """A context of its own, so that hooks and cancel flags never leak."""
    from gacelle_b200 import Context
    c = Context(0)
    yield c
    c.close()


def test_cancel_flag_set_before_the_call(own_ctx):
    y, th0 = _r2s_voxels(512, 1)
    flag = C.c_int32(1)
    _lib.check(_lib.lib().gx_set_cancel_flag(own_ctx.ptr, C.byref(flag)))
    for path in ("fused", "plain"):
        with pytest.raises(_lib.GacelleError) as e:
            run_engine("r2s", y, th0, fitting(iteration=100), NAMES["r2s"], path=path, context=own_ctx)
        assert e.value.status == _lib.GX_ECANCELLED, path
        assert e.value.identifier == "GACELLE:b200:cancelled"
    flag.value = 0
    res = run_engine("r2s", y, th0, fitting(iteration=100), NAMES["r2s"], context=own_ctx)
    assert np.all(np.isfinite(res["final_theta"]))
    _lib.check(_lib.lib().gx_set_cancel_flag(own_ctx.ptr, None))


def test_cancel_flag_set_while_a_fit_runs(own_ctx):
    """The op-by-op path polls the flag after every epoch: a flag raised by
    another host thread ends a long fit early."""
    y, th0 = _r2s_voxels(4096, 2)
    f = fitting(iteration=20000)
    flag = C.c_int32(0)
    _lib.check(_lib.lib().gx_set_cancel_flag(own_ctx.ptr, C.byref(flag)))
    # the same fit without cancellation takes > 1 s (20000 epochs, one launch per operation)
    timer = threading.Timer(0.3, lambda: setattr(flag, "value", 1))
    t0 = time.perf_counter()
    timer.start()
    with pytest.raises(_lib.GacelleError) as e:
        run_engine("r2s", y, th0, f, NAMES["r2s"], path="plain", context=own_ctx)
    dt = time.perf_counter() - t0
    timer.cancel()
    assert e.value.status == _lib.GX_ECANCELLED
    assert dt < 3.0, dt
    _lib.check(_lib.lib().gx_set_cancel_flag(own_ctx.ptr, None))


def test_grid_barrier_wait_runs_out_and_the_context_recovers(own_ctx):
    y, th0, kw = _tv_volume()
    f = _tv_fitting()
    good = run_engine("r2s", y, th0, f, NAMES["r2s"], context=own_ctx, **kw)
    assert good["timing"]["tv_path"] & _lib.TV_PERSISTENT
    _hooks(own_ctx, wait_limit_cycles=2_000_000, barrier_extra_arrivals=1)
    t0 = time.perf_counter()
    with pytest.raises(_lib.GacelleError) as e:
        run_engine("r2s", y, th0, f, NAMES["r2s"], context=own_ctx, **kw)
    assert e.value.status == _lib.GX_ETIMEOUT
    assert "grid barrier" in str(e.value)
    assert time.perf_counter() - t0 < 5.0
    # a short bound alone (no missing arrival) does not fire on a small volume
    _hooks(own_ctx, wait_limit_cycles=200_000_000)
    again = run_engine("r2s", y, th0, f, NAMES["r2s"], context=own_ctx, **kw)
    _clear(own_ctx)
    after = run_engine("r2s", y, th0, f, NAMES["r2s"], context=own_ctx, **kw)
    for r in (again, after):
        np.testing.assert_array_equal(r["final_theta"], good["final_theta"])
        np.testing.assert_array_equal(r["min_theta"], good["min_theta"])


def test_non_finite_data_reports_enumeric_with_the_partial_result(own_ctx):
    """A NaN measurement makes the loss NaN: the call returns GX_ENUMERIC and
    still writes the result.  Without TV the voxels are independent (the loss
    normalisation counts voxels, not values), so every other voxel equals the
    fit in which the NaN is replaced by a finite value."""
    y, th0 = _r2s_voxels(1000, 4)
    bad = y.copy()
    bad[5, 17] = np.nan
    f = fitting(iteration=150)
    clean = run_engine("r2s", y, th0, f, NAMES["r2s"], context=own_ctx)
    for path in ("fused", "plain"):
        with pytest.raises(_lib.GacelleError) as e:
            run_engine("r2s", bad, th0, f, NAMES["r2s"], path=path, context=own_ctx)
        assert e.value.status == _lib.GX_ENUMERIC, path
        assert e.value.identifier == "GACELLE:b200:numeric"
        part = e.value.partial
        assert not np.isfinite(part["final_loss"])
        keep = np.ones(1000, bool)
        keep[17] = False
        ref = clean if path == "fused" else run_engine("r2s", y, th0, f, NAMES["r2s"], path="plain",
                                                       context=own_ctx)
        np.testing.assert_array_equal(part["final_theta"][:, keep], ref["final_theta"][:, keep])


@pytest.mark.parametrize("case", ["fused", "plain", "tv_persistent", "mcmc"])
def test_injected_allocation_failure_at_every_request(own_ctx, case):
    """Each device workspace request of a call fails in turn (GX_ENOMEM, the
    engine's out-of-memory status); the context is then still usable and the
    undisturbed call gives the same result as before."""
    if case == "mcmc":
        from gacelle_b200 import mcmc_solver as gxm
        from gacelle_b200.models import _GxModelHandle
        y, th0 = _r2s_voxels(256, 5)
        x0 = np.vstack([th0, np.full(256, 0.01, np.float32)])
        fg = gxm.check_set_default_basic({"algorithm": "GW", "iteration": 20, "thinning": 1, "burnin": 0.0,
                                          "Nwalker": 16, "lb": [0.0, 0.1, 0.01], "ub": [2.0, 200.0, 0.01],
                                          "seed": 4})

        class _R2s:
            seed = 4

            def _gx_model(self):
                return _GxModelHandle(_lib.MODEL_R2S, te=np.arange(2.0, 40.6, 3.5) * 1e-3)

        def run():
            return gxm.mcmc(own_ctx)._run(_R2s(), y, None, x0, None, ["M0", "R2star", "noise"], fg, True)
        key = "posterior"
    else:
        if case == "tv_persistent":
            y, th0, kw = _tv_volume()
            f = _tv_fitting(100)
        else:
            y, th0 = _r2s_voxels(700, 6)
            kw = {}
            f = fitting(iteration=100)

        def run():
            return run_engine("r2s", y, th0, f, NAMES["r2s"], path="plain" if case == "plain" else "fused",
                              context=own_ctx, **kw)
        key = "final_theta"
    ref = run()
    failures = 0
    for k in range(1, 80):
        _hooks(own_ctx, fail_alloc_at=k)
        try:
            got = run()
        except _lib.GacelleError as e:
            assert e.status == _lib.GX_ENOMEM, (k, str(e))
            assert "injected" in str(e)
            failures += 1
            continue
        # k exceeds the call's requests: nothing was refused
        np.testing.assert_array_equal(got[key], ref[key])
        break
    else:
        pytest.fail("more than 80 workspace requests in one call")
    assert failures >= 5, failures
    _clear(own_ctx)
    np.testing.assert_array_equal(run()[key], ref[key])


def test_test_hooks_reject_negative_settings(own_ctx):
    h = _lib.GxTestHooks(-1, 0, 0)
    assert _lib.lib().gx_context_set_test_hooks(own_ctx.ptr, C.byref(h)) == _lib.GX_EINVAL
