"""GPU test of gx_askadam_noalloc, the askAdam entry point that allocates no
memory.  It exists for callers that cannot call cudaMalloc while running:
applications whose framework owns all device memory through its own
allocator, or pipelines that reserve memory up front and must not allocate
or run out of memory later.  They pass device buffers in and out and the
engine works in a fixed array inside the library.

The entry point must give the same parameters as gx_askadam (the existing
entry point) within the parity tolerance of the other tests (relative RMSE
1e-4; in practice identical), on two calls in a row, because every call
reuses the same fixed working array; and the device's free memory must not
change across a call.  This file is collected last so that a
run stopping at the first failure has already run every other test; it also
passes alone in a fresh process.
"""
import ctypes as C
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(kind, nvox, seed):
    import oracle
    from gacelle_b200 import _lib
    from gacelle_b200.models import _GxModelHandle
    rng = np.random.default_rng(seed)
    if kind == "r2s":
        te = np.arange(2.0, 40.6, 3.5) * 1e-3
        th = np.vstack([rng.uniform(0.5, 1.5, nvox), rng.uniform(10, 60, nvox)])
        s = oracle.forward(oracle.r2s(te), th)
        model = _GxModelHandle(_lib.MODEL_R2S, te=te)
        lb, ub, names = [0.0, 0.1], [2.0, 200.0], ["M0", "R2star"]
        th0 = np.tile(np.array([[1.0], [30.0]], np.float32), (1, nvox))
    else:
        b = np.tile([1.0, 2.5, 4.0, 6.0, 8.0, 10.0], 4)
        d = np.repeat([20.0, 27.0, 35.0, 49.0], 6)
        th = np.vstack([rng.uniform(0.2, 0.8, nvox), rng.uniform(1, 3, nvox), rng.uniform(0.5, 1.5, nvox),
                        rng.uniform(0.02, 0.2, nvox)])
        s = oracle.forward(oracle.nexi(b, d, nx=14), th)
        model = _GxModelHandle(_lib.MODEL_NEXI, bval=b, delta=d, nx=14)
        lb, ub = [2.2e-16, 2.2e-16, 2.2e-16, 1 / 250], [1.0, 3.0, 3.0, 1.0]
        names = ["fa", "Da", "De", "ra"]
        th0 = np.tile(np.array([[0.4], [2.0], [1.0], [0.05]], np.float32), (1, nvox))
    y = (s + 0.01 * rng.standard_normal(s.shape)).astype(np.float32)
    return model, y, th0, lb, ub, names


@pytest.mark.parametrize("kind,nvox,iters", [("r2s", 3001, 300), ("nexi", 700, 60)])
def test_noalloc_matches_askadam_on_two_calls(kind, nvox, iters):
    import torch
    from gacelle_b200 import Context, _lib, askadam_solver

    model, y, th0, lb, ub, names = _problem(kind, nvox, 31)
    f = askadam_solver.check_set_default_basic({
        "iteration": iters, "initialLearnRate": 0.01, "lossFunction": "mse", "tol": 0.0,
        "patienceConvergence": float("inf"), "convergenceStepTol": 0.0, "convergenceGradTol": 0.0})
    opts = askadam_solver.build_opts(f, names, lb, ub)

    # the existing entry point
    ctx = Context.default(0)
    solver = askadam_solver.askadam(ctx)
    ref = solver._run(model, y, None, th0, None, None, np.arange(nvox, dtype=np.int32), (nvox, 1, 1), opts,
                      y.shape[0], len(names))

    # the allocation-free entry point on device buffers the caller owns
    dev = torch.device("cuda", 0)
    d_y = torch.from_numpy(y).to(dev)
    d_th0 = torch.from_numpy(th0).to(dev)
    d_out = torch.full((len(names), nvox), float("nan"), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    L = _lib.lib()
    for call in range(2):
        d_out.fill_(float("nan"))
        loss = C.c_double(0.0)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        st = L.gx_askadam_noalloc(C.byref(model.s), d_y.data_ptr(), d_th0.data_ptr(), nvox, C.byref(opts),
                                  C.c_void_p(stream.cuda_stream), d_out.data_ptr(), C.byref(loss))
        assert st == _lib.GX_OK, L.gx_last_error()
        free1 = torch.cuda.mem_get_info(dev)[0]
        if call == 1:
            # the first call may load the library's kernels onto the device; the
            # second one finds everything in place and allocates nothing
            assert free1 == free0, (free0, free1)
        out = d_out.cpu().numpy()
        assert np.all(np.isfinite(out)), call
        for k in range(len(names)):
            a, b = out[k].astype(np.float64), ref["final_theta"][k].astype(np.float64)
            err = np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2))
            assert err <= 1e-4, (call, k, err)
        assert loss.value == pytest.approx(ref["final_loss"], rel=1e-6), call


def test_noalloc_rejects_problems_beyond_its_fixed_memory():
    import torch
    from gacelle_b200 import _lib, askadam_solver

    model, y, th0, lb, ub, names = _problem("r2s", 64, 32)
    f = askadam_solver.check_set_default_basic({
        "iteration": 10, "lossFunction": "mse", "tol": 0.0, "patienceConvergence": float("inf"),
        "convergenceStepTol": 0.0, "convergenceGradTol": 0.0})
    opts = askadam_solver.build_opts(f, names, lb, ub)
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    L = _lib.lib()
    # 50 million voxels cannot fit the 32 MiB array: rejected before any device work
    st = L.gx_askadam_noalloc(C.byref(model.s), d.data_ptr(), d.data_ptr(), 50_000_000, C.byref(opts), None,
                              d.data_ptr(), None)
    assert st == _lib.GX_EINVAL
    msg = L.gx_last_error().decode()
    m = re.search(r"at most (\d+) voxels", msg)
    assert m, msg
    nmax = int(m.group(1))
    assert 100_000 < nmax < 50_000_000
    # the reported maximum is accepted, one voxel more is not
    big_y = torch.zeros((y.shape[0], nmax + 1), dtype=torch.float32, device="cuda")
    big_th = torch.ones((2, nmax + 1), dtype=torch.float32, device="cuda")
    big_th[1] = 30.0
    big_out = torch.empty((2, nmax + 1), dtype=torch.float32, device="cuda")
    st = L.gx_askadam_noalloc(C.byref(model.s), big_y.data_ptr(), big_th.data_ptr(), nmax + 1, C.byref(opts),
                              None, big_out.data_ptr(), None)
    assert st == _lib.GX_EINVAL
    st = L.gx_askadam_noalloc(C.byref(model.s), big_y.data_ptr(), big_th.data_ptr(), nmax, C.byref(opts), None,
                              big_out.data_ptr(), None)
    assert st == _lib.GX_OK, L.gx_last_error()
    assert torch.isfinite(big_out[:, :nmax]).all()
    # stopping criteria cannot be honoured without the host-driven path
    f2 = dict(f, tol=1e-3)
    o2 = askadam_solver.build_opts(f2, names, lb, ub)
    st = L.gx_askadam_noalloc(C.byref(model.s), d.data_ptr(), d.data_ptr(), 64, C.byref(o2), None,
                              d.data_ptr(), None)
    assert st == _lib.GX_EUNSUPPORTED
    # robustConvergence belongs to gx_askadam's op-by-op path: refused, not silently ignored
    o3 = askadam_solver.build_opts(f, names, lb, ub)
    o3.robust_convergence = 1
    st = L.gx_askadam_noalloc(C.byref(model.s), d.data_ptr(), d.data_ptr(), 64, C.byref(o3), None,
                              d.data_ptr(), None)
    assert st == _lib.GX_EUNSUPPORTED
    # unknown loss / optimiser / transform kinds are rejected as gx_askadam rejects them
    for field, bad in (("loss", 17), ("optimiser", 9), ("transform", 5)):
        o4 = askadam_solver.build_opts(f, names, lb, ub)
        setattr(o4, field, bad)
        st = L.gx_askadam_noalloc(C.byref(model.s), d.data_ptr(), d.data_ptr(), 64, C.byref(o4), None,
                                  d.data_ptr(), None)
        assert st == _lib.GX_EINVAL, field
