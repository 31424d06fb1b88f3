"""Slab segmentation and the multi-rank fit on CPU ranks (gloo, world size 2).

Each rank's solver is the FP64 oracle (the engine needs a GPU); what is under
test is the segmentation (utils/utils.m:868-979), the owned-slice restore
(:1348-1470) and the all-gather across ranks, plus a rank that fails.
"""
import datetime
import os
import socket

import numpy as np

import oracle
from gacelle_b200 import phantoms, segments, utils

from helpers import fitting

TE = np.arange(2.0, 40.6, 3.5) * 1e-3


def test_balanced_boundaries_hand_cases():
    m = np.ones((2, 2, 4), dtype=bool)  # 4 voxels per slice
    b = segments.build_balanced_boundaries(m, 8, 1)
    assert [list(x) for x in b] == [[0, 1], [2, 3]]
    # densities 1, 5, 1, 1 (cumulative 1, 6, 7, 8), target 4: the candidate cuts
    # give 1 or 6 voxels, |1 - 4| = 3 > |6 - 4| = 2, so the cut follows slice 1
    m = np.zeros((5, 1, 4), dtype=bool)
    m[0, 0, 0] = True
    m[:, 0, 1] = True
    m[0, 0, 2] = True
    m[0, 0, 3] = True
    b = segments.build_balanced_boundaries(m, 4, 1)
    assert [list(x) for x in b] == [[0, 1], [2, 3]]
    assert len(segments.build_balanced_boundaries(m, 100, 3)) == 3


def test_halo_only_on_internal_faces():
    owned = [np.arange(0, 3), np.arange(3, 7), np.arange(7, 10)]
    s = segments.expand_segments_with_halo(owned, 2, 10)
    assert list(s[0]["fit"]) == [0, 1, 2, 3, 4] and list(s[0]["local"]) == [0, 1, 2]
    assert list(s[1]["fit"]) == list(range(1, 9)) and list(s[1]["local"]) == [2, 3, 4, 5]
    assert list(s[2]["fit"]) == [5, 6, 7, 8, 9] and list(s[2]["local"]) == [2, 3, 4]


def test_rank_segments_partition_the_mask():
    mask = phantoms.ellipsoid_mask((16, 14, 11), 1.0)
    for world in (1, 2, 3, 5):
        segs = segments.rank_segments(mask, world, overlap=1)
        owned = np.concatenate([s["owned"] for s in segs])
        assert list(owned) == list(range(11))
        counts = [mask[:, :, s["owned"]].sum() for s in segs]
        assert max(counts) - min(counts) <= mask.sum(axis=(0, 1)).max()


def _oracle_fit(f):
    """Per-slab solver for the CPU ranks: the FP64 oracle on the slab."""
    def fit(data, mask, extradata, pars0):
        idx = utils.mask_index(mask)
        y = utils.reshape_ND2GD(data, idx)
        th0 = np.tile([[1.0], [30.0]], (1, y.shape[1]))
        lam = float(np.atleast_1d(f["lambda"])[0])
        ff = dict(f, _reg_index=[1], _reg_lambda=[lam]) if lam > 0 else f
        o = oracle.adam_opts([0.0, 0.1], [2.0, 200.0], ff)
        vol = oracle.Volume(y.astype(np.float64), dims=mask.shape, grid_index=idx.astype(np.int32),
                            theta0=th0)
        r = oracle.askadam(oracle.r2s(TE), vol, o)
        maps = {k: utils.reshape_GD2ND(r["final"][i], mask).reshape(mask.shape, order="F")
                for i, k in enumerate(("M0", "R2star"))}
        return {"final": maps, "loss": r["final_loss"]}
    return fit


def _volume(shape=(10, 9, 8), seed=70):
    mask = phantoms.ellipsoid_mask(shape, 1.0)
    data, _ = phantoms.r2s_phantom(mask, seed)
    return data, mask


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    try:
        data, mask = _volume()
        if case == "fail":
            f = fitting(iteration=30)
            base = _oracle_fit(f)

            def fit(d, m, e, p):
                if rank == 1:
                    raise RuntimeError("rank 1 failed")
                return base(d, m, e, p)
            try:
                segments.fit_distributed(fit, data, mask)
                q.put((rank, "no error"))
            except Exception as ex:  # noqa: BLE001
                q.put((rank, type(ex).__name__ + ": " + str(ex)[:80]))
            return
        tv = case == "tv"
        f = fitting(iteration=60, **({"lambda": [1e-3], "regmap": ["R2star"], "TVmode": "3D"} if tv else {}))
        out = segments.fit_distributed(_oracle_fit(f), data, mask, overlap=2 if tv else 0)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _run(case):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, case, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, v = q.get(timeout=120)
        res[r] = v
    for p in procs:
        p.join(timeout=60)
    return res


def test_two_ranks_match_serial_segments_and_whole_fit():
    """No TV, no overlap: the slab fits gathered across two ranks equal the
    serial segmented fit, and stay close to the whole-volume fit (each slab's
    loss is a mean over its own voxels, which Adam absorbs up to its epsilon)."""
    res = _run("plain")
    data, mask = _volume()
    fit = _oracle_fit(fitting(iteration=60))
    segs = segments.rank_segments(mask, 2, overlap=0)
    serial = segments.restore_segments([fit(data[:, :, s["fit"]], mask[:, :, s["fit"]], None, None)
                                        for s in segs], segs, mask.shape)
    whole = fit(data, mask, None, None)
    for r in (0, 1):
        for k in ("M0", "R2star"):
            np.testing.assert_allclose(res[r]["final"][k], serial["final"][k], rtol=1e-12, atol=1e-15)
            np.testing.assert_allclose(res[r]["final"][k], whole["final"][k], rtol=1e-3, atol=1e-6)
        assert res[r]["loss"].shape == (2,)


def test_two_ranks_match_serial_segmented_tv_fit():
    """3-D TV with two halo slices: the distributed result equals the serial
    segmented fit with the same segments (the reference's segmented run)."""
    res = _run("tv")
    data, mask = _volume()
    f = fitting(iteration=60, **{"lambda": [1e-3], "regmap": ["R2star"], "TVmode": "3D"})
    segs = segments.rank_segments(mask, 2, overlap=2)
    fit = _oracle_fit(f)
    parts = [fit(data[:, :, s["fit"]], mask[:, :, s["fit"]], None, None) for s in segs]
    serial = segments.restore_segments(parts, segs, mask.shape)
    for r in (0, 1):
        for k in ("M0", "R2star"):
            np.testing.assert_allclose(res[r]["final"][k], serial["final"][k], rtol=1e-12, atol=1e-15)


def test_failing_rank_does_not_hang_the_other():
    """A rank that raises before the gather: the other rank's collective ends
    with an error (process-group timeout) instead of waiting forever."""
    res = _run("fail")
    assert "rank 1 failed" in res[1]
    assert res[0] != "no error"


def test_fit_segmented_slices_fits_and_restores():
    """The segment loop of estimate() (R2star/gpuR2starMapping.m:128-157,
    NEXI/gpuNEXI.m:209-236): each slab sees its haloed slices of data, mask,
    pars0 and (recursively) extradata; only owned slices are written back;
    scalars become one value per segment."""
    rng = np.random.default_rng(5)
    shape = (4, 3, 9)
    mask = rng.random(shape) > 0.3
    data = rng.random(shape + (2,))
    ex = {"b1": rng.random(shape), "mu": {"fa": rng.random(shape)}, "bval": np.arange(2.0), "dr": 0.5}
    p0 = {"fa": rng.random(shape)}
    seen = []

    def fit(d, m, e, p):
        seen.append(m.shape[2])
        assert d.shape[:3] == m.shape == e["b1"].shape == e["mu"]["fa"].shape == p["fa"].shape
        assert e["bval"].shape == (2,) and e["dr"] == 0.5
        return {"final": {"x": (d[..., 0] + e["b1"] + e["mu"]["fa"] + p["fa"]) * m, "loss": float(m.sum())}}

    out = segments.fit_segmented(fit, data, mask, 3, 1, ex, p0)
    # the other merge rules of restore_field (utils/utils.m:1446-1474)
    parts = [{"res": np.full((2, 3), k), "hist": np.arange(4.0) + k, "post": np.full((2, 5, 6), k),
              "other": np.full((2, 2, 2, 2), k)} for k in range(2)]
    segs2 = segments.rank_segments(mask, 2, 0)
    r = segments.restore_segments(parts, segs2, mask.shape)
    assert r["res"].shape == (2, 6) and r["res"][0, 3] == 1         # concatenated along voxels
    assert r["hist"].shape == (8,) and r["post"].shape == (4, 5, 6)
    assert r["other"].max() == 0                                     # kept from the first segment
    assert len(seen) == 3 and sum(seen) == 9 + 4            # three slabs, halos on the two internal faces
    np.testing.assert_allclose(out["final"]["x"], (data[..., 0] + ex["b1"] + ex["mu"]["fa"] + p0["fa"]) * mask)
    assert out["final"]["loss"].shape == (3,)
    whole = segments.fit_segmented(fit, data, mask, 1, 0, ex, p0)
    np.testing.assert_allclose(whole["final"]["x"], out["final"]["x"])
