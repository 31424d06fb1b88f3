"""Surface-based fitting on the host: FreeSurfer surface files, mesh
adjacency (utils/utils.m:1615-1821), the surface total variation
(NEXI/gpuNEXI.m:1165-1254) in the oracle against autograd, and the
gpuNEXI surface data checks (NEXI/gpuNEXI.m:482-548)."""
import os

import numpy as np
import pytest
import torch

import oracle
from gacelle_b200 import GacelleError, gpuNEXI, utils
from gacelle_b200.askadam_solver import askadam
from gacelle_b200.surface import get_surface_neighbours, mesh_neighbours, read_surf, write_surf


def sheet(nx, ny, flip=False, bump=0.3, scale=1.0):
    """A triangulated nx x ny sheet with a bump (vertices, faces); flip
    swaps the diagonal of every square, changing the adjacency."""
    x, y = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64), indexing="ij")
    z = bump * np.sin(x / 2.0) * np.cos(y / 3.0)
    v = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1) * scale
    idx = np.arange(nx * ny).reshape(nx, ny)
    f = []
    for i in range(nx - 1):
        for j in range(ny - 1):
            a, b, c, d = idx[i, j], idx[i + 1, j], idx[i, j + 1], idx[i + 1, j + 1]
            f += [[a, b, d], [a, d, c]] if not flip else [[a, b, c], [b, d, c]]
    return v, np.array(f)


def write_subject(tmp, nx=12, ny=10):
    """lh and rh white/pial surfaces with the same vertex count and different
    triangulations."""
    for h, flip in (("lh", False), ("rh", True)):
        v, f = sheet(nx, ny, flip)
        write_surf(os.path.join(tmp, f"{h}.white"), v, f)
        write_surf(os.path.join(tmp, f"{h}.pial"), v + np.array([0.0, 0.0, 2.0]) + 0.1 * v, f)
    return nx * ny


def brute_neighbours(faces, nv):
    """The reference's loop: per face corner, grow a sorted unique list."""
    lists = [[] for _ in range(nv)]
    for fc in faces:
        for j in range(3):
            vtx = fc[j]
            lists[vtx] = sorted(set(lists[vtx]) | {fc[(j + 1) % 3], fc[(j + 2) % 3]})
    return lists


def test_read_write_surf_roundtrip(tmp_path):
    v, f = sheet(5, 4)
    p = str(tmp_path / "lh.white")
    write_surf(p, v, f)
    v2, f2 = read_surf(p)
    np.testing.assert_array_equal(v2, v.astype(np.float32))
    np.testing.assert_array_equal(f2, f)
    with open(p, "rb") as fh:
        raw = fh.read()
    with open(p, "wb") as fh:
        fh.write(raw[:-10])                              # truncated
    with pytest.raises(GacelleError):
        read_surf(p)
    with open(p, "wb") as fh:
        fh.write(b"\xff\xff\xff" + raw[3:])             # quad-file magic
    with pytest.raises(GacelleError):
        read_surf(p)


def test_mesh_neighbours_match_reference_loop():
    for flip in (False, True):
        v, f = sheet(7, 6, flip)
        nb, pad = mesh_neighbours(f, v.shape[0])
        ref = brute_neighbours(f, v.shape[0])
        assert nb.shape[1] == max(len(r) for r in ref)
        for i, r in enumerate(ref):
            assert list(nb[i, :len(r)]) == r
            assert np.all(nb[i, len(r):] == i) and np.all(pad[i, len(r):]) and not pad[i, :len(r)].any()


def test_get_surface_neighbours_layout(tmp_path):
    nv = write_subject(str(tmp_path))
    nb, dr, edge = get_surface_neighbours(str(tmp_path), 0.5, ["lh", "rh"])
    assert nb.shape[:3] == (1, nv, 2) and dr.shape == nb.shape + (3,) and edge.shape == nb.shape
    for h, hemi in enumerate(("lh", "rh")):
        vw, fw = read_surf(str(tmp_path / f"{hemi}.white"))
        vp, _ = read_surf(str(tmp_path / f"{hemi}.pial"))
        mid = vw + 0.5 * (vp - vw)
        ref = brute_neighbours(fw, nv)
        for i in (0, 5, nv // 2, nv - 1):
            k = len(ref[i])
            assert list(nb[0, i, h, :k] - 1) == ref[i]                 # 1-based, per hemisphere
            assert np.all(nb[0, i, h, k:] == i + 1)                     # padding: the vertex itself
            np.testing.assert_allclose(edge[0, i, h, :k], np.linalg.norm(mid[ref[i]] - mid[i], axis=1))
            assert np.all(edge[0, i, h, k:] == 1e6)
    with pytest.raises(GacelleError):
        get_surface_neighbours(str(tmp_path), 0.5, ["xh"])


def _surface_problem(seed=0, nx=9, ny=8):
    rng = np.random.default_rng(seed)
    v, f = sheet(nx, ny)
    v2, f2 = sheet(nx, ny, flip=True)
    nv = nx * ny
    nbs, lens = [], []
    for vv, ff in ((v, f), (v2, f2)):
        nb, _ = mesh_neighbours(ff, nv)
        nbs.append(nb)
        lens.append(np.linalg.norm(vv[nb] - vv[:, None, :], axis=2))
    maxnb = max(n.shape[1] for n in nbs)
    for i in range(2):
        w = maxnb - nbs[i].shape[1]
        nbs[i] = np.concatenate([nbs[i], np.repeat(np.arange(nv)[:, None], w, axis=1)], axis=1)
        lens[i] = np.concatenate([lens[i], np.zeros((nv, w))], axis=1)
    neighbours = np.stack(nbs, axis=1)[None] + 1
    edge = np.stack(lens, axis=1)[None]
    edge[edge == 0] = 1e6
    mask = rng.random((1, nv, 2)) > 0.2
    return neighbours, edge.astype(np.float32), mask


def test_oracle_surface_tv_matches_autograd_and_host_loss():
    """The oracle's surface TV (exact adjoint scattered to both ends of every
    slot) against torch autograd of the reference's loss, and the host
    surface_total_variation on the same maps."""
    neighbours, edge, mask = _surface_problem()
    idx = utils.mask_index(mask)
    nvox = idx.size
    tables = askadam._surface_tables((neighbours, edge), mask, idx)
    rng = np.random.default_rng(1)
    th = np.vstack([rng.uniform(0.2, 0.8, nvox), rng.uniform(1, 3, nvox), rng.uniform(0.5, 1.5, nvox),
                    rng.uniform(0.01, 0.3, nvox)])
    lam = [3e-3, 1e-3]
    from test_oracle import _fitting
    f = _fitting(**{"lambda": lam, "regmap": ["fa", "ra"], "dataType": "surface"})
    f["_reg_index"], f["_reg_lambda"] = [0, 3], lam
    om = oracle.nexi(np.array([1.0, 2.0]), np.array([20.0, 20.0]))
    vol = oracle.Volume(np.zeros((2, nvox)), dims=mask.shape, grid_index=idx.astype(np.int32),
                        neighbours=tables[0], edge_length=tables[1])
    _, g, _, _, reg = oracle.model_gradient(om, vol, oracle.adam_opts([0, 0, 0, 0.004], [1, 3, 3, 1], f), th)
    f0 = _fitting(**{"lambda": [0.0]})
    _, g0, _, _, _ = oracle.model_gradient(om, vol, oracle.adam_opts([0, 0, 0, 0.004], [1, 3, 3, 1], f0), th)
    g = g - g0                                                    # the regulariser's part
    # torch: the reference's computation on the vertex grid
    ngrid = mask.size
    nbg = (neighbours.reshape((-1, neighbours.shape[3]), order="F") - 1
           + (np.arange(ngrid) // mask.shape[1] * mask.shape[1])[:, None])
    lg = torch.tensor(edge.reshape((-1, edge.shape[3]), order="F").astype(np.float64))
    t = torch.tensor(th, requires_grad=True)
    loss = 0
    for r, k in enumerate([0, 3]):
        img = torch.zeros(ngrid, dtype=torch.float64).index_put((torch.tensor(idx),), t[k])
        q = (img[:, None] - img[torch.tensor(nbg)]) / lg
        loss = loss + torch.sum(torch.abs(q[torch.tensor(idx)])) / nvox * lam[r]
    loss.backward()
    assert reg == pytest.approx(loss.item(), rel=1e-12)
    np.testing.assert_allclose(g, t.grad.numpy(), rtol=1e-10, atol=1e-15)
    host = gpuNEXI.surface_total_variation({"fa": th[0][None].astype(np.float32), "ra": th[3][None].astype(np.float32)},
                                           mask, neighbours, lam, ["fa", "ra"], edge)
    assert host == pytest.approx(reg, rel=1e-5)


def test_gpunexi_surface_data_checks(tmp_path):
    nv = write_subject(str(tmp_path))
    m = gpuNEXI([1.0, 2.0], [20.0, 20.0])
    f = m.check_set_default({"dataType": "surface", "lambda": [1e-3]})
    data = np.full((1, nv, 2, 2), 0.5)
    mask = np.ones((1, nv, 2), bool)
    with pytest.raises(GacelleError):                        # no surf_dir
        m.prepare_dwi_data(data, mask, {"hemisphere": ["lh", "rh"]}, 0, f)
    with pytest.raises(GacelleError):                        # hemisphere count != Nhemi
        m.prepare_dwi_data(data, mask, {"surf_dir": str(tmp_path), "hemisphere": ["lh"]}, 0, f)
    with pytest.raises(GacelleError):                        # not [1, Nvertex, Nhemi]
        m.prepare_dwi_data(np.full((2, nv, 1, 2), 0.5), np.ones((2, nv, 1), bool),
                           {"surf_dir": str(tmp_path), "hemisphere": ["lh"]}, 0, f)
    with pytest.raises(GacelleError):                        # arbitrary split
        m.prepare_dwi_data(data, mask, {"surf_dir": str(tmp_path), "hemisphere": ["lh", "rh"]}, 0,
                           dict(f, NSegmentUser=3))
    d, mk, ex = m.prepare_dwi_data(data, mask, {"surf_dir": str(tmp_path), "hemisphere": ["lh", "rh"]}, 0, f)
    assert ex["neighbours"].shape[:3] == (1, nv, 2) and ex["dr"].shape == ex["neighbours"].shape
    assert mk.all()
    nb2, _ = m.get_surface_geometry(str(tmp_path), 0.5, ["lh", "rh"])
    assert nb2 is ex["neighbours"]                           # cached geometry
    with pytest.raises(GacelleError):                        # fit without the geometry
        m.fit(data, mask, dict(f, start="default"))
