"""Cortical-surface geometry for surface-based fitting (fitting.dataType
'surface'): the mesh adjacency and edge lengths that the surface total
variation of gpuNEXI regularises over (utils/utils.m:1615-1821,
utils.get_surface_neighbours).

Surfaces are FreeSurfer triangle files (``lh.white``, ``lh.pial``, ...),
read by :func:`read_surf` from the published binary layout: a 3-byte
big-endian magic number 0xFFFFFE, a creation line and an empty line, then
big-endian int32 vertex and face counts, float32 xyz per vertex and int32
vertex triplets per face (0-based).  The reference reads them with the
FreeSurfer MATLAB toolbox's ``read_surf``, which is not part of it.

Host-side numpy; the geometry is computed once per subject, not per
iteration.
"""
from __future__ import annotations

import os

import numpy as np

from ._lib import GacelleError, GX_EINVAL, GX_EUNSUPPORTED

TRIANGLE_MAGIC = 0xFFFFFE
EDGE_LENGTH_SENTINEL = 1e6  # utils/utils.m:1815: zero lengths (padding) become this


def read_surf(path):
    """(vertices [Nv, 3] float64, faces [Nf, 3] int64, 0-based) of a FreeSurfer
    triangle surface file."""
    with open(path, "rb") as fh:
        raw = fh.read()
    if len(raw) < 3:
        raise GacelleError(GX_EINVAL, f"{path}: not a FreeSurfer surface file")
    magic = int.from_bytes(raw[:3], "big")
    if magic != TRIANGLE_MAGIC:
        raise GacelleError(GX_EUNSUPPORTED, f"{path}: only FreeSurfer triangle surfaces are read "
                                            f"(magic {magic:#x})")
    try:
        # creation line, then an empty line
        p = raw.index(b"\n", 3) + 1
        p = raw.index(b"\n", p) + 1
        nv, nf = (int(x) for x in np.frombuffer(raw, dtype=">i4", count=2, offset=p))
        p += 8
        v = np.frombuffer(raw, dtype=">f4", count=3 * nv, offset=p).reshape(-1, 3)
        p += 12 * nv
        f = np.frombuffer(raw, dtype=">i4", count=3 * nf, offset=p).reshape(-1, 3)
    except ValueError as exc:
        raise GacelleError(GX_EINVAL, f"{path}: truncated FreeSurfer surface file ({exc})") from None
    if f.size and (f.min() < 0 or f.max() >= nv):
        raise GacelleError(GX_EINVAL, f"{path}: face vertex index outside [0, {nv})")
    return v.astype(np.float64), f.astype(np.int64)


def write_surf(path, vertices, faces, created_by="gacelle_b200"):
    """Write a FreeSurfer triangle surface file (the layout :func:`read_surf`
    reads)."""
    vertices = np.asarray(vertices, dtype=">f4").reshape(-1, 3)
    faces = np.asarray(faces, dtype=">i4").reshape(-1, 3)
    with open(path, "wb") as fh:
        fh.write(TRIANGLE_MAGIC.to_bytes(3, "big"))
        fh.write(f"created by {created_by}\n\n".encode())
        fh.write(np.array([vertices.shape[0], faces.shape[0]], dtype=">i4").tobytes())
        fh.write(vertices.tobytes())
        fh.write(faces.tobytes())


def mesh_neighbours(faces, nvertex):
    """Per-vertex neighbour lists of a triangle mesh, each sorted ascending
    without repeats (the reference grows ``unique([...])`` per face corner,
    utils/utils.m:1709-1716), as a [Nv, maxNeighbours] array of 0-based
    indices padded with the vertex's own index, plus the padding mask."""
    f = np.asarray(faces, dtype=np.int64)
    src = np.concatenate([f[:, 0], f[:, 0], f[:, 1], f[:, 1], f[:, 2], f[:, 2]])
    dst = np.concatenate([f[:, 1], f[:, 2], f[:, 2], f[:, 0], f[:, 0], f[:, 1]])
    pairs = np.unique(src * nvertex + dst)
    s, d = pairs // nvertex, pairs % nvertex
    counts = np.bincount(s, minlength=nvertex)
    maxnb = int(counts.max()) if counts.size else 0
    start = np.concatenate([[0], np.cumsum(counts)[:-1]])
    slot = np.arange(s.size) - start[s]
    nb = np.repeat(np.arange(nvertex)[:, None], max(maxnb, 1), axis=1)
    pad = np.ones_like(nb, dtype=bool)
    nb[s, slot] = d
    pad[s, slot] = False
    return nb[:, :maxnb], pad[:, :maxnb]


def get_surface_neighbours(surf_dir, depth=0.5, hemisphere=("lh", "rh")):
    """utils.get_surface_neighbours (utils/utils.m:1615-1821): adjacency of the
    white-matter mesh and edge vectors on the surface at ``depth`` between
    white (0) and pial (1).  Returns (neighbours, dr, edgeLength) in the
    reference's [1, Nvertex, Nhemi, maxNeighbours(, 3)] layout with 1-based
    per-hemisphere vertex indices; padding slots name the vertex itself, and
    every zero edge length becomes 1e6."""
    depth = 0.5 if depth is None else float(depth)
    if isinstance(hemisphere, str):
        hemisphere = [hemisphere]
    hemisphere = list(hemisphere)
    if not hemisphere or any(h not in ("lh", "rh") for h in hemisphere):
        raise GacelleError(GX_EINVAL, f"hemisphere must be a non-empty subset of {{'lh','rh'}}, got {hemisphere}")
    if not os.path.isdir(surf_dir):
        raise GacelleError(GX_EINVAL, f"surf_dir does not exist: {surf_dir}")
    per = []
    for h in hemisphere:
        vw, fw = read_surf(os.path.join(surf_dir, h + ".white"))
        vp, _ = read_surf(os.path.join(surf_dir, h + ".pial"))
        mid = vw + depth * (vp - vw)
        nb, pad = mesh_neighbours(fw, vw.shape[0])
        dr = mid[nb] - mid[:, None, :]
        per.append((nb, dr, pad, vw.shape[0]))
    nverts = {p[3] for p in per}
    if len(nverts) > 1:
        raise GacelleError(GX_EINVAL, "Requested hemispheres have different vertex counts "
                                      f"({' '.join(str(p[3]) for p in per)}) and cannot be concatenated.")
    nvert = per[0][3]
    maxnb = max(p[0].shape[1] for p in per)
    nbs, drs = [], []
    for nb, dr, _, _ in per:
        w = maxnb - nb.shape[1]
        if w > 0:
            nb = np.concatenate([nb, np.repeat(np.arange(nvert)[:, None], w, axis=1)], axis=1)
            dr = np.concatenate([dr, np.zeros((nvert, w, 3))], axis=1)
        nbs.append(nb)
        drs.append(dr)
    neighbours = np.stack(nbs, axis=1)[None] + 1            # [1, Nv, Nhemi, maxNb], 1-based
    dr = np.stack(drs, axis=1)[None]                          # [1, Nv, Nhemi, maxNb, 3]
    edge = np.sqrt(np.sum(dr ** 2, axis=4))
    edge[edge == 0] = EDGE_LENGTH_SENTINEL
    return neighbours, dr, edge
