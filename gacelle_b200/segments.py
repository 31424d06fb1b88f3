"""Slab segmentation of a volume and its fit across ranks.

The reference divides volumes that exceed GPU memory into z-slabs
(utils/utils.m:592-836 find_optimal_segment_3D, :868-937
build_balanced_boundaries, :939-979 expand_segments_with_halo) and fits each
slab independently: "owned" slice ranges partition the volume with about equal
voxel counts, internal faces get ``segmentOverlap`` halo slices so that a 3-D
TV regulariser sees its neighbours, and only the owned slices of each fit are
written back (restore_segment_structure, :1348-1470).

On the B200 engine a whole volume fits one GPU, so the same segmentation is
used to spread one volume over ranks: rank r fits segment r on its own GPU and
the owned slices are all-gathered.  No collective enters the fit itself (the
slabs are independent, exactly as in the reference's segmented run), so this
is weak scaling over slabs; the result equals the reference's segmented fit
with the same boundaries, which "may not be exactly the same as 1 segment"
(utils/utils.m:798) when TV couples the slabs.
"""
from __future__ import annotations

import math
from typing import Callable

import numpy as np


def build_balanced_boundaries(mask, nvox_per_seg: int, nseg_min: int = 1) -> list[np.ndarray]:
    """utils.build_balanced_boundaries (utils/utils.m:868-937): contiguous
    owned slice ranges (0-based) with about equal masked-voxel counts, each at
    most ``nvox_per_seg`` where possible, at least ``nseg_min`` of them."""
    mask = np.asarray(mask) > 0
    density = mask.reshape(mask.shape[0] * mask.shape[1], -1, order="F").sum(axis=0)
    dims3 = density.size
    total = int(density.sum())
    nseg = max(math.ceil(total / max(nvox_per_seg, 1)), nseg_min)
    target = total / nseg
    cum = np.cumsum(density)
    bounds, start = [], 0
    for ks in range(1, nseg + 1):
        if ks < nseg:
            t = ks * target
            below = np.flatnonzero(cum < t)
            above = np.flatnonzero(cum >= t)
            if below.size == 0:
                end = start
            elif above.size == 0:
                end = dims3 - 1
            else:
                b, a = below[-1], above[0]
                vb = cum[b] - (ks - 1) * target
                va = cum[a] - (ks - 1) * target
                end = b if abs(vb - target) <= abs(va - target) else a
            end = max(end, start)
        else:
            end = dims3 - 1
        bounds.append(np.arange(start, end + 1))
        start = end + 1
    return [b for b in bounds if b.size]


def expand_segments_with_halo(owned: list[np.ndarray], h: int, dims3: int) -> list[dict]:
    """utils.expand_segments_with_halo (utils/utils.m:939-979): per segment the
    owned slices, the fitted slices (owned plus ``h`` halo slices on internal
    faces, clamped to the volume) and the owned slices' positions in the fit."""
    n = len(owned)
    seg = []
    for ks, own in enumerate(owned):
        lo = h if ks > 0 else 0
        hi = h if ks < n - 1 else 0
        fit = np.arange(max(0, own[0] - lo), min(dims3 - 1, own[-1] + hi) + 1)
        seg.append({"owned": own, "fit": fit, "local": own - fit[0]})
    return seg


def rank_segments(mask, world: int, overlap: int = 0) -> list[dict]:
    """``world`` segments of about equal voxel counts (NSegmentUser = world,
    segmentOverlap = overlap, utils/utils.m:817-826)."""
    mask = np.asarray(mask) > 0
    owned = build_balanced_boundaries(mask, math.ceil(int(mask.sum()) / world), world)
    return expand_segments_with_halo(owned, overlap, mask.shape[2] if mask.ndim >= 3 else 1)


def _slab(a, sl):
    a = np.asarray(a)
    return a[:, :, sl, ...] if a.ndim >= 3 else a


def restore_segments(parts: list[dict], segs: list[dict], shape3) -> dict:
    """restore_segment_structure / restore_field (utils/utils.m:1348-1484)
    over whole segments: arrays whose third dimension spans a segment's
    fitted slices contribute their owned slices at the owned positions;
    scalars become one value per segment; voxel-indexed matrices [Nm, Nv]
    (second dimension above 1) are concatenated along voxels, vectors along
    their length and 3-D arrays with equal trailing dimensions along the
    first; anything else is kept from the first segment."""
    def merge(vals, path):
        first = vals[0]
        if isinstance(first, dict):
            return {k: merge([v[k] for v in vals], path + (k,)) for k in first}
        if isinstance(first, (str, bytes, bool, np.bool_)):
            return first  # character / logical scalars: kept from the first segment
        if np.isscalar(first) or (isinstance(first, np.ndarray) and first.ndim == 0):
            return np.array([float(v) for v in vals])
        if isinstance(first, np.ndarray) and first.ndim >= 3 and all(
                v.shape[2] == s["fit"].size for v, s in zip(vals, segs)):
            out = np.zeros(tuple(shape3[:2]) + (shape3[2],) + first.shape[3:], dtype=first.dtype)
            for v, s in zip(vals, segs):
                out[:, :, s["owned"], ...] = v[:, :, s["local"], ...]
            return out
        if isinstance(first, np.ndarray) and len(vals) > 1:
            if first.ndim == 2 and first.shape[1] > 1 and all(v.ndim == 2 for v in vals):
                return np.concatenate(vals, axis=1)
            if first.ndim == 1 or (first.ndim == 2 and first.shape[1] == 1):
                return np.concatenate([np.asarray(v).reshape(-1, *first.shape[1:]) for v in vals], axis=0)
            if first.ndim == 3 and all(v.shape[1:] == first.shape[1:] for v in vals):
                return np.concatenate(vals, axis=0)
        return first
    return merge(parts, ())


def slice_extradata_recursive(extradata, sl):
    """gpuNEXI.slice_extradata_recursive (NEXI/gpuNEXI.m:884-897): arrays of
    three or more dimensions are cut to the slices ``sl``, nested dicts (e.g.
    the prior's mu / sigma maps) recursively, anything else is passed on."""
    if extradata is None:
        return None
    out = {}
    for k, v in extradata.items():
        if isinstance(v, dict):
            out[k] = slice_extradata_recursive(v, sl)
        elif np.ndim(v) >= 3:
            out[k] = _slab(v, sl)
        else:
            out[k] = v
    return out


def fit_segmented(fit: Callable, data, mask, nseg: int, overlap: int = 0, extradata: dict | None = None,
                  pars0: dict | None = None) -> dict:
    """The segment loop of the models' estimate() (e.g.
    R2star/gpuR2starMapping.m:128-157, NEXI/gpuNEXI.m:209-236) on one GPU:
    ``nseg`` slabs of about equal voxel counts (fitting.NSegmentUser; the
    engine needs no memory-driven split), each fitted independently with
    ``overlap`` halo slices (fitting.segmentOverlap), cropped to its owned
    slices and written back (crop_segment_output,
    restore_segment_structure).  ``fit(data_slab, mask_slab, extradata_slab,
    pars0_slab) -> out``."""
    mask = np.asarray(mask)
    shape3 = mask.shape + (1,) * (3 - mask.ndim)
    m3 = mask.reshape(shape3, order="F")
    segs = rank_segments(m3, max(int(nseg), 1), int(overlap))
    parts = []
    for s in segs:
        p0 = None if pars0 is None else {k: _slab(v, s["fit"]) if np.ndim(v) >= 3 else v for k, v in pars0.items()}
        parts.append(fit(_slab(np.asarray(data), s["fit"]), _slab(m3, s["fit"]),
                         slice_extradata_recursive(extradata, s["fit"]), p0))
    return restore_segments(parts, segs, shape3)


def fit_distributed(fit: Callable, data, mask, extradata: dict | None = None, pars0: dict | None = None,
                    overlap: int = 0, group=None) -> dict:
    """Fit one volume split into one slab per rank.

    ``fit(data_slab, mask_slab, extradata_slab, pars0_slab) -> out`` runs on
    this rank (e.g. ``lambda d, m, e, p: model.fit(d, m, fitting, ...)`` with
    the rank's GPU selected).  The owned slices of every rank's result are
    all-gathered through ``torch.distributed`` (any backend; no process group
    or a world of 1 runs the whole volume here) and the assembled output is
    returned on every rank.
    """
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    mask = np.asarray(mask)
    shape3 = mask.shape + (1,) * (3 - mask.ndim)
    segs = rank_segments(mask.reshape(shape3, order="F"), world, overlap)
    if len(segs) < world:
        raise ValueError(f"{world} ranks but only {len(segs)} non-empty slabs")
    s = segs[rank]
    sub = lambda a: None if a is None else (_slab(a, s["fit"]) if np.ndim(a) >= 3 else a)  # noqa: E731
    ex = slice_extradata_recursive(extradata, s["fit"])
    p0 = None if pars0 is None else {k: sub(v) for k, v in pars0.items()}
    mine = fit(_slab(np.asarray(data), s["fit"]), _slab(mask.reshape(shape3, order="F"), s["fit"]), ex, p0)
    if world == 1:
        return restore_segments([mine], segs, shape3)
    parts = [None] * world
    dist.all_gather_object(parts, mine, group=group)
    return restore_segments(parts, segs, shape3)
