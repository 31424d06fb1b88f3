"""Layout helpers between MATLAB-style N-D images and the engine's SoA layout.

GACELLE works in two layouts (utils/utils.m:157-238): N-D images
``[x, y, z, meas]`` (column-major) and G-D matrices ``[Nmeas, Nvox]`` of the
masked voxels.  The engine's layout is ``[K][Nvox]`` with the voxel index
fastest, which is exactly a C-contiguous numpy array of shape ``(K, Nvox)``,
i.e. the G-D matrix itself.  Mask indices follow MATLAB's ``find(mask)``
(column-major order).
"""
from __future__ import annotations

import numpy as np


def dims3(mask) -> tuple:
    """size(mask, 1:3)."""
    s = tuple(np.shape(mask)) + (1, 1, 1)
    return tuple(int(x) for x in s[:3])


def mask_index(mask) -> np.ndarray:
    """find(mask > 0) as 0-based column-major linear indices."""
    return np.flatnonzero(np.asarray(mask).ravel(order="F") > 0).astype(np.int64)


def reshape_ND2GD(data, mask_idx) -> np.ndarray:
    """utils.reshape_ND2GD (utils/utils.m:157-163): [x,y,z,k...] -> [K, Nvox]."""
    data = np.asarray(data)
    d3 = dims3(data)
    flat = data.reshape((d3[0] * d3[1] * d3[2], -1), order="F")
    return np.ascontiguousarray(flat[mask_idx].T)


def to_GD(data, mask, mask_idx=None) -> np.ndarray:
    """askadam/mcmc input masking (utils/askadam.m:157-158): N-D data is masked
    through reshape_ND2GD; 2-D (G-D) data keeps the columns of the mask."""
    if mask_idx is None:
        mask_idx = mask_index(mask)
    data = np.asarray(data)
    if data.ndim > 2:
        return reshape_ND2GD(data, mask_idx)
    return np.ascontiguousarray(data[:, mask_idx])


def reshape_GD2ND(gd, mask) -> np.ndarray:
    """utils.reshape_ND2image (utils/utils.m:299-315): [K, Nvox] -> image
    [x,y,z,K] with zeros outside the mask ([x,y,z] when K == 1)."""
    gd = np.asarray(gd)
    if gd.ndim == 1:
        gd = gd[None, :]
    d3 = dims3(mask)
    idx = mask_index(mask)
    img = np.zeros((d3[0] * d3[1] * d3[2], gd.shape[0]), dtype=gd.dtype)
    img[idx] = gd.T
    img = img.reshape(d3 + (gd.shape[0],), order="F")
    return img[..., 0] if gd.shape[0] == 1 else img


def param_to_GD(value, mask, mask_idx, nvox) -> np.ndarray:
    """A parameter map (scalar, [1,Nvox] row, or N-D image) as a [Nvox] vector."""
    v = np.asarray(value, dtype=np.float64)
    if v.size == 1:
        return np.full(nvox, float(v.ravel()[0]))
    if v.ndim <= 2 and v.size == nvox:
        return v.ravel(order="F")
    flat = v.reshape(-1, order="F")
    return flat[mask_idx]


def set_nan_inf_zero(data):
    """utils.set_nan_inf_zero (utils/utils.m:347-351)."""
    data = np.array(data, copy=True)
    bad = ~np.isfinite(data)
    data[bad] = 0
    return data, bad


def initialise_x0(dims, model_params, start_point) -> dict:
    """utils.initialise_x0 (utils/utils.m:1586-1592): constant start maps."""
    return {p: np.full(dims, float(v), dtype=np.float32) for p, v in zip(model_params, start_point)}


def _mat_value(v):
    """A value scipy.io.savemat can write as MATLAB would hold it: nested dicts
    become structs, None becomes [] and tuples of numbers arrays."""
    if isinstance(v, dict):
        return {k: _mat_value(x) for k, x in v.items()}
    if v is None:
        return np.zeros((0, 0))
    if isinstance(v, (list, tuple)) and all(isinstance(x, str) for x in v):
        return np.array(v, dtype=object)
    return v


def save_output(filename, out):
    """askadam.save_askadam_output / mcmc.save_mcmc_output
    (utils/askadam.m:993-1009, utils/mcmc.m:702-718): with a non-empty file
    name, create its folder and save the output structure as the variable
    ``out`` of a MAT-file (MATLAB's level-5 format).  Returns whether a file
    was written."""
    if filename is None or (not isinstance(filename, str) and np.size(filename) == 0) or filename == "":
        return False
    import os

    import scipy.io
    folder = os.path.dirname(str(filename))
    if folder and not os.path.isdir(folder):
        os.makedirs(folder)
    scipy.io.savemat(str(filename), {"out": _mat_value(out)}, do_compression=True)
    print(f"Estimation output is saved at {filename}")
    return True
