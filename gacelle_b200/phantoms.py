"""Seeded synthetic phantoms for the benchmark workloads and tests.

No public dataset is involved: every input is generated here from a fixed
seed with the shapes, protocols and parameter distributions of the workloads
(mono-exponential R2*, joint R1-R2* vFA multi-echo GRE, NEXI), the way the
reference's noise-propagation demos simulate ground truth, forward-model it
and add noise (R2star/demo_gpuR2starMapping_NoisePropagation.m,
NEXI/demo_gpuNEXI_NoisePropagation.m).  Signals are computed in float64 with
the closed-form model equations and rounded to float32 once.
"""
from __future__ import annotations

import numpy as np

R2S_TE = np.arange(2.0, 40.5 + 1e-9, 3.5) * 1e-3           # 12 echoes, 2:3.5:40.5 ms, in s
R1R2S_TE = np.linspace(2.0, 40.0, 12) * 1e-3               # 12 echoes, 2-40 ms, in s
R1R2S_FA = np.array([5.0, 20.0])                           # deg
R1R2S_TR = 30e-3                                           # s
NEXI_B = np.array([1.0, 2.5, 4.0, 6.0, 8.0, 10.0])         # ms/um^2
NEXI_DELTA = np.array([20.0, 27.0, 35.0, 49.0])            # ms
NEXI_SMALL_DELTA = 4.5                                     # ms (narrow-pulse model: unused)
C3_NVOX = (50_000, 110_000, 170_000, 230_000, 300_000, 400_000)


def ellipsoid_mask(dims=(128, 128, 64), scale=1.05) -> np.ndarray:
    """Voxel-centred ellipsoid with semi-axes dims/2 scaled by `scale`
    (128x128x64 -> 629,432 voxels, 60.03%)."""
    c = [np.arange(n) - (n - 1) / 2.0 for n in dims]
    X, Y, Z = np.meshgrid(*c, indexing="ij")
    return (X / (dims[0] / 2)) ** 2 + (Y / (dims[1] / 2)) ** 2 + (Z / (dims[2] / 2)) ** 2 <= scale ** 2


def r2s_signal(M0, R2s, te):
    return M0[..., None] * np.exp(-np.asarray(te) * R2s[..., None])


def r2s_phantom(mask: np.ndarray, seed: int, sigma=0.01, te=R2S_TE, s0=(0.5, 1.5), r2=(10.0, 60.0)):
    """Mono-exponential phantom on `mask`: S0~U(s0), R2*~U(r2) [1/s], Gaussian
    noise sigma.  Returns (data [x,y,z,nte] float32, gt dict of maps)."""
    rng = np.random.default_rng(seed)
    shape = mask.shape
    M0 = rng.uniform(*s0, size=shape) * mask
    R2 = rng.uniform(*r2, size=shape) * mask
    y = r2s_signal(M0, R2, te) + sigma * rng.standard_normal(shape + (len(te),))
    return y.astype(np.float32), {"M0": M0, "R2star": R2}


def r1r2s_signal(M0, R1, R2s, te=R1R2S_TE, fa_deg=R1R2S_FA, tr=R1R2S_TR, b1=1.0):
    a = np.deg2rad(np.asarray(fa_deg))[None, :] * np.asarray(b1).reshape(-1, 1)
    E1 = np.exp(-tr * R1)[:, None]
    A = M0[:, None] * np.sin(a) * (1 - E1) / (1 - np.cos(a) * E1)          # [v, fa]
    E2 = np.exp(-np.asarray(te)[None, :] * R2s[:, None])                    # [v, te]
    return (A[:, None, :] * E2[:, :, None]).reshape(len(M0), -1, order="F")  # TE fastest


def r1r2s_volume(nvox: int, seed: int, sigma=0.01):
    """One masked volume (1-D) of the joint R1-R2* workload: GD data [24, nvox]."""
    rng = np.random.default_rng(seed)
    M0 = rng.uniform(0.5, 2.0, nvox)
    R1 = rng.uniform(0.4, 1.5, nvox)
    R2 = rng.uniform(10.0, 60.0, nvox)
    s = r1r2s_signal(M0, R1, R2)
    y = s + sigma * rng.standard_normal(s.shape)
    return np.ascontiguousarray(y.T.astype(np.float32)), {"M0": M0, "R1": R1, "R2star": R2}


def nexi_shells():
    """24 shells in the order of the gpuNEXI constructor (Delta, then b)."""
    b = np.tile(NEXI_B, len(NEXI_DELTA))
    d = np.repeat(NEXI_DELTA, len(NEXI_B))
    return b, d


def nexi_signal(fa, Da, De, ra, b, delta, nx=100, chunk=8192):
    """float64 NEXI Sl0 (narrow pulse) by an nx-node trapezoid; [v, shell]."""
    if len(fa) > chunk:
        return np.concatenate([nexi_signal(fa[i:i + chunk], Da[i:i + chunk], De[i:i + chunk], ra[i:i + chunk],
                                           b, delta, nx, chunk) for i in range(0, len(fa), chunk)])
    fa = np.maximum(fa, 1e-8)[:, None, None]
    bb = np.asarray(b)[None, :, None]
    dd = np.asarray(delta)[None, :, None]
    x = np.linspace(0, 1, nx)[None, None, :]
    Dai = bb * Da[:, None, None]
    Dej = bb * De[:, None, None]
    r1 = dd * ra[:, None, None]
    r2 = r1 * fa / (1 - fa)
    d1 = Dai * x ** 2
    l1 = (r1 + r2 + d1 + Dej) / 2
    l2 = np.maximum(np.sqrt((r1 - r2 + d1 - Dej) ** 2 + 4 * r1 * r2) / 2, 1e-8)
    lm = l1 - l2
    Pp = (fa * d1 + (1 - fa) * Dej - lm) / (2 * l2)
    M = Pp * np.exp(-(l1 + l2)) + (1 - Pp) * np.exp(-lm)
    S = np.trapezoid(M, x[0, 0], axis=-1)
    return np.minimum(S, 1.0)


def nexi_volume(nvox: int, seed: int, sigma=0.02, rician=True, nx=100):
    """NEXI workload: f~U(0.1,0.9), Da~U(1,3), De~U(0.5,1.5), tex~U(2,50) ms,
    ra = (1-f)/tex (tex redrawn until ra >= 1/250, the contract bound);
    y = |S + sigma (n1 + i n2)| (Rician) or S + sigma n (Gaussian)."""
    rng = np.random.default_rng(seed)
    fa = rng.uniform(0.1, 0.9, nvox)
    Da = rng.uniform(1.0, 3.0, nvox)
    De = rng.uniform(0.5, 1.5, nvox)
    tex = rng.uniform(2.0, 50.0, nvox)
    ra = (1 - fa) / tex
    bad = ra < 1 / 250
    while bad.any():
        tex[bad] = rng.uniform(2.0, 50.0, bad.sum())
        ra = (1 - fa) / tex
        bad = ra < 1 / 250
    b, d = nexi_shells()
    S = nexi_signal(fa, Da, De, ra, b, d, nx)
    n1 = rng.standard_normal(S.shape)
    if rician:
        n2 = rng.standard_normal(S.shape)
        y = np.sqrt((S + sigma * n1) ** 2 + (sigma * n2) ** 2)
    else:
        y = S + sigma * n1
    return np.ascontiguousarray(y.T.astype(np.float32)), {"fa": fa, "Da": Da, "De": De, "ra": ra}


def r2s_tv_volume(seed: int = 1002, dims=(128, 128, 64)):
    """The mono-exponential + 3-D TV workload: ellipsoid mask (629,432 voxels
    on 128x128x64), 12 echoes, seeded phantom; masked data [12, nvox], grid
    indices, and the start (M0, R2*) = (1, 30) of every voxel."""
    from . import utils
    mask = ellipsoid_mask(tuple(dims), 1.05)
    data, gt = r2s_phantom(mask, seed)
    idx = utils.mask_index(mask)
    y = utils.reshape_ND2GD(data, idx)
    th0 = np.tile(np.array([[1.0], [30.0]], np.float32), (1, y.shape[1]))
    return {"mask": mask, "y": y, "idx": idx.astype(np.int32), "th0": th0, "nvox": y.shape[1], "gt": gt}
