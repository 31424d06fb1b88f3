"""Second, independent restatement of the reference formulas in torch float64.

TEST INFRASTRUCTURE ONLY.  It follows the MATLAB code's vectorised form line
by line (broadcast over [meas, voxel, node]) so that it shares no code with
the C oracle; autograd of these functions checks the oracle's hand-written
adjoints.  Arrays are [k, nvox] (parameter or measurement index first).
"""
from __future__ import annotations

import math

import torch

EPS = 1e-8  # askadam.epsilon (utils/askadam.m:14)


def r2s_fwd(theta, te):
    """R2star/gpuR2starMapping.m:427-434: m0 .* exp(-te .* r2s)."""
    M0, R2s = theta[0], theta[1]
    te = torch.as_tensor(te, dtype=theta.dtype)[:, None]
    return M0[None, :] * torch.exp(-te * R2s[None, :])


def r1r2s_fwd(theta, te, fa_deg, tr, b1=None):
    """R1R2s/gpuJointR1R2starMapping.m:383-417,513-525 (TE dim 4, FA dim 5)."""
    M0, R1, R2s = theta[0], theta[1], theta[2]
    te = torch.as_tensor(te, dtype=theta.dtype)
    fa = torch.as_tensor(fa_deg, dtype=theta.dtype) * math.pi / 180.0
    nv = theta.shape[1]
    b1 = torch.ones(nv, dtype=theta.dtype) if b1 is None else torch.as_tensor(b1, dtype=theta.dtype)
    a = b1[None, None, :] * fa[:, None, None]                       # [fa, 1, v]
    E1 = torch.exp(-tr * R1)[None, None, :]
    s = (M0[None, None, :] * torch.sin(a) * (1 - E1) / (1 - torch.cos(a) * E1)
         * torch.exp(-te[None, :, None] * R2s[None, None, :]))      # [fa, te, v]
    return s.reshape(len(fa) * len(te), nv)                          # TE fastest


def nexi_fwd(theta, bval, delta, lmax=0, nx=14):
    """NEXI/gpuNEXI.m:902-996 (Slmax2) with M from :1090-1097, trapz from
    utils/gacelle_trapz.m and the final min(s,1)."""
    fa = torch.clamp(theta[0], min=EPS)
    Da, De, ra = theta[1], theta[2], theta[3]
    b = torch.as_tensor(bval, dtype=theta.dtype)[:, None, None]
    D = torch.as_tensor(delta, dtype=theta.dtype)[:, None, None]
    Da = b * Da[None, :, None]
    De = b * De[None, :, None]
    r1 = D * ra[None, :, None]
    r2 = r1 * fa[None, :, None] / (1 - fa[None, :, None])
    x = torch.linspace(0, 1, nx, dtype=theta.dtype)[None, None, :]
    f = fa[None, :, None]
    d1 = Da * x ** 2
    l1 = (r1 + r2 + d1 + De) / 2
    l2 = torch.sqrt((r1 - r2 + d1 - De) ** 2 + 4 * r1 * r2) / 2
    l2 = torch.clamp(l2, min=EPS)
    lm = l1 - l2
    Pp = (f * d1 + (1 - f) * De - lm) / (l2 * 2)
    M = Pp * torch.exp(-(l1 + l2)) + (1 - Pp) * torch.exp(-lm)
    w = x[..., 1:] - x[..., :-1]
    S = torch.sum((M[..., :-1] + M[..., 1:]) * (w / 2), dim=-1)      # [shell, v]
    if lmax == 2:
        M2 = M * (3 * x ** 2 - 1) / 2
        Sl2 = torch.sum((M2[..., :-1] + M2[..., 1:]) * (w / 2), dim=-1)
        S = torch.cat([S, theta[4][None, :] * torch.abs(Sl2)], dim=0)
    return torch.clamp(S, max=1.0)


def _besseli_trapz(nu, z, nx=34):
    """mybesseli (NEXI/gpuNEXIrice.m:751-755): (1/pi) trapz over t in
    linspace(0, pi, nx) of exp(z cos t) cos(nu t)."""
    t = torch.linspace(0, math.pi, nx, dtype=z.dtype)
    f = torch.exp(z[..., None] * torch.cos(t)) * torch.cos(nu * t)
    h = t[1] - t[0]
    return (torch.sum(f, dim=-1) - 0.5 * (f[..., 0] + f[..., -1])) * h / math.pi


def rice_mean(nu, sigma):
    """myriceM1 / myL12 (NEXI/gpuNEXIrice.m:726-744): max(sigma sqrt(pi/2)
    L12(-nu^2/(2 sigma^2)), nu) with x clamped at -170."""
    x = torch.clamp(-nu ** 2 / (2 * sigma ** 2), min=-170.0)
    L = torch.exp(x / 2) * ((1 - x) * _besseli_trapz(0, -x / 2) - x * _besseli_trapz(1, -x / 2))
    return torch.maximum(sigma * math.sqrt(math.pi / 2) * L, nu)


def nexi_rice_fwd(theta, bval, delta, sigma, nx=14):
    """gpuNEXIrice.FWD (NEXI/gpuNEXIrice.m:635-688): fa = max(fa, eps),
    re = ra fa / max(1 - fa, eps), Sl0, Rician mean, min(s, 1)."""
    fa = torch.clamp(theta[0], min=EPS)
    Da, De, ra = theta[1], theta[2], theta[3]
    b = torch.as_tensor(bval, dtype=theta.dtype)[:, None, None]
    D = torch.as_tensor(delta, dtype=theta.dtype)[:, None, None]
    f = fa[None, :, None]
    r1 = D * ra[None, :, None]
    r2 = r1 * f / torch.clamp(1 - f, min=EPS)
    d2 = b * De[None, :, None]
    x = torch.linspace(0, 1, nx, dtype=theta.dtype)[None, None, :]
    d1 = b * Da[None, :, None] * x ** 2
    l1 = (r1 + r2 + d1 + d2) / 2
    l2 = torch.clamp(torch.sqrt((r1 - r2 + d1 - d2) ** 2 + 4 * r1 * r2) / 2, min=EPS)
    lm = l1 - l2
    Pp = (f * d1 + (1 - f) * d2 - lm) / (l2 * 2)
    M = Pp * torch.exp(-(l1 + l2)) + (1 - Pp) * torch.exp(-lm)
    w = x[..., 1:] - x[..., :-1]
    S = torch.sum((M[..., :-1] + M[..., 1:]) * (w / 2), dim=-1)      # [shell, v]
    sig = torch.as_tensor(sigma, dtype=theta.dtype)
    return torch.clamp(rice_mean(S, sig[None, :] if sig.ndim else sig), max=1.0)


def loss_elem(kind, s, y, w=None, sigma=1.0, mse_scale=0.5, huber_delta=1.0):
    """utils/askadam.m:86-95 elementwise losses, plus Gaussian/Rician NLL."""
    r = s - y
    w = torch.ones_like(s) if w is None else w
    if kind == "l1":
        return w * torch.abs(r)
    if kind == "l2":
        return w * r ** 2
    if kind == "huber":
        a = torch.abs(r)
        return w * torch.where(a <= huber_delta, 0.5 * r ** 2, huber_delta * a - 0.5 * huber_delta ** 2)
    if kind == "mse":
        return mse_scale * r ** 2
    if kind == "gauss":
        s2 = sigma ** 2
        return w * (r ** 2 / (2 * s2) + 0.5 * torch.log(2 * math.pi * s2 * torch.ones_like(s)))
    if kind == "rician":
        s2 = sigma ** 2
        x = y * s / s2
        logI0 = torch.abs(x) + torch.log(torch.special.i0e(x))
        c = torch.where(y > 0, -torch.log(torch.clamp(y, min=1e-300) / s2), torch.zeros_like(y))
        return w * ((y ** 2 + s ** 2) / (2 * s2) - logI0 + c)
    raise ValueError(kind)


def tv_cost(img, mask, tv_3d=True, voxel_size=(2.0, 2.0, 2.0)):
    """utils/spatial_total_variation.m:45-66: circshift forward differences."""
    G = [(torch.roll(img, -1, 0) - img) / voxel_size[0], (torch.roll(img, -1, 1) - img) / voxel_size[1]]
    if tv_3d:
        G.append((torch.roll(img, -1, 2) - img) / voxel_size[2])
    cost = sum(torch.abs(mask * g) for g in G)
    return torch.sum(torch.abs(cost))
