"""Diffusion-MRI input preparation: shell bookkeeping and rotationally
invariant signals (utils/DWIutility.m), the step that turns a full DWI
acquisition ``[x, y, z, volumes]`` into the per-shell signal the NEXI models
fit.

The invariant of order l of one shell is the norm of the shell's signal
projected on the degree-l spherical harmonics:

    S_l = || f_l || / sqrt(4 pi (2 l + 1)),

with ``f_lm`` the least-squares real-SH coefficients (up to ``lmax``) of the
shell's samples, each direction doubled by its antipode because a diffusion
signal is even (utils/DWIutility.m:402-417; the toolbox it calls is
utils/Spherical-Harmonic-Transform/leastSquaresSHT.m and getSH.m).  ``S_0``
is the spherical mean.  The norm over m does not depend on which orthonormal
real basis spans degree l, so the basis here is built from its own
associated-Legendre recursion.

Everything is numpy on the host, in the input's float type (float32 stays
float32, as MATLAB keeps single data single): a one-off pass over the input,
not part of the iterated fit.  Images follow MATLAB's column-major voxel
order.
"""
from __future__ import annotations

import math

import numpy as np


def _as_vec(v, n, empty_value):
    """Broadcast an acquisition parameter to one value per volume: ``None``
    or empty gives ``empty_value``, a scalar is repeated."""
    if v is None:
        return np.full(n, float(empty_value))
    a = np.asarray(v, dtype=np.float64).ravel()
    if a.size == 0:
        return np.full(n, float(empty_value))
    if a.size == 1:
        return np.full(n, float(a[0]))
    return a


def _vox_by_vol(dwi):
    """[x, y, z, vol] -> ([Nvox, vol] in column-major voxel order, dims); a
    float32 or float64 input keeps its type (MATLAB computes in the input's
    class), anything else becomes float64."""
    dwi = np.asarray(dwi)
    if dwi.dtype not in (np.float32, np.float64):
        dwi = dwi.astype(np.float64)
    if dwi.ndim < 4:
        dwi = dwi.reshape(dwi.shape + (1,) * (4 - dwi.ndim))
    dims = dwi.shape[:3]
    return dwi.reshape((-1, dwi.shape[3]), order="F"), dims


def _image(flat, dims):
    """[Nvox, K] -> [x, y, z, K] (column-major voxel order)."""
    return flat.reshape(tuple(dims) + (flat.shape[1],), order="F")


def _legendre_nocs(n, x):
    """Associated Legendre functions P_n^m(x), m = 0..n, WITHOUT the
    Condon-Shortley phase (getSH.m cancels it for the real basis), from the
    standard three-term recursion in degree at fixed order."""
    x = np.asarray(x, dtype=np.float64)
    s = np.sqrt(np.maximum(1.0 - x * x, 0.0))
    out = np.zeros((n + 1,) + x.shape)
    pmm = np.ones_like(x)
    for m in range(n + 1):
        if m > 0:
            pmm = pmm * (2 * m - 1) * s          # P_m^m = (2m-1)!! s^m
        if m == n:
            out[m] = pmm
            continue
        p_prev, p = pmm, x * (2 * m + 1) * pmm  # P_{m+1}^m
        for l in range(m + 2, n + 1):
            p_prev, p = p, ((2 * l - 1) * x * p - (l + m - 1) * p_prev) / (l - m)
        out[m] = p
    return out


class DWIutility:
    """Host mirror of utils/DWIutility.m for the functions the NEXI models'
    data preparation calls."""

    # ------------------------------------------------------------ shells
    @staticmethod
    def unique_shell(bval, ldelta, BDELTA):
        """utils/DWIutility.m:498-529: non-zero b-values, unique per little
        delta (ascending), then big delta (ascending), then b (ascending)."""
        bval = np.asarray(bval, dtype=np.float64).ravel()
        ld = _as_vec(ldelta, bval.size, 0.0)
        bd = _as_vec(BDELTA, bval.size, 0.0)
        bs, lds, bds = [], [], []
        for lv in np.unique(ld):
            il = ld == lv
            for dv in np.unique(bd[il]):
                bu = np.unique(bval[il & (bd == dv)])
                bu = bu[bu > 0]
                bs += list(bu)
                lds += [lv] * bu.size
                bds += [dv] * bu.size
        return np.array(bs), np.array(lds), np.array(bds)

    @staticmethod
    def unique_shell_keepb0(bval, ldelta=None, BDELTA=None, te=None, discardB0=False):
        """utils/DWIutility.m:647-775: shells ordered TE -> little delta ->
        big delta -> b; b = 0 kept once per TE (at the smallest little delta,
        then smallest big delta of that TE) unless ``discardB0`` and the
        protocol has a single TE.  Empty ``te`` means one TE; empty deltas
        mean 0."""
        bval = np.asarray(bval, dtype=np.float64).ravel()
        n = bval.size
        te = _as_vec(te, n, 1.0)
        ld = _as_vec(ldelta, n, 0.0)
        bd = _as_vec(BDELTA, n, 0.0)
        te_u = np.unique(te)
        multi = te_u.size > 1
        out = [[], [], [], []]

        def add(b, l, d, t):
            out[0].append(b), out[1].append(l), out[2].append(d), out[3].append(t)

        for tv in te_u:
            it = te == tv
            if np.any(bval[it] == 0) and not (discardB0 and not multi):
                ld1 = ld[it].min()
                add(0.0, ld1, bd[it & (ld == ld1)].min(), tv)
            for lv in np.unique(ld[it]):
                il = it & (ld == lv)
                for dv in np.unique(bd[il]):
                    bu = np.unique(bval[il & (bd == dv)])
                    for b in bu[bu > 0]:
                        add(b, lv, dv, tv)
        return tuple(np.array(o, dtype=np.float64) for o in out)

    # ------------------------------------------------------------ SH
    @staticmethod
    def cart2sph_incl(g):
        """utils/DWIutility.m:491-495: [azimuth, inclination] per direction
        (MATLAB cart2sph, inclination = pi/2 - elevation).  A zero vector
        maps to azimuth 0, inclination pi/2."""
        g = np.asarray(g, dtype=np.float64)
        azi = np.arctan2(g[:, 1], g[:, 0])
        elev = np.arctan2(g[:, 2], np.hypot(g[:, 0], g[:, 1]))
        return np.stack([azi, np.pi / 2 - elev], axis=1)

    @staticmethod
    def getSH(N, dirs):
        """Orthonormal real spherical harmonics up to degree N at
        ``dirs`` = [azimuth, inclination] (K x 2) as a K x (N+1)^2 matrix;
        columns per degree n in order m = -n..n, sin(|m| phi) for m < 0,
        cos(m phi) for m > 0, the layout of
        utils/Spherical-Harmonic-Transform/getSH.m ('real')."""
        dirs = np.asarray(dirs, dtype=np.float64)
        phi, ct = dirs[:, 0], np.cos(dirs[:, 1])
        Y = np.zeros((dirs.shape[0], (N + 1) ** 2))
        col = 0
        for n in range(N + 1):
            P = _legendre_nocs(n, ct)
            for m in range(-n, n + 1):
                am = abs(m)
                norm = math.sqrt((2 * n + 1) / (4 * math.pi)
                                 * math.factorial(n - am) / math.factorial(n + am))
                if m == 0:
                    Y[:, col] = norm * P[0]
                elif m > 0:
                    Y[:, col] = math.sqrt(2) * norm * P[am] * np.cos(am * phi)
                else:
                    Y[:, col] = math.sqrt(2) * norm * P[am] * np.sin(am * phi)
                col += 1
        return Y

    def SHrotinv(self, S, g, lmax):
        """utils/DWIutility.m:402-417: S is [Ndir, Nvox] (one shell), g the
        [Ndir, 3] directions; returns [lmax/2+1, Nvox] invariants S_0, S_2, ...
        The least-squares fit is the pseudo-inverse (leastSquaresSHT.m:33,
        unweighted) of the basis up to ``lmax`` at the doubled directions."""
        S = np.asarray(S)
        if S.dtype not in (np.float32, np.float64):
            S = S.astype(np.float64)
        g = np.asarray(g, dtype=np.float64)
        n = g.shape[0]
        g2 = np.concatenate([g, -g], axis=0)
        Y = self.getSH(int(lmax), self.cart2sph_incl(g2))
        P = np.linalg.pinv(Y)
        # the samples are doubled ([S; S]), so P [S; S] = (P[:, :n] + P[:, n:]) S
        F = (P[:, :n] + P[:, n:]).astype(S.dtype) @ S
        out = np.zeros((int(lmax) // 2 + 1, S.shape[1]), dtype=S.dtype)
        for l in range(0, int(lmax) + 1, 2):
            out[l // 2] = np.sqrt(np.sum(F[l * l:(l + 1) ** 2] ** 2, axis=0)) / math.sqrt(4 * math.pi * (2 * l + 1))
        return out

    @staticmethod
    def _bvec_rows(bvec):
        """bvec as [Nvol, 3]: a 3-row input is transposed, as the reference
        does (utils/DWIutility.m:322-324)."""
        b = np.asarray(bvec, dtype=np.float64)
        return b.T if b.shape[0] == 3 else b

    # ------------------------------------------------------------ per group
    def Sl(self, dwi, bval, bvec, lmax):
        """utils/DWIutility.m:306-358: invariants of every non-zero shell of
        one acquisition group, normalised by the group's mean b = 0 signal
        (1 when the group has none); [x, y, z, Nshell * (lmax/2+1)] laid out
        as all shells' S_0, then all shells' S_2; also the shells' b."""
        flat, dims = _vox_by_vol(dwi)
        bval = np.asarray(bval, dtype=np.float64).ravel()
        g = self._bvec_rows(bvec)
        b0 = bval == 0
        dwi_b0 = flat[:, b0].mean(axis=1) if b0.any() else np.ones(flat.shape[0])
        bu = np.unique(bval)
        bu = bu[bu != 0]
        nsh = int(lmax) // 2 + 1
        out = np.zeros((flat.shape[0], nsh * bu.size), dtype=flat.dtype)
        with np.errstate(divide="ignore", invalid="ignore"):
            for k, b in enumerate(bu):
                ind = bval == b
                F = self.SHrotinv((flat[:, ind] / dwi_b0[:, None]).T, g[ind], lmax)
                out[:, k::bu.size] = F.T
        return _image(out, dims), bu

    def Sl_no_normalise(self, dwi, bval, bvec, lmax):
        """utils/DWIutility.m:361-400: as :meth:`Sl` without normalisation,
        one entry per unique b (b = 0 included if present)."""
        flat, dims = _vox_by_vol(dwi)
        bval = np.asarray(bval, dtype=np.float64).ravel()
        g = self._bvec_rows(bvec)
        bu = np.unique(bval)
        nsh = int(lmax) // 2 + 1
        out = np.zeros((flat.shape[0], nsh * bu.size), dtype=flat.dtype)
        for k, b in enumerate(bu):
            ind = bval == b
            out[:, k::bu.size] = self.SHrotinv(flat[:, ind].T, g[ind], lmax).T
        return _image(out, dims), bu

    # ------------------------------------------------------------ all groups
    def get_Sl_all(self, dwi, bval, bvec, ldelta, BDELTA, lmax):
        """utils/DWIutility.m:276-302: :meth:`Sl` per (little delta, big
        delta) group, groups ordered by little delta then big delta
        (ascending); output [x, y, z, Ntotal * (lmax/2+1)] with all groups'
        S_0 first, then all S_2; also the b of each output shell."""
        flat, dims = _vox_by_vol(dwi)
        bval = np.asarray(bval, dtype=np.float64).ravel()
        g = self._bvec_rows(bvec)
        ld = _as_vec(ldelta, bval.size, 0.0)
        bd = _as_vec(BDELTA, bval.size, 0.0)
        nsh = int(lmax) // 2 + 1
        blocks, b_all = [], []
        for lv in np.unique(ld):
            il = ld == lv
            for dv in np.unique(bd[il]):
                idx = np.flatnonzero(il & (bd == dv))
                s, bu = self.Sl(_image(flat[:, idx], dims), bval[idx], g[idx], lmax)
                blocks.append(s.reshape((-1, nsh * bu.size), order="F").reshape((-1, nsh, bu.size)))
                b_all += list(bu)
        return self._stack_blocks(blocks, dims, nsh), np.array(b_all)

    @staticmethod
    def _stack_blocks(blocks, dims, nsh):
        """Concatenate [Nvox, nsh, Nshell_g] blocks along shells and lay the
        result out as [x, y, z, Nshell * nsh], degree-major."""
        if not blocks:
            return np.zeros(tuple(dims) + (0,))
        allb = np.concatenate(blocks, axis=2)
        return _image(allb.reshape((allb.shape[0], -1)), dims)

    def get_Sl_all_no_normalise(self, dwi, bval, bvec, ldelta, BDELTA, te, lmax):
        """utils/DWIutility.m:168-273: per TE (ascending), first the mean of
        all that TE's b = 0 volumes (S_0 = mean, higher orders 0), then the
        non-zero shells of each (little delta, big delta) group through
        :meth:`Sl_no_normalise`; output degree-major as in
        :meth:`get_Sl_all`, plus the b of each shell."""
        flat, dims = _vox_by_vol(dwi)
        bval = np.asarray(bval, dtype=np.float64).ravel()
        n = bval.size
        g = self._bvec_rows(bvec)
        te = _as_vec(te, n, 0.0)
        ld = _as_vec(ldelta, n, 0.0)
        bd = _as_vec(BDELTA, n, 0.0)
        nsh = int(lmax) // 2 + 1
        blocks, b_out = [], []
        for tv in np.unique(te):
            it = te == tv
            ib0 = it & (bval == 0)
            if ib0.any():
                blk = np.zeros((flat.shape[0], nsh, 1), dtype=flat.dtype)
                blk[:, 0, 0] = flat[:, ib0].mean(axis=1)
                blocks.append(blk)
                b_out.append(0.0)
            for lv in np.unique(ld[it]):
                il = it & (ld == lv)
                for dv in np.unique(bd[il]):
                    idx = np.flatnonzero(il & (bd == dv) & (bval > 0))
                    if idx.size == 0:
                        continue
                    s, bu = self.Sl_no_normalise(_image(flat[:, idx], dims), bval[idx], g[idx], lmax)
                    blocks.append(s.reshape((-1, nsh * bu.size), order="F").reshape((-1, nsh, bu.size)))
                    b_out += list(bu)
        return self._stack_blocks(blocks, dims, nsh), np.array(b_out)

    def compute_rotationally_invariant_signal(self, dwi, bval, bvec, ldelta=None, BDELTA=None, te=None, lmax=0):
        """utils/DWIutility.m:10-165.  Empty or scalar little delta / big
        delta broadcast (empty = 1), empty TE = 0.  With one TE the output is
        normalised by the first shell's S_0 (the b = 0 mean when the protocol
        has b = 0, floored at 1e-8) and the b = 0 shell is dropped; with
        several TEs nothing is normalised, and b = 0 shells stay in the S_0
        block only.  Returns (dwi_out, bval_out, ldelta_out, BDELTA_out,
        te_out), the descriptors aligned with the last axis of dwi_out."""
        bval = np.asarray(bval, dtype=np.float64).ravel()
        n = bval.size
        ld = _as_vec(ldelta, n, 1.0)
        bd = _as_vec(BDELTA, n, 1.0)
        te = _as_vec(te, n, 0.0)
        lmax = int(lmax)
        nsl = lmax // 2 + 1
        raw, b_loop = self.get_Sl_all_no_normalise(dwi, bval, bvec, ld, bd, te, lmax)
        nshell = b_loop.size
        isb0 = b_loop == 0
        # shell descriptors in the loop order of get_Sl_all_no_normalise
        ld_loop, bd_loop, te_loop = [], [], []
        for tv in np.unique(te):
            it = te == tv
            if np.any(bval[it] == 0):
                ld1 = ld[it].min()
                ld_loop.append(ld1)
                bd_loop.append(bd[it & (ld == ld1)].min())
                te_loop.append(tv)
            for lv in np.unique(ld[it]):
                il = it & (ld == lv)
                for dv in np.unique(bd[il]):
                    bu = np.unique(bval[il & (bd == dv)])
                    k = int(np.sum(bu > 0))
                    ld_loop += [lv] * k
                    bd_loop += [dv] * k
                    te_loop += [tv] * k
        ld_loop, bd_loop, te_loop = (np.array(v, dtype=np.float64) for v in (ld_loop, bd_loop, te_loop))
        nonb0 = np.flatnonzero(~isb0)
        if np.unique(te).size == 1:
            sel = np.concatenate([kl * nshell + nonb0 for kl in range(nsl)])
            norm = np.maximum(raw[..., 0], 1e-8)
            out = raw[..., sel] / norm[..., None]
            desc = [np.tile(v[~isb0], nsl) for v in (b_loop, ld_loop, bd_loop, te_loop)]
        else:
            sel = np.concatenate([np.arange(nshell)] + [kl * nshell + nonb0 for kl in range(1, nsl)])
            out = raw[..., sel]
            desc = [np.concatenate([v] + [v[~isb0]] * (nsl - 1)) for v in (b_loop, ld_loop, bd_loop, te_loop)]
        return (out,) + tuple(desc)
