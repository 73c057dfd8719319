"""Host-side spherical-harmonic set-up for amp2sh (FP64, numpy).

The real, even-order SH basis of MRtrix3 (core/math/SH.h:46-104: index
l(l+1)/2 + m, sqrt(2) cos / sin for m != 0, normalised associated Legendre
functions of core/math/legendre.h:101-123), the amplitude mapping of
DWI::compute_SH2amp_mapping (core/dwi/gradient.h:326-374: lmax from the
direction count, at most 8 unless requested, lowered while the mapping's
condition number is 100 or more) and Math::pinv (least_squares.h:39-45).
"""
from __future__ import annotations

import math

import numpy as np


def n_for_l(lmax: int) -> int:
    return (lmax + 1) * (lmax + 2) // 2


def l_for_n(n: int) -> int:
    """SH::LforN (SH.h:70-73), with its single-precision square root."""
    return 2 * int(math.floor((float(np.sqrt(np.float32(1 + 8 * n))) - 3.0) / 4.0)) if n else 0


def plm_sph(lmax: int, m: int, x: np.ndarray) -> np.ndarray:
    """[lmax+1][n] normalised associated Legendre values of order m at x = cos(el)."""
    x = np.asarray(x, np.float64)
    out = np.zeros((lmax + 1,) + x.shape)
    x2 = x * x
    v = np.full(x.shape, 0.282094791773878)
    if m:
        h = np.ones_like(x)
        mm = 2.0 * m
        while mm >= 1.0:
            h = h * (1.0 - x2) * (mm - 1.0) / mm
            mm -= 2.0
        v = v * np.sqrt((2 * m + 1) * h)
        v = np.where(x2 >= 1.0, 0.0, v)
    if m & 1:
        v = -v
    out[m] = v
    if lmax > m:
        f = math.sqrt(2 * m + 3)
        out[m + 1] = x * f * out[m]
        for n in range(m + 2, lmax + 1):
            out[n] = x * out[n - 1] - out[n - 2] / f
            f = math.sqrt((4 * n * n - 1) / (n * n - m * m))
            out[n] = out[n] * f
    return out


def init_transform(dirs_azel: np.ndarray, lmax: int) -> np.ndarray:
    """SH -> amplitude matrix [ndir][nSH] for [az el] directions (SH.h:82-104)."""
    dirs = np.asarray(dirs_azel, np.float64)
    az, el = dirs[:, 0], dirs[:, 1]
    out = np.zeros((len(dirs), n_for_l(lmax)))
    z = np.cos(el)
    for m in range(lmax + 1):
        P = plm_sph(lmax, m, z)
        for l in range(m + (m & 1), lmax + 1, 2):
            c = l * (l + 1) // 2
            if m == 0:
                out[:, c] = P[l]
            else:
                out[:, c + m] = math.sqrt(2.0) * P[l] * np.cos(m * az)
                out[:, c - m] = math.sqrt(2.0) * P[l] * np.sin(m * az)
    return out


def cartesian_to_azel(xyz: np.ndarray) -> np.ndarray:
    """Math::Sphere::cartesian2spherical: [az el] of each row."""
    xyz = np.asarray(xyz, np.float64)
    r = np.linalg.norm(xyz, axis=1)
    return np.stack([np.arctan2(xyz[:, 1], xyz[:, 0]), np.arccos(np.clip(xyz[:, 2] / r, -1.0, 1.0))], axis=1)


def sh2amp_mapping(dirs_azel: np.ndarray, lmax: int | None = None, default_lmax: int = 8):
    """(mapping [ndir][nSH], lmax) as DWI::compute_SH2amp_mapping chooses it:
    a requested lmax is capped by the direction count and kept; otherwise
    lmax starts at min(LforN(ndir), default_lmax) and drops by 2 while the
    condition number is 100 or more."""
    from_ndir = l_for_n(len(dirs_azel))
    requested = lmax is not None
    if requested:
        if lmax % 2 or lmax < 0:
            raise ValueError("lmax must be an even, non-negative number")
        lmax = min(lmax, from_ndir)
    else:
        lmax = min(from_ndir, default_lmax)
    while True:
        mapping = init_transform(dirs_azel, lmax)
        s = np.linalg.svd(mapping, compute_uv=False)
        cond = s[0] / s[-1] if s[-1] > 0 else np.inf
        if cond < 100.0 or requested or lmax < 2:
            return mapping, lmax
        lmax -= 2


def pinv(m: np.ndarray) -> np.ndarray:
    """Math::pinv (least_squares.h:39-45): (M^T M)^-1 M^T."""
    return np.linalg.solve(m.T @ m, m.T)
