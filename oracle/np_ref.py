"""TEST INFRASTRUCTURE ONLY: an independent numpy/scipy CSD used to cross-check
the C oracle.  It shares no code with csd_oracle.c: the SH basis comes from
scipy.special.sph_harm_y (complex SH with the Condon-Shortley phase; the
MRtrix real basis of core/math/SH.h:82-104 is sqrt(2)*Re / sqrt(2)*Im for
m>0), pinv from numpy.linalg, and the per-voxel solve from scipy.linalg's
Cholesky.  It follows src/dwi/sdeconv/csd.h:117-198 and 237-269.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla
import scipy.special as sps


def sh_basis(dirs_azel: np.ndarray, lmax: int) -> np.ndarray:
    az, el = dirs_azel[:, 0], dirs_azel[:, 1]
    n = (lmax + 1) * (lmax + 2) // 2
    out = np.zeros((len(az), n))
    for l in range(0, lmax + 1, 2):
        c = l * (l + 1) // 2
        out[:, c] = sps.sph_harm_y(l, 0, el, az).real
        for m in range(1, l + 1):
            y = sps.sph_harm_y(l, m, el, az)
            out[:, c + m] = math.sqrt(2.0) * y.real
            out[:, c - m] = math.sqrt(2.0) * y.imag
    return out


def shared(grad, response, hr_dirs, lmax=0, neg_lambda=1.0, norm_lambda=1.0, threshold=0.0):
    """Single-shell case only (all b > 10 volumes form one shell)."""
    grad = np.asarray(grad, np.float64)
    dwis = np.nonzero(grad[:, 3] > 10.0)[0]
    g = grad[dwis, :3] / np.linalg.norm(grad[dwis, :3], axis=1, keepdims=True)
    dirs = np.stack([np.arctan2(g[:, 1], g[:, 0]), np.arccos(np.clip(g[:, 2], -1, 1))], 1)
    ndw = len(dwis)
    lmax_data = 2 * int(math.floor((math.sqrt(1 + 8 * ndw) - 3) / 4))
    lresp = 2 * (len(response) - 1)
    lmax = lmax or min(lresp, 8)
    lresp = min(lresp, lmax_data, lmax)
    RH = np.array([response[k] / math.sqrt((4 * k + 1) / (4 * math.pi)) for k in range(len(response))])
    RH = np.concatenate([RH, np.zeros(max(0, lmax // 2 + 1 - len(RH)))])
    filt = np.zeros(lresp // 2 + 1)
    filt[:3] = 1.0
    fconv = sh_basis(dirs, lresp)
    k = min(fconv.shape)
    fconv[np.arange(k), np.arange(k)] += 1e-2
    rconv = np.linalg.solve(fconv.T @ fconv, fconv.T)
    lvec = np.concatenate([[l] * (2 * l + 1) for l in range(0, lresp + 1, 2)])
    rconv *= (filt[lvec // 2] / RH[lvec // 2])[:, None]
    n = (lmax + 1) * (lmax + 2) // 2
    lvec_full = np.concatenate([[l] * (2 * l + 1) for l in range(0, lmax + 1, 2)])
    M = sh_basis(dirs, lmax) * RH[lvec_full // 2][None, :]
    c = neg_lambda * 50.0 * response[0] / len(hr_dirs)
    H = sh_basis(np.asarray(hr_dirs, np.float64), lmax) * c
    MtM = M.T @ M
    if norm_lambda:
        MtM[np.diag_indices(n)] += norm_lambda * 2e-4 * MtM[0, 0]
    return dict(dwis=dwis, rconv=rconv, M=M, H=H, MtM=MtM, threshold=threshold * c, n=n, nr=rconv.shape[0])


def solve_voxel(sh, signal_all_vols, niter=50):
    S = np.maximum(np.asarray(signal_all_vols, np.float64)[sh["dwis"]], 0.0)
    F = np.zeros(sh["n"])
    F[:sh["nr"]] = sh["rconv"] @ S
    b = sh["M"].T @ S
    old = None
    it = 0
    for it in range(1, niter + 1):
        neg = np.nonzero(sh["H"] @ F < sh["threshold"])[0]
        if old is not None and np.array_equal(neg, old):
            break
        Hn = sh["H"][neg]
        W = sh["MtM"] + Hn.T @ Hn
        F = sla.cho_solve(sla.cho_factor(W, lower=True), b)
        old = neg
    else:
        it = niter
    return F, it, (old if old is not None else np.array([], int))
