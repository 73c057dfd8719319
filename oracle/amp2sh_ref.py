"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of MRtrix3's amp2sh
per-voxel fit (cmd/amp2sh.cpp:108-197), the checker of the GPU amp2sh
(never imported by the product path).

get_amps (:157-171): a = the selected volumes' amplitudes, times
nb0 / (1 + the b=0 amplitudes summed in order) with -normalise.  Plain fit:
c = pinv(SH2amp) a.  -rician (:129-150 with get_rician_bias :180-197): from
that c, up to 20 rounds of ap = max(SH2amp c, 0), t = (ap / noise)^2.25,
w = ((t + 1.7) / (t + 1.12))^2, diff = a - noise (t + 1.65)^(1 / 2.25);
stop when sum diff^2 / sum a^2 < 1e-8, else c = argmin ||diag(w) (SH2amp c -
(ap + diff))|| by the normal equations (Cholesky, as LLT there).
"""
from __future__ import annotations

import numpy as np

RICIAN_POWER = 2.25


def amps(row, dwis, bzeros=(), normalise=False):
    row = np.asarray(row, np.float64)
    norm = 1.0
    if normalise:
        t = 1.0
        for i in bzeros:
            t += row[i]
        norm = len(bzeros) / t
    return row[np.asarray(dwis)] * norm


def fit_rician(a, sh2amp, fit, noise):
    a = np.asarray(a, np.float64)
    c = fit @ a
    for _ in range(20):
        ap = np.maximum(sh2amp @ c, 0.0)
        t = (ap / noise) ** RICIAN_POWER
        w = ((t + 1.7) / (t + 1.12)) ** 2
        diff = a - noise * (t + 1.65) ** (1.0 / RICIAN_POWER)
        if np.sum(diff * diff) / np.sum(a * a) < 1e-8:
            break
        ap = ap + diff
        H = sh2amp * w[:, None]
        Q = H.T @ H
        L = np.linalg.cholesky(Q)
        c = np.linalg.solve(L.T, np.linalg.solve(L, H.T @ ap))
    return c
