"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of dwi2tensor's IWLS fit
(cmd/dwi2tensor.cpp:106-135), tensor2FA (src/dwi/tensor.h:95-104) and the
principal eigenvector (tensor2metric -vector, modulated by FA), the checker
of the GPU tensor fit (never imported by the product path)."""
from __future__ import annotations

import numpy as np


def fit(dwi_row, B, iter=2, ols=False):
    s = np.asarray(dwi_row, np.float64).copy()
    small = 1.0e-6 * s.max()
    s = np.where(s < small, small, s)
    w = np.ones_like(s) if ols else s.copy()
    y = np.log(s)
    p = None
    for it in range(iter + 1):
        Bw = B * (w * w)[:, None]
        A = B.T @ Bw
        r = Bw.T @ y
        L = np.linalg.cholesky(A)
        p = np.linalg.solve(L.T, np.linalg.solve(L, r))
        if it < iter:
            w = np.exp(B @ p)
    return p


def fa(dt):
    tr = (dt[0] + dt[1] + dt[2]) / 3.0
    a = np.array([dt[0] - tr, dt[1] - tr, dt[2] - tr])
    off = dt[3] ** 2 + dt[4] ** 2 + dt[5] ** 2
    nrm = dt[0] ** 2 + dt[1] ** 2 + dt[2] ** 2 + 2.0 * off
    return np.sqrt(1.5 * (a @ a + 2.0 * off) / nrm) if nrm else 0.0


def principal(dt):
    M = np.array([[dt[0], dt[3], dt[4]], [dt[3], dt[1], dt[5]], [dt[4], dt[5], dt[2]]])
    w, V = np.linalg.eigh(M)
    return V[:, np.argmax(w)]
