"""TEST INFRASTRUCTURE ONLY: FP64 restatement of MSMT_CSD::Shared::init
(src/dwi/sdeconv/msmt_csd.h:90-211), the checker of the GPU multi-tissue
CSD (never imported by the product path).

Forward matrix C [volumes][sum of tissue parameters]: for tissue t with
lmax L_t, shell s and volume v of that shell, C[v, (l, m) of t] =
Y_lm(direction of v) * R_t[s, l / 2] / Y_l0(pole), with Y_l0(pole) =
sqrt((2l + 1) / 4 pi); a b=0 volume (no direction) keeps only its l = 0 term.
Constraints A: per tissue, its SH basis on the constraint directions (a
single row, the l = 0 basis value, for an lmax-0 tissue), block-diagonal.
The problem is then min ||C x - b||^2 s.t. A x >= 0 with solution and
constraint regularisation 1e-10 (msmt_csd.h:31-32, 203-204), solved by the
ICLS restatement (oracle/icls_ref.py).
"""
from __future__ import annotations

import math

import numpy as np

from . import icls_ref
from . import oracle as O


def _basis(dirs_azel, lmax):
    return O.init_transform(np.ascontiguousarray(dirs_azel, np.float64), lmax)


def forward_matrix(grad, shells, responses, lmax):
    """C for the unit-normalised gradient table ``grad``, the shells' volume
    lists (ascending b) and per tissue a [shells][lmax/2 + 1] response."""
    grad = np.asarray(grad, np.float64)
    n = [(L + 1) * (L + 2) // 2 for L in lmax]
    C = np.zeros((grad.shape[0], sum(n)))
    p0 = 0
    for t, L in enumerate(lmax):
        for s, vols in enumerate(shells):
            for v in vols:
                g = grad[v, :3]
                if np.linalg.norm(g) == 0.0:
                    row = np.zeros(n[t])
                    row[0] = 1.0 / math.sqrt(4.0 * math.pi)
                else:
                    az = math.atan2(g[1], g[0])
                    z = g[2] / np.linalg.norm(g)
                    el = 0.0 if z >= 1.0 else (math.pi if z <= -1.0 else math.acos(z))
                    row = _basis(np.array([[az, el]]), L)[0]
                for l in range(0, L + 1, 2):
                    pole = math.sqrt((2 * l + 1) / (4.0 * math.pi))
                    k = l // 2
                    r = responses[t][s, k] if k < responses[t].shape[1] else 0.0
                    for m in range(-l, l + 1):
                        C[v, p0 + l * (l + 1) // 2 + m] = row[l * (l + 1) // 2 + m] * r / pole
        p0 += n[t]
    return C


def constraint_matrix(hr_dirs, lmax):
    n = [(L + 1) * (L + 2) // 2 for L in lmax]
    m = [len(hr_dirs) if L > 0 else 1 for L in lmax]
    A = np.zeros((sum(m), sum(n)))
    r0 = c0 = 0
    for t, L in enumerate(lmax):
        A[r0:r0 + m[t], c0:c0 + n[t]] = _basis(hr_dirs, L)[:m[t]]
        r0 += m[t]
        c0 += n[t]
    return A


def problem(grad, shells, responses, lmax, hr_dirs, norm_lambda=1e-10, neg_lambda=1e-10):
    C = forward_matrix(grad, shells, responses, lmax)
    A = constraint_matrix(hr_dirs, lmax)
    return icls_ref.Problem(C, A, None, 0, solution_reg=norm_lambda, constraint_reg=neg_lambda)


def solve(P, dwi):
    """[n][parameters] solutions and [n] solver rounds for the rows of ``dwi``."""
    dwi = np.asarray(dwi, np.float64)
    x = np.zeros((len(dwi), P.H.shape[1]))
    it = np.zeros(len(dwi), int)
    for i, b in enumerate(dwi):
        x[i], it[i] = icls_ref.solve(P, b)
    return x, it
