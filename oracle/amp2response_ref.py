"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of MRtrix3's
amp2response fit (cmd/amp2response.cpp:83-190, 330-351), the checker of the
GPU amp2response (never imported by the product path).

Per single-fibre voxel: the rotation of gen_rotation_matrix (:83-100: the
fibre direction as the new z axis, the other two axes from a random vector,
here a fixed one), the shell's directions rotated and turned into [az el]
(Math::Sphere::cartesian2spherical), elevations above pi/2 folded back
(:165-173), the zonal transform at those elevations (ZSH::init_amp_transform,
the normalised Legendre P_l0), then M += T^T T, b += T^T a.  The fit: M^-1 b
for lmax 0 or without constraints; otherwise the ICLS problem in standard
form with the amplitude and its elevation derivative non-negative at
0..90 degrees and regularisation 1e-10 (oracle/icls_ref.py).
"""
from __future__ import annotations

import math

import numpy as np

from . import icls_ref
from . import oracle as O


def _zonal(els, lmax, m=0):
    out = np.zeros((len(els), lmax // 2 + 1))
    for i, e in enumerate(els):
        p = O.plm_sph(lmax, m, math.cos(e)) if np.isfinite(e) else np.full(lmax + 1, np.nan)
        if not np.isfinite(e):
            p[0] = 0.282094791773878 if m == 0 else np.nan
        for l in range(0, lmax + 1, 2):
            if m == 0:
                out[i, l // 2] = p[l]
            elif l >= 2:
                out[i, l // 2] = p[l] * math.sqrt(l * (l + 1))
    return out


def accumulate(amp, fibre_dirs, mask, shell_dirs, volumes, lmax):
    amp = np.asarray(amp, np.float64)
    nz = lmax // 2 + 1
    M = np.zeros((nz, nz))
    b = np.zeros(nz)
    helper = np.array([0.3, -0.7, 0.64])
    for v in np.nonzero(mask)[0]:
        f = np.asarray(fibre_dirs[v, :3], np.float64)
        f = f / np.linalg.norm(f)
        e2 = np.cross(f, helper)
        e2 /= np.linalg.norm(e2)
        e3 = np.cross(f, e2)
        e3 /= np.linalg.norm(e3)
        R = np.stack([e2, e3, f])
        rot = shell_dirs @ R.T
        with np.errstate(invalid="ignore"):
            el = np.arccos(np.clip(rot[:, 2] / np.linalg.norm(rot, axis=1), -1.0, 1.0))
        el = np.where(el > math.pi / 2, math.pi - el, el)
        T = _zonal(el, lmax)
        a = amp[v, volumes]
        M += T.T @ T
        b += T.T @ a
    return M, b


def constraints(lmax):
    els = np.arange(91) * math.pi / 180.0
    return np.vstack([_zonal(els, lmax, 0), _zonal(els, lmax, 1)])


def fit(M, b, lmax, constrained=True):
    if lmax == 0 or not constrained:
        L = np.linalg.cholesky(M)
        return np.linalg.solve(L.T, np.linalg.solve(L, b))
    P = icls_ref.Problem(M, constraints(lmax), None, 0, solution_reg=1e-10, constraint_reg=1e-10,
                         standard_form=True)
    x, _ = icls_ref.solve(P, b)
    return x
