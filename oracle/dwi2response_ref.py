"""TEST INFRASTRUCTURE ONLY: dwi2response tournier / tax with every GPU step
replaced by its FP64 CPU restatement, the checker of the GPU pipeline
(never imported by the product path).

The loops themselves are mrtrix3_b200.dwi2response.tournier_loop / tax_loop
(restating lib/mrtrix3/dwi2response/tournier.py:53-150 and tax.py:53-160;
their control flow is tested on the CPU with fake steps).  Here their steps
are ``dwi2fod csd`` by oracle/oracle.py (csd.h), ``fod2fixel
-fmls_no_thresholds`` by oracle/fmls_oracle.c (fmls.cpp; equal to the
literal restatement oracle/fmls_ref.py on its fixtures) and ``amp2response``
by oracle/amp2response_ref.py (amp2response.cpp), so that the GPU run and
this one differ only in the steps' arithmetic.  Parity unpinned against
reference-run output (the scripts' test data are absent).
"""
from __future__ import annotations

import os

import numpy as np

from . import amp2response_ref as AREF
from . import fmls_ref
from . import oracle as O


def _csd_lmax(rf):
    return min(2 * (len(rf) - 1), 8)  # csd.h: lmax = min(lmax_response, 8) without -lmax


def iterative_ref(algo, grad_shell, dwi_shell, mask, dims, hr_dirs, number=300, iter_voxels=0, dilate_passes=1,
                  max_iters=None, lmax=None, peak_ratio=0.1, convergence=0.5):
    """(response, single-fibre rows, iterations) for dwi_shell [n][volumes of
    the single shell] and its scheme grad_shell (normalised, [volumes][4])."""
    from mrtrix3_b200 import dwi2response as D
    from mrtrix3_b200 import msmt
    dwi = np.asarray(dwi_shell, np.float64)
    dirs = msmt.direction_matrix(grad_shell, np.arange(len(grad_shell)))
    cart = np.stack([np.cos(dirs[:, 0]) * np.sin(dirs[:, 1]), np.sin(dirs[:, 0]) * np.sin(dirs[:, 1]),
                     np.cos(dirs[:, 1])], axis=1)

    segs = {}

    def step(rf, voxels):
        v = np.asarray(voxels, bool)
        sh_lmax = _csd_lmax(rf)
        nsh = (sh_lmax + 1) * (sh_lmax + 2) // 2
        F = np.zeros((len(dwi), nsh))
        if v.any():
            F[v] = O.OracleShared(grad_shell, np.asarray(rf, np.float64), hr_dirs).solve(
                dwi[v].astype(np.float32))["F"]
        F = F.astype(np.float32).astype(np.float64)   # the FOD image is float32
        if sh_lmax not in segs:
            segs[sh_lmax] = fmls_ref.Segmenter(sh_lmax, 0.0, 0.0, 1.0)
        p1 = np.zeros(len(dwi), np.float32)
        p2 = np.zeros(len(dwi), np.float32)
        d1 = np.full((len(dwi), 3), np.nan, np.float32)
        idx = np.nonzero(v)[0]
        if len(idx):
            c, fx = fmls_ref.segment_batch_c(segs[sh_lmax], F[idx], max_out=2, nthreads=os.cpu_count() or 1)
            p1[idx] = np.where(c >= 1, fx[:, 0, 7], 0.0)
            p2[idx] = np.where(c >= 2, fx[:, 1, 7], 0.0)
            d1[idx] = np.where((c >= 1)[:, None], fx[:, 0, 0:3], np.nan)
        return p1, p2, d1

    def fit(sf, first_dir, L):
        L = L if L is not None else 10
        M, b = AREF.accumulate(dwi.astype(np.float32), np.nan_to_num(first_dir), np.asarray(sf, bool), cart,
                               np.arange(len(grad_shell)), L)
        return np.array([float(f"{x:.10g}") for x in AREF.fit(M, b, L)])

    if algo == "tournier":
        return D.tournier_loop(step, fit, mask, dims, number=number, iter_voxels=iter_voxels,
                               dilate_passes=dilate_passes, max_iters=max_iters or 10, lmax=lmax)
    mean, std = D.masked_mean_std(dwi.astype(np.float32), mask)
    mean, std = mean * np.sqrt(4.0 * np.pi), std * np.sqrt(4.0 * np.pi)
    return D.tax_loop(step, fit, mask, [mean, -0.5 * std, 0.25 * std * std / mean], peak_ratio=peak_ratio,
                      max_iters=max_iters or 20, convergence=convergence, lmax=lmax)
