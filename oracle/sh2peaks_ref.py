"""TEST INFRASTRUCTURE ONLY: FP64 CPU restatement of MRtrix3's ``sh2peaks``,
the checker of the GPU peak finder (never imported by the product path).

Follows cmd/sh2peaks.cpp:99-303 (Direction, Processor, check_input) and
core/math/SH.h:515-650 (get_peak: Newton steps on the sphere from a seed,
at most 50, step capped at MAX_DIR_CHANGE = 0.2 rad, converged below
ANGLE_TOLERANCE = 1e-4; derivatives: amplitude and first / second
derivatives in elevation and azimuth from the normalised associated
Legendre functions), with Plm_sph's cos / sin overload
(core/math/legendre.h:125-153).  The reference computes in float; this
restatement in double, vectorised over the seeds of a voxel.
"""
from __future__ import annotations

import math

import numpy as np

MAX_DIR_CHANGE = 0.2
ANGLE_TOLERANCE = 1e-4
DOT_THRESHOLD = 0.99


def _helper(x, m):
    # legendre.h:65-68 (recursive product)
    out = np.ones_like(x)
    while m >= 1.0:
        out = out * x * (m - 1.0) / m
        m -= 2.0
    return out


def plm_sph(lmax: int, m: int, x, sin_x):
    """[lmax+1][n] normalised associated Legendre values of order m (rows < m unused)."""
    x = np.asarray(x, np.float64)
    sin2 = np.asarray(sin_x, np.float64) ** 2
    out = np.zeros((lmax + 1,) + x.shape)
    start = np.full(x.shape, 0.282094791773878)
    if m:
        start = start * np.sqrt((2 * m + 1) * _helper(sin2, 2.0 * m))
    if m & 1:
        start = -start
    zero = (sin2 == 0.0) if m else np.zeros(x.shape, bool)
    out[m] = start
    if lmax > m:
        f = math.sqrt(2 * m + 3)
        out[m + 1] = x * f * out[m]
        for n in range(m + 2, lmax + 1):
            out[n] = x * out[n - 1] - out[n - 2] / f
            f = math.sqrt((4 * n * n - 1) / (n * n - m * m))
            out[n] = out[n] * f
    out[m:, zero] = 0.0
    return out


def _idx(l, m):
    return l * (l + 1) // 2 + m


def _mpos(l, m):
    return l * l // 4 + m


def derivatives(sh, lmax, el, az):
    """SH.h:569-650 for arrays of (el, az): amplitude, d/del, d/daz, d2/del2, d2/deldaz, d2/daz2."""
    sel, cel = np.sin(el), np.cos(el)
    atpole = sel < 1e-4
    AL = np.zeros(((lmax // 2 + 1) ** 2,) + np.shape(el))
    for m in range(lmax + 1):
        buf = plm_sph(lmax, m, cel, sel)
        for l in range(m + 1 if m & 1 else m, lmax + 1, 2):
            AL[_mpos(l, m)] = buf[l]
    amp = sh[0] * AL[0]
    d_el = np.zeros_like(amp)
    d_az = np.zeros_like(amp)
    d2_el = np.zeros_like(amp)
    d2_elaz = np.zeros_like(amp)
    d2_az = np.zeros_like(amp)
    for l in range(2, lmax + 1, 2):
        v = sh[_idx(l, 0)]
        amp = amp + v * AL[_mpos(l, 0)]
        d_el = d_el + v * math.sqrt(l * (l + 1)) * AL[_mpos(l, 1)]
        d2_el = d2_el + v * (math.sqrt(l * (l + 1) * (l - 1) * (l + 2)) * AL[_mpos(l, 2)] - l * (l + 1) * AL[_mpos(l, 0)]) / 2.0
    for m in range(1, lmax + 1):
        caz = math.sqrt(2.0) * np.cos(m * az)
        saz = math.sqrt(2.0) * np.sin(m * az)
        for l in range(m + 1 if m & 1 else m, lmax + 1, 2):
            vp, vm = sh[_idx(l, m)], sh[_idx(l, -m)]
            amp = amp + (vp * caz + vm * saz) * AL[_mpos(l, m)]
            tmp = math.sqrt((l + m) * (l - m + 1)) * AL[_mpos(l, m - 1)]
            if l > m:
                tmp = tmp - math.sqrt((l - m) * (l + m + 1)) * AL[_mpos(l, m + 1)]
            tmp = tmp / -2.0
            d_el = d_el + (vp * caz + vm * saz) * tmp
            tmp2 = -((l + m) * (l - m + 1) + (l - m) * (l + m + 1)) * AL[_mpos(l, m)]
            if m == 1:
                tmp2 = tmp2 - math.sqrt((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2)) * AL[_mpos(l, 1)]
            else:
                tmp2 = tmp2 + math.sqrt((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2)) * AL[_mpos(l, m - 2)]
            if l > m + 1:
                tmp2 = tmp2 + math.sqrt((l - m) * (l + m + 1) * (l - m - 1) * (l + m + 2)) * AL[_mpos(l, m + 2)]
            tmp2 = tmp2 / 4.0
            d2_el = d2_el + (vp * caz + vm * saz) * tmp2
            d_az = d_az + np.where(atpole, (vm * caz - vp * saz) * tmp, m * (vm * caz - vp * saz) * AL[_mpos(l, m)])
            d2_elaz = d2_elaz + np.where(atpole, 0.0, m * (vm * caz - vp * saz) * tmp)
            d2_az = d2_az - np.where(atpole, 0.0, (vp * caz + vm * saz) * m * m * AL[_mpos(l, m)])
    safe = np.where(atpole, 1.0, sel)
    d_az = np.where(atpole, d_az, d_az / safe)
    d2_elaz = np.where(atpole, d2_elaz, d2_elaz / safe)
    d2_az = np.where(atpole, d2_az, d2_az / (safe * safe))
    return amp, d_el, d_az, d2_el, d2_elaz, d2_az


def get_peaks(sh, lmax, v0):
    """get_peak (SH.h:515-560) from every row of v0 [n][3]; returns (amplitude, v), NaN where it fails."""
    v = np.array(v0, np.float64)
    n = len(v)
    amp_out = np.full(n, np.nan)
    active = np.ones(n, bool)
    for _ in range(50):
        if not active.any():
            break
        idx = np.nonzero(active)[0]
        u = v[idx]
        az = np.arctan2(u[:, 1], u[:, 0])
        el = np.arctan2(np.hypot(u[:, 0], u[:, 1]), u[:, 2])
        amp, dSH_del, dSH_daz, d2_del2, d2_deldaz, d2_daz2 = derivatives(sh, lmax, el, az)
        dl = np.sqrt(dSH_del ** 2 + dSH_daz ** 2)
        nz = dl != 0.0
        daz = np.where(nz, dSH_daz / np.where(nz, dl, 1.0), 0.0)
        dl2 = np.where(nz, dSH_del / np.where(nz, dl, 1.0), dl)
        dSH_dt = daz * dSH_daz + dl2 * dSH_del
        d2SH_dt2 = daz * daz * d2_daz2 + 2.0 * daz * dl2 * d2_deldaz + dl2 * dl2 * d2_del2
        dt = np.where(d2SH_dt2 != 0.0, -dSH_dt / np.where(d2SH_dt2 != 0.0, d2SH_dt2, 1.0), MAX_DIR_CHANGE)
        dt = np.minimum(np.abs(dt), MAX_DIR_CHANGE)
        de, da = dl2 * dt, daz * dt
        u = u + np.stack([de * np.cos(az) * np.cos(el) - da * np.sin(az),
                          de * np.sin(az) * np.cos(el) + da * np.cos(az),
                          -de * np.sin(el)], axis=1)
        u = u / np.linalg.norm(u, axis=1, keepdims=True)
        v[idx] = u
        done = dt < ANGLE_TOLERANCE
        amp_out[idx[done]] = amp[done]
        active[idx[done]] = False
    v[active] = np.nan
    return amp_out, v


def seed_vectors(seeds_azel):
    """Direction(phi, theta) of sh2peaks.cpp:104: v = [cos phi sin theta, sin phi sin theta, cos theta]."""
    az, el = seeds_azel[:, 0], seeds_azel[:, 1]
    return np.stack([np.cos(az) * np.sin(el), np.sin(az) * np.sin(el), np.cos(el)], axis=1)


def voxel_peaks(sh, lmax, seeds_azel, npeaks=3, threshold=-np.inf, targets=None):
    """Processor::operator() (sh2peaks.cpp:183-262) for one voxel: [npeaks][3] amplitude-scaled
    directions, NaN-padded; ``targets`` [npeaks][3] selects, per target, the peak of largest |dot|."""
    out = np.full((npeaks, 3), np.nan)
    sh = np.asarray(sh, np.float64)
    if np.isnan(sh).any() or not np.any(sh[1:] != 0.0):
        return out
    amps, vs = get_peaks(sh, lmax, seed_vectors(np.asarray(seeds_azel, np.float64)))
    kept = []
    for a, v in zip(amps, vs):
        if np.isfinite(a):
            if any(abs(np.dot(v, k[1])) > DOT_THRESHOLD for k in kept):
                continue
            if a >= threshold:
                kept.append((a, v))
    if targets is not None:
        chosen = []
        for t in np.asarray(targets, np.float64):
            t = t / np.linalg.norm(t)
            best, mdot = None, 0.0
            for a, v in kept:
                f = abs(np.dot(t, v))
                if f > mdot:
                    mdot, best = f, (a, v)
            chosen.append(best)
    else:
        chosen = sorted(kept, key=lambda p: -p[0])[:npeaks]
    for i, p in enumerate(chosen[:min(npeaks, len(kept))]):
        if p is not None:
            out[i] = p[0] * p[1]
    return out
