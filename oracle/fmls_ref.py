"""TEST INFRASTRUCTURE ONLY: FP64 CPU restatement of MRtrix3's FMLS FOD
segmenter (``fod2fixel``), the checker of the GPU segmenter (never imported
by the product path).

Follows src/dwi/fmls.cpp:159-311 (Segmenter::operator()) and the FOD_lobe
class of src/dwi/fmls.h:60-160 literally: a vector of lobes with direction
masks, lobes merged and erased by vector index, retrospective assignments
re-indexed on every merge; get_peak's Newton search (core/math/SH.h:515-560)
with derivatives from the PrecomputedAL table (SH.h:399-463, 569-650) that
the segmenter uses (2 x 1281 elevations, linear interpolation); and
fod2fixel's per-fixel outputs (cmd/fod2fixel.cpp:109-125, 250-286).  The
direction set, its adjacency, grid lookup and integration weights come from
mrtrix3_b200.directions (data tables, checked by their own tests).

Pinning: parity unpinned against reference-run output.  The reference's
golden fixel directories (testing/binaries/tests/fod2fixel, fod2fixel/out1-3)
live in a test-data submodule that is absent, and the reference cannot be
built here.  Only the PrecomputedAL interpolation is pinned, by the
reference's own known-answer test (testing_unit_tests_sh_precomputer.cpp,
restated in tests/test_fmls_host.py).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_CLIB = None

MAX_DIR_CHANGE = 0.2
ANGLE_TOLERANCE = 1e-4


def _mpos(l, m):
    return l * l // 4 + m


def _idx(l, m):
    return l * (l + 1) // 2 + m


class _AL:
    def __init__(self, table):
        self.table = table
        self.ndir = table.shape[0]
        self.inc = math.pi / (self.ndir - 1)

    def get(self, el):
        f2 = el / self.inc
        i = int(f2)
        if i < 0:
            i, f1, f2 = 0, 1.0, 0.0
        elif i >= self.ndir - 1:
            i, f1, f2 = self.ndir - 1, 1.0, 0.0
        else:
            f2 -= i
            f1 = 1.0 - f2
        v = f1 * self.table[i]
        if f2:
            v = v + f2 * self.table[i + 1]
        return v


def derivatives(sh, lmax, el, az, al):
    """SH::derivatives with a precomputer (SH.h:569-650), scalars."""
    sel, cel = math.sin(el), math.cos(el)
    atpole = sel < 1e-4
    AL = al.get(el)
    amp = sh[0] * AL[0]
    d_el = d_az = d2_el = d2_elaz = d2_az = 0.0
    for l in range(2, lmax + 1, 2):
        v = sh[_idx(l, 0)]
        amp += v * AL[_mpos(l, 0)]
        d_el += v * math.sqrt(l * (l + 1)) * AL[_mpos(l, 1)]
        d2_el += v * (math.sqrt(l * (l + 1) * (l - 1) * (l + 2)) * AL[_mpos(l, 2)] - l * (l + 1) * AL[_mpos(l, 0)]) / 2.0
    for m in range(1, lmax + 1):
        caz = math.sqrt(2.0) * math.cos(m * az)
        saz = math.sqrt(2.0) * math.sin(m * az)
        for l in range(m + 1 if m & 1 else m, lmax + 1, 2):
            vp, vm = sh[_idx(l, m)], sh[_idx(l, -m)]
            amp += (vp * caz + vm * saz) * AL[_mpos(l, m)]
            tmp = math.sqrt((l + m) * (l - m + 1)) * AL[_mpos(l, m - 1)]
            if l > m:
                tmp -= math.sqrt((l - m) * (l + m + 1)) * AL[_mpos(l, m + 1)]
            tmp /= -2.0
            d_el += (vp * caz + vm * saz) * tmp
            tmp2 = -((l + m) * (l - m + 1) + (l - m) * (l + m + 1)) * AL[_mpos(l, m)]
            if m == 1:
                tmp2 -= math.sqrt((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2)) * AL[_mpos(l, 1)]
            else:
                tmp2 += math.sqrt((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2)) * AL[_mpos(l, m - 2)]
            if l > m + 1:
                tmp2 += math.sqrt((l - m) * (l + m + 1) * (l - m - 1) * (l + m + 2)) * AL[_mpos(l, m + 2)]
            tmp2 /= 4.0
            d2_el += (vp * caz + vm * saz) * tmp2
            if atpole:
                d_az += (vm * caz - vp * saz) * tmp
            else:
                d_az += m * (vm * caz - vp * saz) * AL[_mpos(l, m)]
                d2_elaz += m * (vm * caz - vp * saz) * tmp
                d2_az -= (vp * caz + vm * saz) * m * m * AL[_mpos(l, m)]
    if not atpole:
        d_az /= sel
        d2_elaz /= sel
        d2_az /= sel * sel
    return amp, d_el, d_az, d2_el, d2_elaz, d2_az


def get_peak(sh, lmax, u, al):
    """SH::get_peak (SH.h:515-560): (amplitude, unit vector), NaN if no convergence."""
    u = np.array(u, np.float64)
    for _ in range(50):
        az = math.atan2(u[1], u[0])
        el = math.atan2(math.hypot(u[0], u[1]), u[2])
        amp, dSH_del, dSH_daz, d2_del2, d2_deldaz, d2_daz2 = derivatives(sh, lmax, el, az, al)
        dl = math.sqrt(dSH_del * dSH_del + dSH_daz * dSH_daz)
        daz = 0.0
        if dl != 0.0:
            daz = dSH_daz / dl
            dl = dSH_del / dl
        dSH_dt = daz * dSH_daz + dl * dSH_del
        d2SH_dt2 = daz * daz * d2_daz2 + 2.0 * daz * dl * d2_deldaz + dl * dl * d2_del2
        dt = (-dSH_dt / d2SH_dt2) if d2SH_dt2 else MAX_DIR_CHANGE
        dt = min(abs(dt), MAX_DIR_CHANGE)
        dl *= dt
        daz *= dt
        u = u + np.array([dl * math.cos(az) * math.cos(el) - daz * math.sin(az),
                          dl * math.sin(az) * math.cos(el) + daz * math.cos(az),
                          -dl * math.sin(el)])
        u = u / math.sqrt(float(u @ u))
        if dt < ANGLE_TOLERANCE:
            return amp, u
    return math.nan, np.full(3, np.nan)


class _Lobe:
    def __init__(self, unit, seed, value, weight):
        self.mask = {seed}
        self.values = {seed: value}
        self.max_peak = abs(value)
        self.peaks = [unit[seed].copy()]
        self.mean = unit[seed] * abs(value) * weight
        self.integral = abs(value * weight)
        self.neg = value <= 0.0

    def add(self, unit, d, value, weight):
        self.mask.add(d)
        self.values[d] = value
        mult = 1.0 if float(self.mean @ unit[d]) > 0.0 else -1.0
        self.mean = self.mean + unit[d] * mult * abs(value) * weight
        self.integral += abs(value * weight)

    def merge(self, that):
        self.mask |= that.mask
        if that.max_peak > self.max_peak:
            self.max_peak = that.max_peak
            self.peaks = that.peaks + self.peaks
        else:
            self.peaks = self.peaks + that.peaks
        mult = 1.0 if float(self.mean @ that.mean) > 0.0 else -1.0
        self.mean = self.mean + that.mean * that.integral * mult
        self.integral += that.integral


class Segmenter:
    """Segmenter (fmls.cpp:118-311) on the 1281-direction set for one lmax."""

    def __init__(self, lmax, integral_threshold=0.0, peak_value_threshold=0.1, merge_ratio=1.0):
        from mrtrix3_b200 import directions, sh
        self.lmax = lmax
        self.unit = directions.unit_vectors(directions.load_tessellation_1281())
        self.adj = directions.adjacency_1281()
        self.lookup = directions.FastLookup(self.unit, self.adj)
        self.weights = directions.integration_weights(self.unit)
        az = np.arctan2(self.unit[:, 1], self.unit[:, 0])
        el = np.arccos(self.unit[:, 2])
        self.sh2amp = sh.init_transform(np.stack([az, el], axis=1), lmax)
        self.al = _AL(directions.precomputed_al(lmax, 2 * len(self.unit)))
        self.integral_threshold = integral_threshold
        self.peak_value_threshold = peak_value_threshold
        self.merge_ratio = merge_ratio

    def __call__(self, coefs):
        """The lobes of one voxel: list of dicts {mean_dir, peak_dir, integral, max_peak}."""
        sh = np.asarray(coefs, np.float64)
        if not (sh[0] > 0.0) or not math.isfinite(sh[0]) or not np.isfinite(sh).all():
            return []
        values = self.sh2amp @ sh
        order = sorted(range(len(values)), key=lambda i: (-abs(values[i]), i))
        if values[order[0]] <= 0.0:
            return []
        out, retro = [], []
        unit, w = self.unit, self.weights
        for d in order:
            v = values[d]
            adj_lobes = [l for l in range(len(out))
                         if (v <= 0.0) == out[l].neg and any(a in out[l].mask for a in self.adj[d])]
            if not adj_lobes:
                out.append(_Lobe(unit, d, v, w[d]))
            elif len(adj_lobes) == 1:
                out[adj_lobes[0]].add(unit, d, v, w[d])
            elif abs(v) / out[adj_lobes[-1]].max_peak > self.merge_ratio:
                adj_lobes.sort()
                for j in adj_lobes[1:]:
                    out[adj_lobes[0]].merge(out[j])
                out[adj_lobes[0]].add(unit, d, v, w[d])
                for r in retro:
                    if r[1] in adj_lobes[1:]:
                        r[1] = adj_lobes[0]
                    else:
                        r[1] -= sum(1 for k in adj_lobes[1:] if k < r[1])
                for j in reversed(adj_lobes[1:]):
                    del out[j]
            else:
                retro.append([d, adj_lobes[0]])
        for d, l in retro:
            out[l].add(unit, d, values[d], w[d])
        result = []
        for lobe in out:
            if lobe.neg or lobe.integral < self.integral_threshold:
                continue
            for pi in range(len(lobe.peaks)):
                val, u = get_peak(sh, self.lmax, lobe.peaks[pi], self.al)
                if math.isfinite(val) and np.isfinite(u).all():
                    max_dp, nearest = 0.0, len(lobe.peaks)
                    for j, p in enumerate(lobe.peaks):
                        dp = abs(float(u @ p))
                        if dp > max_dp:
                            max_dp, nearest = dp, j
                    if nearest == pi and self.lookup.select_direction(u) in lobe.mask:
                        lobe.peaks[pi] = u
                        if pi == 0:
                            lobe.max_peak = val
            if lobe.max_peak < self.peak_value_threshold:
                continue
            nrm = float(lobe.mean @ lobe.mean)
            mean = lobe.mean / math.sqrt(nrm) if nrm > 0.0 else lobe.mean
            result.append({"mean_dir": mean, "peak_dir": lobe.peaks[0], "integral": lobe.integral,
                           "max_peak": lobe.max_peak})
        return result


def fod2fixel(fod_rows, lmax, mask=None, maxnum=0, dirpeak=False, **thresholds):
    """fod2fixel for rows of SH coefficients [n][nsh] (voxel order): per voxel
    counts [n], and per fixel [dir x y z, afd, peak_amp, disp] in voxel order."""
    seg = Segmenter(lmax, **thresholds)
    counts = np.zeros(len(fod_rows), np.int64)
    fixels = []
    for v, row in enumerate(np.asarray(fod_rows, np.float64)):
        if mask is not None and not mask[v]:
            continue
        lobes = seg(row)
        if maxnum:
            lobes = lobes[:maxnum]
        counts[v] = len(lobes)
        for lb in lobes:
            d = np.asarray(lb["peak_dir"] if dirpeak else lb["mean_dir"], np.float32)
            afd, pk = np.float32(lb["integral"]), np.float32(lb["max_peak"])
            fixels.append([d[0], d[1], d[2], afd, pk, np.float32(afd / pk)])
    return counts, np.array(fixels, np.float32).reshape(-1, 6)


def _clib():
    """liboracle_fmls.so (oracle/fmls_oracle.c): the segmenter in C, threaded."""
    global _CLIB
    if _CLIB is None:
        so = os.path.join(HERE, "liboracle_fmls.so")
        src = os.path.join(HERE, "fmls_oracle.c")
        if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", HERE, so])
        L = ctypes.CDLL(so)
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.oracle_fmls_segment.restype = ci
        L.oracle_fmls_segment.argtypes = [ci, ci, ci, vp, vp, vp, vp, vp, ci, ci, cd, vp, ci, ci, cd, cd, cd, cd, vp,
                                          vp, cd, cd, cd, vp, ctypes.c_long, ci, vp, vp, ci]
        _CLIB = L
    return _CLIB


def segment_batch_c(seg: Segmenter, rows, max_out: int = 16, nthreads: int = 1):
    """Segmenter.__call__ for every row of ``rows`` [n][nsh] by the C
    restatement (oracle/fmls_oracle.c): (counts [n], fixels [n][max_out][8]:
    mean dir, peak dir, integral, max peak; float32)."""
    rows = np.ascontiguousarray(rows, np.float64)
    unit = np.ascontiguousarray(seg.unit, np.float64)
    adj_off = np.zeros(len(seg.adj) + 1, np.int32)
    adj_off[1:] = np.cumsum([len(a) for a in seg.adj])
    adj = np.concatenate(seg.adj).astype(np.int32)
    w = np.ascontiguousarray(seg.weights, np.float64)
    sh2amp = np.ascontiguousarray(seg.sh2amp, np.float64)
    al = np.ascontiguousarray(seg.al.table, np.float64)
    lk = seg.lookup
    counts = np.zeros(len(rows), np.int32)
    fixels = np.zeros((len(rows), max_out, 8), np.float32)
    p = lambda a: a.ctypes.data  # noqa: E731
    rc = _clib().oracle_fmls_segment(len(unit), seg.lmax, sh2amp.shape[1], p(unit), p(w), p(adj_off), p(adj),
                                     p(sh2amp), al.shape[0], al.shape[1], seg.al.inc, p(al), lk.num_az, lk.num_el,
                                     lk.az_begin, lk.el_begin, lk.az_step, lk.el_step, p(lk.offsets), p(lk.entries),
                                     seg.integral_threshold, seg.peak_value_threshold, seg.merge_ratio, p(rows),
                                     len(rows), max_out, p(counts), p(fixels), int(nthreads))
    if rc != 0:
        raise RuntimeError("oracle_fmls_segment failed")
    return counts, fixels
