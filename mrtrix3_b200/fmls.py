"""``fod2fixel``'s FMLS segmenter on the GPU: host side (tables and the
binding of csd_fmls_*).

``FMLSTables(lmax)`` holds what Segmenter's constructor builds
(src/dwi/fmls.cpp:118-140): the 1281-direction set with its hull adjacency
and FastLookupSet grid, the integration weights, the SH -> amplitude matrix
of lmax and the PrecomputedAL table of 2 x 1281 elevations, as flat numpy
arrays in the layout of ``csd_fmls_tables`` (include/csd_b200.h).
``Segmenter`` uploads them once and segments device rows of SH coefficients
in one kernel launch (fmls.cu).
"""
from __future__ import annotations

import ctypes
import functools
import math

import numpy as np

from . import directions, sh

INTEGRAL_THRESHOLD_DEFAULT = 0.0   # fmls.h: FMLS_INTEGRAL_THRESHOLD_DEFAULT
PEAK_VALUE_THRESHOLD_DEFAULT = 0.1  # fmls.h: FMLS_PEAK_VALUE_THRESHOLD_DEFAULT
MERGE_RATIO_DEFAULT = 1.0           # fmls.h: FMLS_MERGE_RATIO_BRIDGE_TO_PEAK_DEFAULT
FIXEL_FIELDS = 8                    # mean dir (3), peak dir (3), integral, max peak


@functools.lru_cache(maxsize=None)
def _direction_set():
    """The lmax-independent tables of the 1281-direction set, built once per
    process: unit vectors, neighbour lists (CSR), integration weights, the
    lookup grid."""
    unit = np.ascontiguousarray(directions.unit_vectors(directions.load_tessellation_1281()))
    adj = directions.adjacency_1281()
    adj_off = np.zeros(len(unit) + 1, np.int32)
    adj_off[1:] = np.cumsum([len(a) for a in adj])
    weight = np.ascontiguousarray(directions.integration_weights(unit))
    look = directions.FastLookup(unit, adj)
    for a in (unit, adj_off, weight, look.offsets, look.entries):
        a.setflags(write=False)
    return unit, adj_off, np.concatenate(adj).astype(np.int32), weight, look


@functools.lru_cache(maxsize=None)
def _lmax_tables(lmax: int):
    """The SH -> amplitude matrix and PrecomputedAL table of one lmax."""
    unit = _direction_set()[0]
    az = np.arctan2(unit[:, 1], unit[:, 0])
    el = np.arccos(unit[:, 2])
    sh2amp = np.ascontiguousarray(sh.init_transform(np.stack([az, el], axis=1), lmax))
    al = np.ascontiguousarray(directions.precomputed_al(lmax, 2 * len(unit)))
    sh2amp.setflags(write=False)
    al.setflags(write=False)
    return sh2amp, al


class FMLSTables:
    def __init__(self, lmax: int, integral_threshold: float = INTEGRAL_THRESHOLD_DEFAULT,
                 peak_value_threshold: float = PEAK_VALUE_THRESHOLD_DEFAULT,
                 merge_ratio: float = MERGE_RATIO_DEFAULT):
        if lmax < 0 or lmax % 2 or lmax > 16:
            raise ValueError("fod2fixel: lmax must be even and at most 16")
        self.lmax = lmax
        self.nsh = sh.n_for_l(lmax)
        self.unit, self.adj_off, self.adj, self.weight, look = _direction_set()
        self.ndir = len(self.unit)
        self.sh2amp, self.al = _lmax_tables(lmax)
        self.al_ndir = self.al.shape[0]
        self.n_al = self.al.shape[1]
        self.al_inc = math.pi / (self.al_ndir - 1)
        self.num_az, self.num_el = look.num_az, look.num_el
        self.az_begin, self.el_begin = look.az_begin, look.el_begin
        self.az_step, self.el_step = look.az_step, look.el_step
        self.grid_off, self.grid = look.offsets, look.entries
        self.integral_threshold = float(integral_threshold)
        self.peak_value_threshold = float(peak_value_threshold)
        self.merge_ratio = float(merge_ratio)


class _CTables(ctypes.Structure):
    """csd_fmls_tables (include/csd_b200.h)."""
    _fields_ = [("ndir", ctypes.c_int), ("lmax", ctypes.c_int), ("nsh", ctypes.c_int),
                ("unit", ctypes.c_void_p), ("weight", ctypes.c_void_p), ("adj_off", ctypes.c_void_p),
                ("adj", ctypes.c_void_p), ("n_adj", ctypes.c_int), ("sh2amp", ctypes.c_void_p),
                ("al_ndir", ctypes.c_int), ("n_al", ctypes.c_int), ("al_inc", ctypes.c_double),
                ("al", ctypes.c_void_p), ("num_az", ctypes.c_int), ("num_el", ctypes.c_int),
                ("az_begin", ctypes.c_double), ("el_begin", ctypes.c_double), ("az_step", ctypes.c_double),
                ("el_step", ctypes.c_double), ("grid_off", ctypes.c_void_p), ("grid", ctypes.c_void_p),
                ("n_grid", ctypes.c_int), ("integral_threshold", ctypes.c_double),
                ("peak_value_threshold", ctypes.c_double), ("merge_ratio", ctypes.c_double)]


def c_tables(t: FMLSTables) -> _CTables:
    """The host tables as a csd_fmls_tables struct (the arrays stay owned by t)."""
    p = lambda a: a.ctypes.data  # noqa: E731
    return _CTables(t.ndir, t.lmax, t.nsh, p(t.unit), p(t.weight), p(t.adj_off), p(t.adj), len(t.adj), p(t.sh2amp),
                    t.al_ndir, t.n_al, t.al_inc, p(t.al), t.num_az, t.num_el, t.az_begin, t.el_begin, t.az_step,
                    t.el_step, p(t.grid_off), p(t.grid), len(t.grid), t.integral_threshold,
                    t.peak_value_threshold, t.merge_ratio)


class Segmenter:
    """FMLS::Segmenter (fmls.h:244-291) on the current CUDA device: the tables
    uploaded once (csd_fmls_create); ``segment`` runs csd_fmls_segment."""

    def __init__(self, lmax: int, integral_threshold: float = INTEGRAL_THRESHOLD_DEFAULT,
                 peak_value_threshold: float = PEAK_VALUE_THRESHOLD_DEFAULT,
                 merge_ratio: float = MERGE_RATIO_DEFAULT, builtin: bool = False):
        """builtin: let the library build the tables itself
        (csd_fmls_create_default) instead of passing these host tables."""
        from . import csd
        self.tables = FMLSTables(lmax, integral_threshold, peak_value_threshold, merge_ratio)
        self._lib = csd.lib()
        h = ctypes.c_void_p()
        if builtin:
            csd.check(self._lib.csd_fmls_create_default(lmax, float(integral_threshold), float(peak_value_threshold),
                                                        float(merge_ratio), ctypes.byref(h)))
        else:
            ct = c_tables(self.tables)
            csd.check(self._lib.csd_fmls_create(ctypes.byref(ct), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.csd_fmls_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def segment(self, fod, mask=None, max_fixels: int = 0, stream=None):
        """Lobes of every voxel of ``fod`` (device float [n][nsh], strided
        rows allowed): (counts device int32 [n], fixels device float
        [n][m][8]: mean dir (3), peak dir (3), integral, max peak).
        max_fixels > 0 keeps at most that many lobes a voxel (-maxnum);
        0 keeps them all (voxels with more than 16 run again with room)."""
        import torch

        from . import csd
        n = fod.shape[0]
        if fod.dim() != 2 or fod.shape[1] < self.tables.nsh:
            raise ValueError(f"fod2fixel: expected [n][>= {self.tables.nsh}] SH coefficients")
        if fod.dtype != torch.float32:
            raise ValueError("fod2fixel: SH coefficients must be float32")
        dev = fod.device
        m = None if mask is None else mask.to(device=dev, dtype=torch.uint8).contiguous()
        cap = max_fixels if max_fixels > 0 else 16
        counts = torch.empty(n, dtype=torch.int32, device=dev)
        fixels = torch.zeros((n, cap, FIXEL_FIELDS), dtype=torch.float32, device=dev)
        sp = csd._stream_ptr(stream)

        def run(rows, msk, cnt, fx, width):
            csd.check(self._lib.csd_fmls_segment(
                self._h, ctypes.c_void_p(rows.data_ptr()), rows.shape[0], rows.stride(0), rows.stride(1),
                ctypes.c_void_p(msk.data_ptr()) if msk is not None else None, width,
                ctypes.c_void_p(cnt.data_ptr()), ctypes.c_void_p(fx.data_ptr()), ctypes.c_void_p(sp)))

        run(fod, m, counts, fixels, cap)
        if max_fixels > 0:
            return torch.clamp(counts, max=max_fixels), fixels
        over = torch.nonzero(counts > cap).flatten()
        if over.numel():
            width = int(counts.max().item())
            rows = fod.index_select(0, over)
            c2 = torch.empty(over.numel(), dtype=torch.int32, device=dev)
            f2 = torch.zeros((over.numel(), width, FIXEL_FIELDS), dtype=torch.float32, device=dev)
            run(rows, None, c2, f2, width)
            wide = torch.zeros((n, width, FIXEL_FIELDS), dtype=torch.float32, device=dev)
            wide[:, :cap] = fixels
            wide[over] = f2
            fixels = wide
        return counts, fixels


def pack(counts, fixels, dirpeak: bool = False):
    """fod2fixel's receiver (cmd/fod2fixel.cpp:109-125, 250-286) on host
    arrays: per voxel [count, offset] with fixels contiguous in voxel order,
    and per fixel its direction (mean, or peak with -dirpeak), AFD
    (integral), peak amplitude and dispersion (integral / peak, in float)."""
    counts = np.asarray(counts, np.int64)
    fixels = np.asarray(fixels, np.float32)
    offsets = np.zeros_like(counts)
    offsets[1:] = np.cumsum(counts)[:-1]
    sel = np.arange(fixels.shape[1])[None, :] < counts[:, None]
    flat = fixels[sel]
    d = flat[:, 3:6] if dirpeak else flat[:, 0:3]
    afd, peak = flat[:, 6], flat[:, 7]
    with np.errstate(divide="ignore", invalid="ignore"):
        disp = (afd / peak).astype(np.float32)
    return counts, offsets, np.ascontiguousarray(d), afd.copy(), peak.copy(), disp
