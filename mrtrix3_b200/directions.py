"""Direction sets for fod2fixel's FMLS segmenter (host, FP64 numpy).

``load_tessellation_1281`` gives the 1281 [az el] directions
(src/dwi/directions/predefined.cpp), ``unit_vectors`` their unit vectors
(Set::initialise, set.h:130-139), ``hull_adjacency`` the neighbours of each
direction on the convex hull of the directions and their antipodes: a
restatement of Set::initialise_adjacency (src/dwi/directions/set.cpp:83-318)
in its own order -- the same extreme points, the same initial tetrahedron,
faces taken from the back of the list, the horizon's edges in ascending
order -- so that near-degenerate faces split as there.  ``adjacency_1281``
reads the shipped result (data/tessellation_1281_adjacency.txt).
``integration_weights`` restates FMLS::IntegrationWeights (src/dwi/fmls.cpp:
87-110): the weights that integrate every SH basis function up to
LforN(n) + 2 exactly (least squares).  ``FastLookup`` restates
FastLookupSet's azimuth / elevation grid (set.cpp:365-459), whose
``select_direction`` the segmenter uses to check a refined peak, and
``precomputed_al`` the table of SH::PrecomputedAL (core/math/SH.h:399-433).
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import sh

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def load_tessellation_1281() -> np.ndarray:
    """[1281][2] azimuth / elevation of the shipped tessellation."""
    return np.loadtxt(os.path.join(DATA, "tessellation_1281.txt"), dtype=np.float64)


def unit_vectors(az_el: np.ndarray) -> np.ndarray:
    az, el = az_el[:, 0], az_el[:, 1]
    s = np.sin(el)
    return np.stack([np.cos(az) * s, np.sin(az) * s, np.cos(el)], axis=1)


def adjacency_1281():
    with open(os.path.join(DATA, "tessellation_1281_adjacency.txt")) as f:
        return [np.array([int(v) for v in line.split()], np.int64) for line in f if not line.startswith("#")]


def _plane(V, i, j, k):
    n = np.cross(V[j] - V[i], V[k] - V[j])
    n = n / np.linalg.norm(n)
    return (i, j, k), n, max(V[i] @ n, V[j] @ n, V[k] @ n)


def hull_adjacency(dirs: np.ndarray):
    """Set::initialise_adjacency: sorted neighbour lists of each direction."""
    n = len(dirs)
    V = np.empty((2 * n, 3))
    V[0::2] = dirs
    V[1::2] = -dirs
    index = np.repeat(np.arange(n), 2)
    # extreme points per axis (strict comparisons from 1 / -1)
    ext = [[0, 0], [0, 0], [0, 0]]
    val = [[1.0, -1.0], [1.0, -1.0], [1.0, -1.0]]
    for i in range(2 * n):
        for ax in range(3):
            if V[i, ax] < val[ax][0]:
                val[ax][0], ext[ax][0] = V[i, ax], i
            if V[i, ax] > val[ax][1]:
                val[ax][1], ext[ax][1] = V[i, ax], i
    extrema = [ext[0][0], ext[0][1], ext[1][0], ext[1][1], ext[2][0], ext[2][1]]
    best, pair = 0.0, (0, 0)
    for i in range(6):
        for j in range(i + 1, 6):
            d = np.sum((V[extrema[j]] - V[extrema[i]]) ** 2)
            if d > best:
                best, pair = d, (i, j)
    third, best = 6, 0.0
    a, b = V[extrema[pair[0]]], V[extrema[pair[1]]]
    for i in range(6):
        if i not in pair:
            p = V[extrema[i]]
            d = np.linalg.norm(np.cross(p - a, p - b)) / np.linalg.norm(b - a)
            if d > best:
                best, third = d, i
    base = _plane(V, extrema[pair[0]], extrema[pair[1]], extrema[third])
    dots = V @ (-base[1])
    fourth = int(np.argmax(dots)) if dots.max() > 0.0 else 2 * n
    i0, i1, i2 = base[0]
    planes = [base, _plane(V, i0, fourth, i1), _plane(V, i1, fourth, i2), _plane(V, i2, fourth, i0)]
    assigned = np.zeros(2 * n, bool)
    assigned[[i0, i1, i2, fourth]] = True
    hull = []
    while planes:
        idx, nrm, dist = planes[-1]
        cand = np.where(assigned, -np.inf, V @ nrm)
        m = int(np.argmax(cand))  # the first of the largest, as the strict scan there
        if not cand[m] > dist:
            hull.append(planes.pop())
            continue
        vm = V[m]
        visible = [p for p in range(len(planes)) if m not in planes[p][0] and vm @ planes[p][1] > planes[p][2]]
        horizon = set()
        for p in visible:
            t = planes[p][0]
            for e in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
                if (e[1], e[0]) in horizon:
                    horizon.discard((e[1], e[0]))
                else:
                    horizon.add(e)
        for e in sorted(horizon):
            planes.append(_plane(V, e[0], e[1], m))
        vis = set(visible)
        planes = [pl for p, pl in enumerate(planes) if p not in vis]
        assigned[m] = True
    adj = [[] for _ in range(n)]
    for t, _, _ in hull:
        for f, g in ((t[0], t[1]), (t[1], t[0]), (t[1], t[2]), (t[2], t[1]), (t[0], t[2]), (t[2], t[0])):
            a_, b_ = int(index[f]), int(index[g])
            if b_ not in adj[a_]:
                adj[a_].append(b_)
    return [np.array(sorted(a), np.int64) for a in adj]


def integration_weights(dirs_unit: np.ndarray) -> np.ndarray:
    """FMLS::IntegrationWeights (src/dwi/fmls.cpp:87-110): w with
    sum_d w_d Y_k(d) = integral of Y_k over the sphere for every basis
    function up to lmax LforN(n) + 2 (2 sqrt(pi) for Y_00, 0 otherwise),
    in the least-squares sense."""
    n = len(dirs_unit)
    lmax = sh.l_for_n(n) + 2
    az = np.arctan2(dirs_unit[:, 1], dirs_unit[:, 0])
    el = np.arccos(dirs_unit[:, 2])
    A = sh.init_transform(np.stack([az, el], axis=1), lmax).T  # [basis][dirs]
    rhs = np.zeros(A.shape[0])
    rhs[0] = 2.0 * np.sqrt(np.pi)
    w, *_ = np.linalg.lstsq(A, rhs, rcond=None)
    return w


class FastLookup:
    """FastLookupSet (set.cpp:365-459): directions binned on an [az el] grid
    whose step is the mean angle between adjacent directions; each cell lists
    its own directions, those nearest its four corners and all their
    neighbours (ascending).  ``select_direction`` searches the cell of p."""

    def __init__(self, unit: np.ndarray, adj):
        self.unit = np.asarray(unit, np.float64)
        n = len(self.unit)
        s, c = 0.0, 0
        for i in range(n):
            for j in adj[i]:
                if j > i:
                    s += abs(float(self.unit[i] @ self.unit[j]))
                    c += 1
        step = math.acos(s / c)
        self.num_az = int(math.ceil(2.0 * math.pi / step))
        self.num_el = int(math.ceil(math.pi / step))
        self.az_step = 2.0 * math.pi / (self.num_az - 1)
        self.el_step = math.pi / (self.num_el - 1)
        self.az_begin, self.el_begin = -math.pi, 0.0
        cells = [[] for _ in range(self.num_az * self.num_el)]
        for i in range(n):
            cells[self.cell(self.unit[i])].append(i)
        for i, cell in enumerate(cells):
            ai, ei = divmod(i, self.num_el)
            for da, de in ((0, 0), (1, 0), (1, 1), (0, 1)):
                az = self.az_begin + ai * self.az_step + da * self.az_step
                el = self.el_begin + ei * self.el_step + de * self.el_step
                p = np.array([math.cos(az) * math.sin(el), math.sin(az) * math.sin(el), math.cos(el)])
                nearest = int(np.argmax(np.abs(self.unit @ p)))
                if nearest not in cell:
                    cell.append(nearest)
        for cell in cells:
            for d in list(cell):
                for a in adj[d]:
                    if a not in cell:
                        cell.append(int(a))
            cell.sort()
        self.cells = cells
        self.offsets = np.zeros(len(cells) + 1, np.int32)
        self.offsets[1:] = np.cumsum([len(c) for c in cells])
        self.entries = np.array([d for c in cells for d in c], np.int32)

    def cell(self, p) -> int:
        az = math.atan2(p[1], p[0])
        el = math.acos(p[2])
        return int(math.floor((az - self.az_begin) / self.az_step)) * self.num_el + \
            int(math.floor((el - self.el_begin) / self.el_step))

    def select_direction(self, p) -> int:
        cell = self.cells[self.cell(p)]
        best, best_dp = cell[0], abs(float(np.dot(p, self.unit[cell[0]])))
        for d in cell[1:]:
            dp = abs(float(np.dot(p, self.unit[d])))
            if dp > best_dp:
                best, best_dp = d, dp
        return best


def precomputed_al(lmax: int, ndir: int) -> np.ndarray:
    """SH::PrecomputedAL's table (SH.h:416-433): [ndir][NforL_mpos(lmax)]
    normalised associated Legendre values at elevations n pi / (ndir - 1),
    entry (l, m) at l^2/4 + m for even l."""
    n_al = (lmax // 2 + 1) ** 2
    inc = math.pi / (ndir - 1)
    z = np.cos(np.arange(ndir) * inc)
    out = np.zeros((ndir, n_al))
    for m in range(lmax + 1):
        P = sh.plm_sph(lmax, m, z)
        for l in range(m + (m & 1), lmax + 1, 2):
            out[:, l * l // 4 + m] = P[l]
    return out
