"""Multi-shell multi-tissue CSD (``dwi2fod msmt_csd``) on the GPU.

``MSMTShared`` mirrors MSMT_CSD::Shared (src/dwi/sdeconv/msmt_csd.h:43-241):
construct from the gradient table (every b-value shell kept,
select_shells(false, false, false)), ``parse_cmdline_options``,
``set_responses`` (one [shells][even-order zonal coefficients] matrix per
tissue; trailing all-zero columns clipped, prepare_responses :222-237),
``init`` (:90-211): per tissue lmax (default min(8, lmax of its response)),
the forward matrix C [volumes][parameters] (each shell's volumes get the SH
basis at their directions times the tissue's response on that shell divided
by the zonal basis value at the pole), and the non-negativity constraints A
(each tissue's amplitudes on the 300 constraint directions, or its l = 0
term when its lmax is 0).  The constrained least-squares problem is set up
and solved by the library (csd_icls_create / csd_icls_solve), in FP64.

Host set-up in FP64 numpy; the scheme normalisation and shell clustering
follow dwi/gradient.cpp:286-310 and dwi/shells.cpp:300-411 as the library's
single-shell set-up does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import csd, sh

DEFAULT_LMAX = 8
DEFAULT_NORM_LAMBDA = 1.0e-10
DEFAULT_NEG_LAMBDA = 1.0e-10
SHELLS_MIN_LINKAGE = 3


def normalise_scheme(grad) -> np.ndarray:
    """dwi/gradient.cpp:286-310: unit directions; b scaled by |g|^2 when the
    norms stray from 1 by more than exp(0.01)."""
    g = np.array(grad, np.float64, copy=True)
    if g.ndim != 2 or g.shape[1] != 4:
        raise ValueError("gradient table must be [volumes][4]")
    sq = np.sum(g[:, :3] ** 2, axis=1)
    nz = sq > 0
    g[nz, :3] /= np.sqrt(sq[nz])[:, None]
    maxlog = np.max(np.where(nz, np.abs(np.log(np.where(nz, sq, 1.0))), 0.0)) if len(g) else 0.0
    if maxlog > 0.01:
        g[:, 3] *= sq
    return g


def cluster_shells(b, bzero_threshold: float = 10.0, bvalue_epsilon: float = 80.0):
    """Shells::Shells (dwi/shells.cpp:300-411): [volume index arrays], by
    increasing mean b-value; volumes left unassigned are dropped."""
    b = np.asarray(b, np.float64)
    nvol = len(b)
    clusters = np.zeros(nvol, int)
    visited = np.zeros(nvol, bool)

    def region(bv):
        return [i for i in range(nvol) if b[i] > bzero_threshold and abs(bv - b[i]) < bvalue_epsilon]

    cluster = 0
    for i in range(nvol):
        if b[i] <= bzero_threshold:
            visited[i] = True
            cluster = 1
            clusters[i] = 1
    for i in range(nvol):
        if visited[i]:
            continue
        visited[i] = True
        nb = region(b[i])
        if b[i] > bzero_threshold and len(nb) < SHELLS_MIN_LINKAGE:
            clusters[i] = 0
            continue
        cluster += 1
        clusters[i] = cluster
        q = 0
        while q < len(nb):
            v = nb[q]
            if not visited[v]:
                visited[v] = True
                nb2 = region(b[v])
                if len(nb2) >= SHELLS_MIN_LINKAGE:
                    nb.extend(nb2)
            if clusters[v] == 0:
                clusters[v] = cluster
            q += 1
    if cluster < 1 or cluster > np.sqrt(nvol):
        raise ValueError("DWI volumes could not be classified into b-value shells; "
                         "gradient encoding may not represent a HARDI sequence")
    shells = [np.nonzero(clusters == s)[0] for s in range(1, cluster + 1)]
    shells = [v for v in shells if len(v)]
    shells.sort(key=lambda v: float(np.mean(b[v])))
    return shells


def _shell_stats(b, vols):
    """Shell::Shell (dwi/shells.cpp:52-70): mean, sample stdev, min and --
    as computed there -- "max" = max(running min, b) of the last volume."""
    bv = np.asarray(b, np.float64)[np.asarray(vols)]
    mean = float(bv.mean())
    with np.errstate(invalid="ignore", divide="ignore"):
        stdev = float(np.sqrt(np.sum((bv - mean) ** 2) / (len(bv) - 1))) if len(bv) > 1 else float("nan")
    lo = hi = np.inf
    for x in bv:
        lo = min(lo, x)
        hi = max(lo, x)
    return mean, stdev, float(lo), float(hi)


def select_shells(b, shells, requested, bzero_threshold: float = 10.0):
    """Shells::select_shells with the -shells option (dwi/shells.cpp:100-215):
    the indices of the shells to keep for the requested b-values."""
    b = np.asarray(b, np.float64)
    stats = [_shell_stats(b, v) for v in shells]
    has_b0 = stats[0][0] <= bzero_threshold
    keep = [False] * len(shells)
    b0_selected = False

    def take(s, stat):
        if keep[s]:
            raise ValueError(f"User selected a shell more than once: {stat[0]} +- {stat[1]} with {len(shells[s])} "
                             "volumes")
        keep[s] = True

    for want in requested:
        want = float(want)
        if want < 0:
            raise ValueError("Cannot select shells corresponding to negative b-values")
        if want <= bzero_threshold:
            if not has_b0:
                raise ValueError("User selected b=0 shell, but no such data was found")
            if b0_selected:
                raise ValueError("User selected b=0 shell more than once")
            keep[0] = True
            b0_selected = True
            continue
        selected = False
        for s, st in enumerate(stats):
            if st[2] <= want <= st[3]:
                take(s, st)
                selected = True
        if selected:
            continue
        near = [s for s, st in enumerate(stats) if abs(want - st[0]) <= 1.0]
        if len(near) == 1:
            take(near[0], stats[near[0]])
            continue
        zero_stdev = any(not (st[0] <= bzero_threshold) and st[1] < 1.0 for st in stats)
        best, best_n, ambiguous = 0, np.inf, False
        for s, st in enumerate(stats):
            sd = 0.5 * bzero_threshold if st[0] <= bzero_threshold else (np.sqrt(st[0]) if zero_stdev else st[1])
            n = abs((want - st[0]) / sd)
            if n < best_n:
                ambiguous = n >= 0.1 * best_n
                best, best_n = s, n
            else:
                ambiguous = n < 10.0 * best_n
        if ambiguous:
            raise ValueError(f"Unable to robustly select desired shell b={want:g} (detected shells are: "
                             + ", ".join(f"{st[0]:g} +- {st[1]:g}" for st in stats) + ")")
        take(best, stats[best])
    return [s for s in range(len(shells)) if keep[s]]


def direction_matrix(grad, vols) -> np.ndarray:
    """DWI::gen_direction_matrix (gradient.h:77-95): [az el] per volume; a
    zero vector gives a NaN elevation, as there."""
    g = np.asarray(grad, np.float64)[np.asarray(vols)]
    az = np.arctan2(g[:, 1], g[:, 0])
    with np.errstate(invalid="ignore", divide="ignore"):
        z = g[:, 2] / np.linalg.norm(g[:, :3], axis=1)
        el = np.where(z >= 1.0, 0.0, np.where(z <= -1.0, np.pi, np.arccos(np.clip(z, -1.0, 1.0))))
    el = np.where(np.isnan(z), np.nan, el)
    return np.stack([az, el], axis=1)


def _transform_nan0(dirs, lmax):
    with np.errstate(invalid="ignore"):
        m = sh.init_transform(dirs, lmax)
    return np.where(np.isnan(m), 0.0, m)


def load_hr_dirs() -> np.ndarray:
    """The built-in 300 [az, el] constraint directions."""
    return np.loadtxt(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                   "electrostatic_repulsion_300.txt"), dtype=np.float64)


class MSMTShared:
    """MSMT_CSD::Shared.  ``grad`` is the [volumes][4] gradient table."""

    def __init__(self, grad, bzero_threshold: float = 10.0, bvalue_epsilon: float = 80.0, shells=None):
        """``shells``: the -shells b-values to keep (select_shells); default all."""
        self.grad = normalise_scheme(grad)
        self.shells = cluster_shells(self.grad[:, 3], bzero_threshold, bvalue_epsilon)
        if shells is not None:
            keep = select_shells(self.grad[:, 3], self.shells, shells, bzero_threshold)
            self.shells = [self.shells[i] for i in keep]
        self.HR_dirs = load_hr_dirs()
        self.lmax = None
        self.lmax_response = []
        self.responses = []
        self.solution_min_norm_regularisation = DEFAULT_NORM_LAMBDA
        self.constraint_min_norm_regularisation = DEFAULT_NEG_LAMBDA
        self._h = None

    def parse_cmdline_options(self, lmax=None, directions=None, norm_lambda=None, neg_lambda=None):
        """msmt_csd.h:57-71."""
        if lmax is not None:
            self.lmax = [int(v) for v in np.ravel(lmax)]
        if directions is not None:
            self.HR_dirs = np.ascontiguousarray(directions, np.float64)
        if norm_lambda is not None:
            self.solution_min_norm_regularisation = float(norm_lambda)
        if neg_lambda is not None:
            self.constraint_min_norm_regularisation = float(neg_lambda)

    def set_responses(self, responses):
        """msmt_csd.h:75-95 with prepare_responses (:222-237): a path or a
        [shells][coefficients] matrix per tissue."""
        from . import mif
        self.responses, self.lmax_response = [], []
        for r in responses:
            m = mif.load_matrix(r) if isinstance(r, (str, os.PathLike)) else np.array(r, np.float64, ndmin=2)
            nz = np.nonzero(np.any(m != 0.0, axis=0))[0]
            m = m[:, :nz[-1] + 1] if len(nz) else m[:, :0]
            self.responses.append(m)
            self.lmax_response.append(2 * (m.shape[1] - 1) if m.shape[1] else 0)

    def num_shells(self) -> int:
        return len(self.shells)

    def num_tissues(self) -> int:
        return len(self.responses)

    def nparams(self):
        return [sh.n_for_l(l) for l in self.lmax]

    def init(self, upload: bool = True):
        """msmt_csd.h:90-211: the forward and constraint matrices, then (with
        ``upload``) the constrained least-squares problem on the device."""
        if not self.responses:
            raise ValueError("no response functions set")
        if self.lmax is None:
            self.lmax = [min(DEFAULT_LMAX, l) for l in self.lmax_response]
        else:
            if len(self.lmax) != self.num_tissues():
                raise ValueError(f"Number of lmaxes specified ({len(self.lmax)}) does not match number of tissues "
                                 f"({self.num_tissues()})")
            if any(l % 2 or l < 0 for l in self.lmax):
                raise ValueError("Each value of lmax must be a non-negative even integer")
        resp = []
        for t, r in enumerate(self.responses):
            if r.shape[0] != self.num_shells():
                raise ValueError("number of rows in response functions must match number of b-value shells; "
                                 f"number of shells is {self.num_shells()}, but response {t} contains "
                                 f"{r.shape[0]} rows")
            nz = self.lmax[t] // 2 + 1
            p = np.zeros((self.num_shells(), nz))
            k = min(nz, r.shape[1])
            p[:, :k] = r[:, :k]
            resp.append(p)
        n = self.nparams()
        N = int(sum(n))
        maxlmax = max(self.lmax)
        nvol = self.grad.shape[0]
        SHT = _transform_nan0(direction_matrix(self.grad, np.arange(nvol)), maxlmax)
        # zonal basis values at the pole (the non-zero entries of the basis at [0 0])
        dsh_row = sh.init_transform(np.zeros((1, 2)), maxlmax)[0]
        DSH = dsh_row[dsh_row != 0.0]
        C = np.zeros((nvol, N))
        pbegin = 0
        for t in range(self.num_tissues()):
            L, nt = self.lmax[t], n[t]
            for s, vols in enumerate(self.shells):
                r = resp[t][s] / DSH[:L // 2 + 1]
                fconv = np.concatenate([np.full(2 * l + 1, r[l // 2]) for l in range(0, L + 1, 2)])
                C[np.ix_(vols, np.arange(pbegin, pbegin + nt))] = SHT[vols, :nt] * fconv
            pbegin += nt
        HR_SHT = sh.init_transform(self.HR_dirs, maxlmax)
        m = [len(self.HR_dirs) if l > 0 else 1 for l in self.lmax]
        A = np.zeros((int(sum(m)), N))
        bm = bn = 0
        for t in range(self.num_tissues()):
            A[bm:bm + m[t], bn:bn + n[t]] = HR_SHT[:m[t], :n[t]]
            bm += m[t]
            bn += n[t]
        self.C, self.A = C, A
        self.release()
        if not upload:
            return self
        h = ctypes.c_void_p()
        C_ = np.ascontiguousarray(C)
        A_ = np.ascontiguousarray(A)
        csd.check(csd.lib().csd_icls_create(C_.ctypes.data, C.shape[0], N, A_.ctypes.data, A.shape[0], None, 0,
                                            self.solution_min_norm_regularisation,
                                            self.constraint_min_norm_regularisation, 0, 0.0, ctypes.byref(h)))
        self._h = h
        return self

    @property
    def handle(self):
        if self._h is None:
            raise csd.CSDError("MSMTShared.init() has not been called")
        return self._h

    def max_niter(self) -> int:
        info = (ctypes.c_int * 4)()
        csd.check(csd.lib().csd_icls_info(self.handle, info))
        return info[3]

    def release(self):
        if self._h is not None:
            csd.lib().csd_icls_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def solve(self, dwi, mask=None, out=None, niter=None, predicted=None, stream=None):
        """MSMT_Processor over every row of ``dwi`` (device float32 [n][volumes],
        any strides): the concatenated tissue ODFs, device float32 [n][N], and
        the solver's rounds per voxel (device int32 [n]); ``predicted``
        (device float32 [n][volumes], optional) receives C x."""
        return icls_solve(self.handle, dwi, int(sum(self.nparams())), mask, out, niter, stream, predicted)

    def solve_host(self, dwi: np.ndarray, mask: np.ndarray | None = None, predicted: bool = False):
        """``solve`` on host arrays through csd_icls_solve_host (synchronous):
        (x [n][N] float32, rounds [n] int32, predicted [n][volumes] or None)."""
        dwi = np.ascontiguousarray(dwi, np.float32)
        n = dwi.shape[0]
        x = np.empty((n, int(sum(self.nparams()))), np.float32)
        it = np.empty(n, np.int32)
        pred = np.empty((n, self.grad.shape[0]), np.float32) if predicted else None
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        csd.check(csd.lib().csd_icls_solve_host(self.handle, dwi.ctypes.data, n, dwi.shape[1],
                                                m.ctypes.data if m is not None else None, x.ctypes.data,
                                                it.ctypes.data, pred.ctypes.data if pred is not None else None))
        return x, it, pred

    def split(self, x):
        """The per-tissue parts of a [.., N] solution."""
        out, b = [], 0
        for nt in self.nparams():
            out.append(x[..., b:b + nt])
            b += nt
        return out


def icls_solve(handle, b, nparam: int, mask=None, out=None, niter=None, stream=None, predicted=None):
    import torch
    if b.dim() != 2 or b.dtype != torch.float32 or not b.is_cuda:
        raise ValueError("icls_solve: b must be a float32 CUDA tensor [n][measurements]")
    n = b.shape[0]
    if out is None:
        out = torch.empty((n, nparam), dtype=torch.float32, device=b.device)
    if niter is None:
        niter = torch.empty(n, dtype=torch.int32, device=b.device)
    if mask is not None:
        mask = mask.to(torch.uint8)
    if predicted is not None and (predicted.dtype != torch.float32 or predicted.dim() != 2 or
                                  predicted.shape[0] != n or predicted.stride(1) != 1 or
                                  predicted.device != b.device):
        raise ValueError("icls_solve: predicted must be float32 [n][>= measurements] with contiguous rows")
    csd.check(csd.lib().csd_icls_solve(handle, ctypes.c_void_p(b.data_ptr()), n, b.stride(0), b.stride(1),
                                       ctypes.c_void_p(mask.data_ptr()) if mask is not None else None,
                                       ctypes.c_void_p(out.data_ptr()), out.stride(0),
                                       ctypes.c_void_p(niter.data_ptr()),
                                       ctypes.c_void_p(predicted.data_ptr()) if predicted is not None else None,
                                       predicted.stride(0) if predicted is not None else 0,
                                       ctypes.c_void_p(csd._stream_ptr(stream))))
    return out, niter


class ICLSProblem:
    """Math::ICLS::Problem on the device (csd_icls_create): min ||H x - b||^2
    s.t. A x >= t, the last ``num_eq`` rows of A equalities."""

    def __init__(self, H, A, t=None, num_eq: int = 0, solution_reg: float = 0.0, constraint_reg: float = 0.0,
                 max_niter: int = 0, tol: float = 0.0, standard_form: bool = False):
        """``standard_form``: H is H^T H (square) and the right-hand sides are
        H^T b (constrained_least_squares.h:67-70)."""
        H = np.ascontiguousarray(H, np.float64)
        A = np.ascontiguousarray(A, np.float64)
        t = None if t is None or len(t) == 0 else np.ascontiguousarray(t, np.float64)
        self.nparam = H.shape[1]
        h = ctypes.c_void_p()
        tp = t.ctypes.data if t is not None else None
        if standard_form:
            if H.shape[0] != H.shape[1]:
                raise ValueError("ICLSProblem: a problem in standard form needs a square H^T H")
            csd.check(csd.lib().csd_icls_create_standard(H.ctypes.data, H.shape[1], A.ctypes.data, A.shape[0], tp,
                                                         int(num_eq), float(solution_reg), float(constraint_reg),
                                                         int(max_niter), float(tol), ctypes.byref(h)))
        else:
            csd.check(csd.lib().csd_icls_create(H.ctypes.data, H.shape[0], H.shape[1], A.ctypes.data, A.shape[0],
                                                tp, int(num_eq), float(solution_reg), float(constraint_reg),
                                                int(max_niter), float(tol), ctypes.byref(h)))
        self._h = h

    def solve(self, b, mask=None, out=None, niter=None, stream=None, predicted=None):
        return icls_solve(self._h, b, self.nparam, mask, out, niter, stream, predicted)

    def solve_f64(self, b, stream=None):
        """FP64 right-hand sides (device float64 [n][measurements]) -> FP64
        solutions [n][nparam] and rounds [n] (csd_icls_solve_f64)."""
        import torch
        if b.dim() != 2 or b.dtype != torch.float64 or not b.is_cuda:
            raise ValueError("solve_f64: b must be a float64 CUDA tensor [n][measurements]")
        x = torch.empty((b.shape[0], self.nparam), dtype=torch.float64, device=b.device)
        it = torch.empty(b.shape[0], dtype=torch.int32, device=b.device)
        csd.check(csd.lib().csd_icls_solve_f64(self._h, ctypes.c_void_p(b.data_ptr()), b.shape[0], b.stride(0),
                                               b.stride(1), ctypes.c_void_p(x.data_ptr()), x.stride(0),
                                               ctypes.c_void_p(it.data_ptr()),
                                               ctypes.c_void_p(csd._stream_ptr(stream))))
        return x, it

    def __del__(self):
        try:
            csd.lib().csd_icls_destroy(self._h)
        except Exception:
            pass
