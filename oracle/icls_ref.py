"""TEST INFRASTRUCTURE ONLY: FP64 CPU restatement of MRtrix3's inequality-
constrained least-squares solver (core/math/constrained_least_squares.h),
the checker of the GPU ICLS / MSMT-CSD solver (never imported by the
product path).

Problem (constrained_least_squares.h:90-151): min ||H x - b||^2 subject to
A x >= t (the last ``num_eq`` rows of A as equalities).  Set-up: L = chol(H^T
H + solution_reg * max diag) (lower), b2d = H L^-T, B = A L^-T with each row
and its t entry divided by the row's norm; max_niter = 10 * columns unless
given.

Solver (constrained_least_squares.h:241-370), a dual active-set method in
the preconditioned variable y = L^T x: y_u = b2d^T b, c_u = B y_u - t; while
the most violated inequality has c < -tol: activate it, then repeatedly
solve (B_a B_a^T + constraint_reg I) l = -c_u[a] over the active rows in
index order, dropping the active inequality whose multiplier first crosses
zero on the segment from the previous multipliers (smallest lambda_prev /
(lambda_prev - l)), until every multiplier is >= 0; then y = y_u + B_a^T l,
c = B y - t.  Stops when the active set did not change or after more than
max_niter rounds; x = L^-T y.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_CLIB = None


class Problem:
    def __init__(self, H, A, t=None, num_eq: int = 0, solution_reg: float = 0.0, constraint_reg: float = 0.0,
                 max_niter: int = 0, tol: float = 0.0, standard_form: bool = False):
        H = np.asarray(H, np.float64)
        A = np.asarray(A, np.float64)
        if H.shape[1] != A.shape[1]:
            raise ValueError("dimensions of problem and constraint matrices do not match")
        self.H = H
        self.num_eq = int(num_eq)
        self.lambda_min_norm = float(constraint_reg)
        self.tol = float(tol)
        self.max_niter = int(max_niter) if max_niter else 10 * H.shape[1]
        HtH = H.copy() if standard_form else H.T @ H
        HtH = np.tril(HtH)
        HtH = HtH + np.tril(HtH, -1).T
        HtH[np.diag_indices_from(HtH)] += solution_reg * np.max(np.diag(HtH))
        self.L = np.linalg.cholesky(HtH)
        # X L^T = H  ->  X = H L^-T
        rhs = np.eye(H.shape[0], H.shape[1]) if standard_form else H
        self.b2d = np.linalg.solve(self.L, rhs.T).T
        B = np.linalg.solve(self.L, A.T).T
        norms = np.linalg.norm(B, axis=1)
        with np.errstate(invalid="ignore", divide="ignore"):  # a zero row becomes NaN, as there
            self.B = B / norms[:, None]
        self.t = None if t is None or len(t) == 0 else np.asarray(t, np.float64) / norms

    @property
    def num_constraints(self):
        return self.B.shape[0]

    @staticmethod
    def with_equalities(H, A_ineq, A_eq, t_ineq=None, t_eq=None, **kw):
        """The second constructor (constrained_least_squares.h:163-188)."""
        A = np.vstack([A_ineq, A_eq])
        t = None
        if (t_ineq is not None and len(t_ineq)) or (t_eq is not None and len(t_eq)):
            t = np.concatenate([t_ineq, t_eq])
        return Problem(H, A, t, num_eq=len(A_eq), **kw)


def solve(P: Problem, b, trace: list | None = None):
    """Solver::operator() for one right-hand side: (x, niter).  ``trace``
    (optional) receives the active index list after each outer round."""
    b = np.asarray(b, np.float64)
    y_u = P.b2d.T @ b
    c_u = P.B @ y_u
    if P.t is not None:
        c_u = c_u - P.t
    M = P.num_constraints
    num_eq = P.num_eq
    num_ineq = M - num_eq
    lam = np.zeros(M)
    lam_prev = np.zeros(M)
    active = np.zeros(M, bool)
    active[num_ineq:] = True
    c = c_u.copy()
    x = y_u.copy()
    niter = 0
    while num_ineq > 0:
        i_min = _min_coeff(c[:num_ineq])
        if not c[i_min] < -P.tol:
            break
        changed = not active[i_min]
        active[i_min] = True
        while True:
            act = np.nonzero(active)[0]
            Ba = P.B[act]
            BtB = Ba @ Ba.T
            BtB[np.diag_indices_from(BtB)] += P.lambda_min_norm
            Lb = np.linalg.cholesky(BtB)
            l = np.linalg.solve(Lb.T, np.linalg.solve(Lb, -c_u[act]))
            s_min, s_idx = np.inf, 0
            a = 0
            for n in range(num_ineq):
                if active[n]:
                    if l[a] < 0.0:
                        s = lam_prev[n] / (lam_prev[n] - l[a])
                        if s < s_min:
                            s_min, s_idx = s, n
                    lam[n] = l[a]
                    a += 1
                else:
                    lam[n] = 0.0
            if not np.isfinite(s_min):
                x = y_u + Ba.T @ l
                break
            if active[s_idx]:
                changed = True
            active[s_idx] = False
        lam_prev = lam.copy()
        if trace is not None:
            trace.append(np.nonzero(active)[0].copy())
        niter += 1
        if not changed or niter > P.max_niter:
            break
        c = P.B @ x
        if P.t is not None:
            c = c - P.t
    x = np.linalg.solve(P.L.T, x)
    return x, niter


def _min_coeff(v) -> int:
    """Eigen's minCoeff(&index): a scan keeping the first strict minimum, so
    NaN entries are never chosen (unless the first entry is NaN, which then
    stays)."""
    if np.isnan(v[0]):
        return 0
    with np.errstate(invalid="ignore"):
        return int(np.nanargmin(v)) if np.isnan(v).any() else int(np.argmin(v))


def is_approx(x, y, prec: float) -> bool:
    """Eigen's isApprox: ||x - y|| <= prec * min(||x||, ||y||)."""
    return bool(np.linalg.norm(x - y) <= prec * min(np.linalg.norm(x), np.linalg.norm(y)))


def _clib():
    """liboracle_icls.so (oracle/icls_oracle.c): the same solver in C, threaded."""
    global _CLIB
    if _CLIB is None:
        so = os.path.join(HERE, "liboracle_icls.so")
        src = os.path.join(HERE, "icls_oracle.c")
        if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", HERE, so])
        L = ctypes.CDLL(so)
        vp = ctypes.c_void_p
        L.oracle_icls_solve.restype = ctypes.c_int
        L.oracle_icls_solve.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_double, vp, vp, vp, vp, vp, ctypes.c_long, vp, vp,
                                        ctypes.c_int]
        _CLIB = L
    return _CLIB


def solve_batch_c(P: Problem, b, nthreads: int = 1):
    """solve() for every row of ``b`` by the C restatement: (x [n][nparam], niter [n])."""
    b = np.ascontiguousarray(b, np.float64)
    b2d = np.ascontiguousarray(P.b2d)
    B = np.ascontiguousarray(P.B)
    L = np.ascontiguousarray(P.L)
    t = None if P.t is None else np.ascontiguousarray(P.t)
    x = np.zeros((len(b), P.H.shape[1]))
    it = np.zeros(len(b), np.int32)
    rc = _clib().oracle_icls_solve(P.H.shape[0], P.H.shape[1], P.num_constraints, P.num_eq, P.max_niter,
                                   P.lambda_min_norm, P.tol, b2d.ctypes.data, B.ctypes.data,
                                   t.ctypes.data if t is not None else None, L.ctypes.data, b.ctypes.data, len(b),
                                   x.ctypes.data, it.ctypes.data, int(nthreads))
    if rc != 0:
        raise RuntimeError("oracle_icls_solve failed")
    return x, it
