"""TEST INFRASTRUCTURE ONLY: ctypes binding to the FP64 CSD oracle.

liboracle_csd.so (oracle/csd_oracle.c) restates MRtrix3's CSD::Shared::init
(src/dwi/sdeconv/csd.h:117-198) and the per-voxel set/iterate loop
(csd.h:237-269, cmd/dwi2fod.cpp:128-173) in double precision.  Only tests,
the smoke check and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

STATUS_MASKED, STATUS_CONVERGED, STATUS_NITER, STATUS_NONFINITE = 0, 1, 2, 3


def build(force: bool = False) -> str:
    so = os.path.join(HERE, "liboracle_csd.so")
    src = os.path.join(HERE, "csd_oracle.c")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, os.path.join(HERE, "liboracle_csd.so")])
    return so


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(build())
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.oracle_shared_init.restype = ctypes.c_int
        L.oracle_shared_init.argtypes = [dp, ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int,
                                         dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_int]
        L.oracle_shared_free.argtypes = [ctypes.c_void_p]
        L.oracle_shared_dims.argtypes = [ctypes.c_void_p, ip]
        L.oracle_shared_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.oracle_shared_dwis.argtypes = [ctypes.c_void_p, ip]
        L.oracle_solve.restype = ctypes.c_int
        L.oracle_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_long, ctypes.c_long,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.oracle_plm_sph.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.oracle_init_transform.argtypes = [dp, ctypes.c_int, ctypes.c_int, dp]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def plm_sph(lmax: int, m: int, x: float) -> np.ndarray:
    a = np.zeros(lmax + 1)
    lib().oracle_plm_sph(_dp(a), lmax, m, x)
    return a


def init_transform(dirs: np.ndarray, lmax: int) -> np.ndarray:
    dirs = np.ascontiguousarray(dirs, np.float64)
    n = (lmax + 1) * (lmax + 2) // 2
    out = np.zeros((dirs.shape[0], n))
    lib().oracle_init_transform(_dp(dirs), dirs.shape[0], lmax, _dp(out))
    return out


class OracleShared:
    """FP64 CSD::Shared.  Keyword names follow the dwi2fod csd options."""

    def __init__(self, grad, response, hr_dirs, lmax: int = 0, filter=None, neg_lambda: float = 1.0,
                 norm_lambda: float = 1.0, threshold: float = 0.0, niter: int = 50,
                 bzero_threshold: float = 10.0, bvalue_epsilon: float = 80.0):
        grad = np.ascontiguousarray(grad, np.float64)
        response = np.ascontiguousarray(response, np.float64)
        hr = np.ascontiguousarray(hr_dirs, np.float64)
        filt = None if filter is None else np.ascontiguousarray(filter, np.float64)
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(256)
        rc = lib().oracle_shared_init(_dp(grad), grad.shape[0], _dp(response), response.size, _dp(hr),
                                      hr.shape[0], int(lmax), None if filt is None else _dp(filt),
                                      0 if filt is None else filt.size, neg_lambda, norm_lambda, threshold,
                                      int(niter), bzero_threshold, bvalue_epsilon, ctypes.byref(h), err, 256)
        if rc:
            raise RuntimeError(err.value.decode())
        self._h = h
        d = (ctypes.c_int * 8)()
        lib().oracle_shared_dims(h, d)
        (self.lmax, self.lmax_response, self.lmax_data, self.n, self.nr, self.ndw, self.nhr,
         self.niter) = list(d)
        self.nvol = grad.shape[0]
        self.nwords = (self.nhr + 31) // 32

    def __del__(self):
        if getattr(self, "_h", None) is not None and _LIB is not None:
            _LIB.oracle_shared_free(self._h)
            self._h = None

    def _mat(self, which, shape):
        out = np.zeros(shape)
        lib().oracle_shared_copy(self._h, which, _dp(out))
        return out

    @property
    def rconv(self):
        return self._mat(0, (self.nr, self.ndw))

    @property
    def M(self):
        return self._mat(1, (self.ndw, self.n))

    @property
    def Mt_M(self):
        L = np.tril(self._mat(2, (self.n, self.n)))
        return L + np.tril(L, -1).T

    @property
    def HR_trans(self):
        return self._mat(3, (self.nhr, self.n))

    @property
    def DW_dirs(self):
        return self._mat(4, (self.ndw, 2))

    @property
    def scalars(self):
        s = np.zeros(3)
        lib().oracle_shared_copy(self._h, 5, _dp(s))
        return {"threshold": s[0], "norm_lambda": s[1], "neg_lambda": s[2]}

    @property
    def dwis(self):
        out = np.zeros(self.ndw, np.int32)
        lib().oracle_shared_dwis(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return out

    def nSH(self):
        return self.n

    def solve(self, dwi: np.ndarray, mask=None, warm=None, nthreads: int = 0):
        """dwi [nvox][nvol] float32 -> dict(F [nvox][n] f64, iters, negmask, status)."""
        dwi = np.ascontiguousarray(dwi, np.float32)
        nvox, nvol = dwi.shape
        assert nvol == self.nvol
        if nthreads <= 0:
            nthreads = os.cpu_count() or 1
        F = np.zeros((nvox, self.n))
        iters = np.zeros(nvox, np.int32)
        neg = np.zeros((nvox, self.nwords), np.uint32)
        status = np.zeros(nvox, np.uint8)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        w = None if warm is None else np.ascontiguousarray(warm, np.uint32)
        lib().oracle_solve(self._h, dwi.ctypes.data, nvox, nvol, 1,
                           None if m is None else m.ctypes.data, None if w is None else w.ctypes.data,
                           F.ctypes.data, iters.ctypes.data, neg.ctypes.data, status.ctypes.data, nthreads)
        return {"F": F, "iters": iters, "negmask": neg, "status": status}
