"""Python host mirror of MRtrix3's CSD interface over libcsd_b200.so.

``Shared`` mirrors ``MR::DWI::SDeconv::CSD::Shared`` (src/dwi/sdeconv/csd.h:
46-212): construct from the gradient table, set options (the names of
``dwi2fod csd``'s command-line options, csd.cpp:318-346), ``set_response``,
``init``, ``nSH``.  ``dwi2fod_csd`` is the batched replacement of the
ThreadedLoop over ``CSD_Processor`` (cmd/dwi2fod.cpp:120-176, 275-281).
``CSD`` keeps the per-voxel ``set / iterate / FOD`` surface (csd.h:221-271).

Every call goes through the C ABI declared in include/csd_b200.h.  PyTorch
is used only to hold device memory and streams.  There is no CPU fallback:
if the library or a GPU is missing, these calls raise.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcsd_b200.so")

CSD_OK = 0
CSD_ERR_INVALID, CSD_ERR_CUDA, CSD_ERR_TIMEOUT, CSD_ERR_NOMEM, CSD_ERR_UNSUPPORTED = -1, -2, -3, -4, -5
STATUS_MASKED, STATUS_CONVERGED, STATUS_NITER, STATUS_NONFINITE = 0, 1, 2, 3
STATUS_FP64, STATUS_CHOLFAIL, STATUS_WARM_RESTART = 0x10, 0x20, 0x40

# Every symbol include/csd_b200.h declares.
EXPORTED = [
    "csd_params_init", "csd_shared_create", "csd_shared_destroy", "csd_shared_nsh", "csd_shared_info",
    "csd_shared_dwis", "csd_shared_matrix", "csd_solve", "csd_dwi2fod_host", "csd_state_create",
    "csd_state_destroy", "csd_state_set", "csd_state_warm", "csd_state_iterate", "csd_state_run",
    "csd_state_fod",
    "csd_state_stats", "csd_state_assembly_stats", "csd_dwi2fod_host_phased", "csd_sh2peaks", "csd_amp2sh", "csd_amp2sh_rician", "csd_icls_create",
    "csd_icls_destroy", "csd_icls_info", "csd_icls_solve", "csd_icls_solve_host", "csd_icls_create_standard", "csd_icls_solve_f64",
    "csd_amp2response_accumulate", "csd_dwi2tensor", "csd_fmls_create", "csd_fmls_create_default", "csd_fmls_destroy",
    "csd_fmls_segment",
    "csd_last_error",
]


class CSDError(RuntimeError):
    pass


class csd_params(ctypes.Structure):
    _fields_ = [("lmax", ctypes.c_int), ("niter", ctypes.c_int), ("neg_lambda", ctypes.c_double),
                ("norm_lambda", ctypes.c_double), ("threshold", ctypes.c_double),
                ("filter", ctypes.POINTER(ctypes.c_double)), ("n_filter", ctypes.c_int),
                ("bzero_threshold", ctypes.c_double), ("bvalue_epsilon", ctypes.c_double),
                ("fp64_condition", ctypes.c_double), ("refine", ctypes.c_int),
                ("shells", ctypes.POINTER(ctypes.c_double)), ("n_shells", ctypes.c_int)]


class csd_volume(ctypes.Structure):
    _fields_ = [("dwi", ctypes.c_void_p), ("n_voxels", ctypes.c_int64), ("voxel_stride", ctypes.c_int64),
                ("volume_stride", ctypes.c_int64), ("mask", ctypes.c_void_p), ("warm_negmask", ctypes.c_void_p),
                ("fod", ctypes.c_void_p), ("fod_stride", ctypes.c_int64), ("status", ctypes.c_void_p),
                ("iterations", ctypes.c_void_p), ("negmask", ctypes.c_void_p)]


_LIB = None


def lib():
    """Load libcsd_b200.so (built in-tree by mrtrix3_b200.build)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise CSDError(f"{LIB_PATH} is missing: build it with `python -m mrtrix3_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, dp = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)
        L.csd_params_init.argtypes = [ctypes.POINTER(csd_params)]
        L.csd_params_init.restype = None
        L.csd_shared_create.argtypes = [ctypes.POINTER(csd_params), dp, ctypes.c_int, dp, ctypes.c_int, dp,
                                        ctypes.c_int, ctypes.POINTER(vp)]
        L.csd_shared_destroy.argtypes = [vp]
        L.csd_shared_destroy.restype = None
        L.csd_shared_nsh.argtypes = [vp]
        L.csd_shared_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.csd_shared_dwis.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.csd_shared_matrix.argtypes = [vp, ctypes.c_int, dp]
        L.csd_solve.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(csd_volume), ctypes.c_int, vp]
        L.csd_dwi2fod_host.argtypes = [vp, vp, i64, vp, vp, vp, vp]
        L.csd_state_create.argtypes = [vp, i64, ctypes.POINTER(vp)]
        L.csd_state_destroy.argtypes = [vp]
        L.csd_state_destroy.restype = None
        L.csd_state_set.argtypes = [vp, vp, i64, i64, i64, vp, vp]
        L.csd_state_warm.argtypes = [vp, vp, vp]
        L.csd_state_iterate.argtypes = [vp, ctypes.POINTER(i64), vp]
        L.csd_state_run.argtypes = [vp, ctypes.c_int, ctypes.POINTER(i64), vp]
        L.csd_amp2sh.argtypes = [vp, i64, i64, i64, vp, ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int,
                                 vp, i64, vp]
        L.csd_amp2sh_rician.argtypes = [vp, i64, i64, i64, vp, vp, ctypes.c_int, vp, ctypes.c_int, vp,
                                         ctypes.c_int, ctypes.c_int, vp, i64, vp, i64, vp]
        L.csd_icls_create.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                      ctypes.POINTER(vp)]
        L.csd_icls_destroy.argtypes = [vp]
        L.csd_icls_destroy.restype = None
        L.csd_icls_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.csd_icls_solve.argtypes = [vp, vp, i64, i64, i64, vp, vp, i64, vp, vp, i64, vp]
        L.csd_icls_solve_host.argtypes = [vp, vp, i64, i64, vp, vp, vp, vp]
        L.csd_icls_create_standard.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.POINTER(vp)]
        L.csd_icls_solve_f64.argtypes = [vp, vp, i64, i64, i64, vp, i64, vp, vp]
        L.csd_dwi2tensor.argtypes = [vp, i64, i64, i64, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, i64,
                                     vp, vp, vp, vp]
        L.csd_amp2response_accumulate.argtypes = [vp, i64, i64, i64, vp, i64, i64, vp, vp, ctypes.c_int, vp,
                                                  ctypes.c_int, vp, vp, vp]
        L.csd_sh2peaks.argtypes = [vp, i64, i64, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                   vp, ctypes.c_int, vp, vp, vp]
        L.csd_state_fod.argtypes = [vp, vp, i64, vp, vp, vp, vp]
        L.csd_state_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.csd_state_reuse_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.csd_state_assembly_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.csd_state_check.argtypes = [vp, ctypes.c_double, ctypes.POINTER(i64), ctypes.POINTER(i64), vp]
        L.csd_state_run_async.argtypes = [vp, vp, i64, i64, i64, vp, vp, ctypes.c_int, vp]
        L.csd_state_async_result.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(ctypes.c_int), vp]
        L.csd_dwi2fod_host_phased.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp]
        L.csd_fmls_create.argtypes = [vp, ctypes.POINTER(vp)]
        L.csd_fmls_create_default.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                              ctypes.POINTER(vp)]
        L.csd_fmls_destroy.argtypes = [vp]
        L.csd_fmls_destroy.restype = None
        L.csd_fmls_segment.argtypes = [vp, vp, i64, i64, i64, vp, ctypes.c_int, vp, vp, vp]
        L.csd_last_error.restype = ctypes.c_char_p
        _LIB = L
    return _LIB


def check(rc: int):
    if rc != CSD_OK:
        raise CSDError(f"csd error {rc}: {lib().csd_last_error().decode()}")


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ptr(t):
    """Device (or host) address of a torch tensor / numpy array, or None."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def _stream_ptr(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else stream


class Shared:
    """CSD::Shared.  ``grad`` is the [n_volumes][4] gradient table."""

    def __init__(self, grad):
        self.grad = np.ascontiguousarray(grad, np.float64)
        if self.grad.ndim != 2 or self.grad.shape[1] != 4:
            raise CSDError("gradient table must be [n_volumes][4]")
        self.lmax_cmdline = 0
        self.init_filter = None
        self.HR_dirs = None
        self.neg_lambda = 1.0
        self.norm_lambda = 1.0
        self.threshold = 0.0
        self.niter = 50
        self.response = None
        self.bzero_threshold = 10.0
        self.bvalue_epsilon = 80.0
        self.fp64_condition = 1e6
        self.refine = 3
        self.shells = None
        self._h = None

    def parse_cmdline_options(self, lmax=None, filter=None, directions=None, neg_lambda=None,
                              norm_lambda=None, threshold=None, niter=None, shells=None):
        """The options csd.h:71-99 reads; ``directions`` is [n][2] az/el;
        ``shells`` the -shells b-values (one non-b=0 shell, csd.h:64)."""
        if shells is not None:
            self.shells = np.ascontiguousarray(np.ravel(shells), np.float64)
        if lmax is not None:
            if np.ndim(lmax) and len(lmax) != 1:
                raise CSDError("CSD algorithm expects a single lmax to be specified")
            self.lmax_cmdline = int(np.ravel(lmax)[0])
        if filter is not None:
            self.init_filter = np.ascontiguousarray(filter, np.float64)
        if directions is not None:
            self.HR_dirs = np.ascontiguousarray(directions, np.float64)
        if neg_lambda is not None:
            self.neg_lambda = float(neg_lambda)
        if norm_lambda is not None:
            self.norm_lambda = float(norm_lambda)
        if threshold is not None:
            self.threshold = float(threshold)
        if niter is not None:
            self.niter = int(niter)

    def set_response(self, response):
        """csd.h:102-114: a path to a text file or the coefficients themselves."""
        if isinstance(response, (str, os.PathLike)):
            response = np.loadtxt(response, dtype=np.float64, ndmin=1)
        self.response = np.ascontiguousarray(np.ravel(response), np.float64)

    def init(self):
        """csd.h:117-198 on the host in FP64, then upload to the current device."""
        if self.response is None:
            raise CSDError("no response function set")
        p = csd_params()
        lib().csd_params_init(ctypes.byref(p))
        p.lmax = self.lmax_cmdline
        p.niter = self.niter
        p.neg_lambda = self.neg_lambda
        p.norm_lambda = self.norm_lambda
        p.threshold = self.threshold
        if self.init_filter is not None:
            p.filter = _dp(self.init_filter)
            p.n_filter = self.init_filter.size
        p.bzero_threshold = self.bzero_threshold
        p.bvalue_epsilon = self.bvalue_epsilon
        p.fp64_condition = self.fp64_condition
        p.refine = self.refine
        if self.shells is not None and self.shells.size:
            p.shells = _dp(self.shells)
            p.n_shells = self.shells.size
        h = ctypes.c_void_p()
        hr = self.HR_dirs
        check(lib().csd_shared_create(ctypes.byref(p), _dp(self.grad), self.grad.shape[0], _dp(self.response),
                                      self.response.size, None if hr is None else _dp(hr),
                                      0 if hr is None else hr.shape[0], ctypes.byref(h)))
        self.close()
        self._h = h
        info = (ctypes.c_int * 8)()
        check(lib().csd_shared_info(h, info))
        (self.lmax, self.lmax_response, self.lmax_data, self._nsh, self.n_init, self.n_dw, self.n_hr,
         self.niter) = list(info)
        self.nwords = (self.n_hr + 31) // 32
        return self

    @property
    def handle(self):
        if self._h is None:
            raise CSDError("Shared.init() has not been called")
        return self._h

    def nSH(self) -> int:
        return self._nsh

    @property
    def dwis(self) -> np.ndarray:
        out = np.zeros(self.n_dw, np.int32)
        check(lib().csd_shared_dwis(self.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return out

    def _matrix(self, which, shape):
        out = np.zeros(shape)
        check(lib().csd_shared_matrix(self.handle, which, _dp(out)))
        return out

    @property
    def rconv(self):
        return self._matrix(0, (self.n_init, self.n_dw))

    @property
    def M(self):
        return self._matrix(1, (self.n_dw, self._nsh))

    @property
    def Mt_M(self):
        return self._matrix(2, (self._nsh, self._nsh))

    @property
    def HR_trans(self):
        return self._matrix(3, (self.n_hr, self._nsh))

    def close(self):
        if self._h is not None and _LIB is not None:
            _LIB.csd_shared_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_shared(grad, response, lmax=None, **opts) -> Shared:
    s = Shared(grad)
    s.parse_cmdline_options(lmax=lmax, **opts)
    s.set_response(response)
    return s.init()


def solve_volumes(shareds, dwis, masks=None, warm=None, want_negmask=False, stream=None):
    """Deconvolve several device volumes in one persistent launch.

    dwis: list of torch float32 CUDA tensors [n_voxels][n_volumes] (voxel
    interleaved).  Returns a list of dicts with fod / status / iterations (and
    negmask) device tensors.
    """
    import torch
    n = len(dwis)
    arr = (ctypes.c_void_p * n)()
    vols = (csd_volume * n)()
    outs = []
    for i in range(n):
        s, d = shareds[i], dwis[i]
        if not d.is_cuda or d.dtype != torch.float32 or d.dim() != 2:
            raise CSDError("dwi must be a float32 CUDA tensor [n_voxels][n_volumes]")
        nv = d.shape[0]
        o = {"fod": torch.empty((nv, s.nSH()), dtype=torch.float32, device=d.device),
             "status": torch.empty(nv, dtype=torch.uint8, device=d.device),
             "iterations": torch.empty(nv, dtype=torch.uint8, device=d.device)}
        if want_negmask:
            o["negmask"] = torch.empty((nv, s.nwords), dtype=torch.int32, device=d.device)
        arr[i] = s.handle
        v = vols[i]
        v.dwi = d.data_ptr()
        v.n_voxels = nv
        v.voxel_stride = d.stride(0)
        v.volume_stride = d.stride(1)
        m = None if masks is None else masks[i]
        v.mask = _ptr(m)
        w = None if warm is None else warm[i]
        v.warm_negmask = _ptr(w)
        v.fod = o["fod"].data_ptr()
        v.fod_stride = s.nSH()
        v.status = o["status"].data_ptr()
        v.iterations = o["iterations"].data_ptr()
        v.negmask = o["negmask"].data_ptr() if want_negmask else None
        outs.append(o)
    check(lib().csd_solve(arr, vols, n, ctypes.c_void_p(_stream_ptr(stream))))
    return outs


def dwi2fod_csd(shared: Shared, dwi, mask=None, warm=None, want_negmask=False, stream=None):
    """`dwi2fod csd` over one device volume: returns fod [n_voxels][nSH] and per-voxel info."""
    return solve_volumes([shared], [dwi], None if mask is None else [mask],
                         None if warm is None else [warm], want_negmask, stream)[0]


def dwi2fod_csd_host(shared: Shared, dwi: np.ndarray, mask: np.ndarray | None = None):
    """End-to-end call on host arrays (numpy or pinned torch CPU tensors)."""
    nvox = dwi.shape[0]
    fod = np.zeros((nvox, shared.nSH()), np.float32) if not hasattr(dwi, "data_ptr") else None
    if fod is None:
        import torch
        fod = torch.empty((nvox, shared.nSH()), dtype=torch.float32, pin_memory=dwi.is_pinned())
    status = np.zeros(nvox, np.uint8)
    iters = np.zeros(nvox, np.uint8)
    check(lib().csd_dwi2fod_host(shared.handle, ctypes.c_void_p(_ptr(dwi)), nvox,
                                 ctypes.c_void_p(_ptr(mask)) if mask is not None else None,
                                 ctypes.c_void_p(_ptr(fod)), ctypes.c_void_p(status.ctypes.data),
                                 ctypes.c_void_p(iters.ctypes.data)))
    return {"fod": fod, "status": status, "iterations": iters}


def dwi2fod_csd_host_phased(shared: Shared, dwi, mask=None, net=None, fod=None):
    """The phased method (optionally warm-started by a WarmStartNet) on host
    arrays or pinned torch CPU tensors; copies are inside the call."""
    nvox = dwi.shape[0]
    if fod is None:
        fod = np.zeros((nvox, shared.nSH()), np.float32)
    status = np.zeros(nvox, np.uint8)
    iters = np.zeros(nvox, np.uint8)
    check(lib().csd_dwi2fod_host_phased(shared.handle, None if net is None else net._h, ctypes.c_void_p(_ptr(dwi)),
                                        nvox, ctypes.c_void_p(_ptr(mask)) if mask is not None else None,
                                        ctypes.c_void_p(_ptr(fod)), ctypes.c_void_p(status.ctypes.data),
                                        ctypes.c_void_p(iters.ctypes.data)))
    return {"fod": fod, "status": status, "iterations": iters}


def default_peak_seeds() -> np.ndarray:
    """sh2peaks' built-in 60 seed directions [azimuth elevation] (data/sh2peaks_seeds_60.txt)."""
    return np.loadtxt(os.path.join(HERE, "data", "sh2peaks_seeds_60.txt"), dtype=np.float32, ndmin=2)


def sh2peaks(sh, lmax: int | None = None, mask=None, seeds=None, npeaks: int = 3, threshold: float = -np.inf,
             directions=None, peaks=None, stream=None):
    """Peaks of each row of ``sh`` (float32 CUDA tensor [n][nSH]): a CUDA
    tensor [n][3 npeaks] of amplitude-scaled directions, NaN-padded
    (csd_sh2peaks; cmd/sh2peaks.cpp).  ``directions``: unit vectors
    [npeaks][3] to match (-direction); ``peaks``: per-voxel [n][3 npeaks]
    targets (-peaks)."""
    import torch
    n, nsh = sh.shape
    if lmax is None:
        lmax = int(round((math.sqrt(8 * nsh + 1) - 3) / 2))
    if seeds is None:
        seeds = default_peak_seeds()
    seeds = np.ascontiguousarray(seeds, np.float32)
    dirs = None if directions is None else np.ascontiguousarray(directions, np.float32)
    if dirs is not None:
        npeaks = len(dirs)
    if peaks is not None:
        npeaks = peaks.shape[1] // 3
    out = torch.empty((n, 3 * npeaks), dtype=torch.float32, device=sh.device)
    check(lib().csd_sh2peaks(ctypes.c_void_p(sh.data_ptr()), n, sh.stride(0), lmax,
                             ctypes.c_void_p(_ptr(mask)) if mask is not None else None,
                             ctypes.c_void_p(seeds.ctypes.data), len(seeds), npeaks, float(threshold),
                             ctypes.c_void_p(dirs.ctypes.data) if dirs is not None else None,
                             0 if dirs is None else len(dirs),
                             ctypes.c_void_p(peaks.data_ptr()) if peaks is not None else None,
                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(_stream_ptr(stream))))
    return out


class Amp2SHCommon:
    """The fit of amp2sh held on the device (Amp2SHCommon, cmd/amp2sh.cpp:86-104):
    ``fit`` = pinv(SH2amp) [nSH][len(dwis)] (numpy, FP64), ``dwis`` the
    volumes it applies to, ``bzeros`` the b=0 volumes for ``normalise``.
    Calling it on amplitudes runs csd_amp2sh."""

    def __init__(self, fit, dwis, bzeros=None, normalise: bool = False, device=None, sh2amp=None):
        import torch
        fit = np.asarray(fit, np.float64)
        self.dwis = np.asarray(dwis, np.int64).reshape(-1)
        self.bzeros = np.asarray([] if bzeros is None else bzeros, np.int64).reshape(-1)
        if fit.ndim != 2 or fit.shape[1] != len(self.dwis):
            raise ValueError("amp2sh: the fit matrix needs one column per selected volume")
        if (self.dwis < 0).any() or (self.bzeros < 0).any():
            raise ValueError("amp2sh: volume index out of range")
        self.normalise = bool(normalise)
        self.nsh, self.nd = fit.shape
        # the highest volume index: the kernel reads the amplitude rows at
        # these indices unchecked, so every call checks the rows are long enough
        self.max_volume = int(max(self.dwis.max(initial=-1), self.bzeros.max(initial=-1)))
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.fit_d = torch.from_numpy(np.ascontiguousarray(fit)).to(dev)
        self.dwis_d = torch.from_numpy(np.ascontiguousarray(self.dwis, np.int32)).to(dev)
        self.b0_d = torch.from_numpy(np.ascontiguousarray(self.bzeros, np.int32)).to(dev) if len(self.bzeros) else None
        # the mapping itself, for the Rician correction ([len(dwis)][nSH])
        self.sh2amp_d = None
        if sh2amp is not None:
            sh2amp = np.asarray(sh2amp, np.float64)
            if sh2amp.shape != (self.nd, self.nsh):
                raise ValueError("amp2sh: sh2amp must be [selected volumes][nSH]")
            self.sh2amp_d = torch.from_numpy(np.ascontiguousarray(sh2amp)).to(dev)

    def __call__(self, amp, out=None, stream=None, noise=None):
        """SH coefficients of each row of ``amp`` (float32 CUDA tensor
        [n][volumes], any strides) into ``out`` (float32 [n][>= nSH], unit
        column stride; allocated when None).  ``noise`` (float32 CUDA [n]):
        the Rician-corrected fit (needs ``sh2amp`` at construction).
        Returns ``out``."""
        import torch
        if amp.dim() != 2 or amp.dtype != torch.float32 or amp.device != self.fit_d.device:
            raise ValueError("amp2sh: amplitudes must be a float32 tensor [n][volumes] on the fit's device")
        if self.max_volume >= amp.shape[1]:
            raise ValueError("amp2sh: volume index out of range")
        if out is None:
            out = torch.empty((amp.shape[0], self.nsh), dtype=torch.float32, device=amp.device)
        if (out.dim() != 2 or out.dtype != torch.float32 or out.device != amp.device or out.shape[0] != amp.shape[0]
                or out.shape[1] < self.nsh or out.stride(1) != 1):
            raise ValueError("amp2sh: output must be float32 [n][>= nSH] with contiguous rows")
        if noise is not None:
            if self.sh2amp_d is None:
                raise ValueError("amp2sh: the Rician correction needs the sh2amp mapping")
            if noise.dtype != torch.float32 or noise.dim() != 1 or noise.shape[0] != amp.shape[0] or \
                    noise.device != amp.device:
                raise ValueError("amp2sh: noise must be a float32 tensor [n] on the amplitudes' device")
            check(lib().csd_amp2sh_rician(
                ctypes.c_void_p(amp.data_ptr()), amp.shape[0], amp.stride(0), amp.stride(1),
                ctypes.c_void_p(self.fit_d.data_ptr()), ctypes.c_void_p(self.sh2amp_d.data_ptr()), self.nsh,
                ctypes.c_void_p(self.dwis_d.data_ptr()), self.nd,
                ctypes.c_void_p(self.b0_d.data_ptr()) if self.b0_d is not None else None, len(self.bzeros),
                int(self.normalise), ctypes.c_void_p(noise.data_ptr()), noise.stride(0),
                ctypes.c_void_p(out.data_ptr()), max(out.stride(0), self.nsh), ctypes.c_void_p(_stream_ptr(stream))))
            return out
        check(lib().csd_amp2sh(ctypes.c_void_p(amp.data_ptr()), amp.shape[0], amp.stride(0), amp.stride(1),
                               ctypes.c_void_p(self.fit_d.data_ptr()), self.nsh,
                               ctypes.c_void_p(self.dwis_d.data_ptr()), self.nd,
                               ctypes.c_void_p(self.b0_d.data_ptr()) if self.b0_d is not None else None,
                               len(self.bzeros), int(self.normalise), ctypes.c_void_p(out.data_ptr()),
                               max(out.stride(0), self.nsh), ctypes.c_void_p(_stream_ptr(stream))))
        return out


def amp2sh(amp, fit, dwis, bzeros=None, normalise: bool = False, stream=None):
    """SH coefficients of each row of ``amp`` (float32 CUDA tensor [n][nvol]):
    one-off Amp2SHCommon(fit, dwis, bzeros, normalise)(amp).  Returns a
    float32 CUDA tensor [n][nSH]."""
    import torch
    if not isinstance(amp, torch.Tensor) or not amp.is_cuda:
        raise ValueError("amp2sh: amplitudes must be a float32 CUDA tensor [n][volumes]")
    return Amp2SHCommon(fit, dwis, bzeros, normalise, device=amp.device)(amp, stream=stream)


def negmask_to_bool(negmask, n_hr: int) -> np.ndarray:
    """[n][nwords] uint32/int32 words -> [n][n_hr] bool."""
    a = np.ascontiguousarray(np.asarray(negmask).astype(np.uint32))
    bits = np.unpackbits(a.view(np.uint8).reshape(a.shape[0], -1), axis=1, bitorder="little")
    return bits[:, :n_hr].astype(bool)


class State:
    """Batch of CSD objects driven one ``iterate()`` at a time (csd_state_*)."""

    def __init__(self, shared: Shared, capacity: int):
        self.shared = shared
        self.capacity = int(capacity)
        h = ctypes.c_void_p()
        check(lib().csd_state_create(shared.handle, self.capacity, ctypes.byref(h)))
        self._h = h
        self.n = 0

    def set(self, dwi, mask=None, stream=None):
        """CSD::set for each row of ``dwi`` (device float32 [n][n_volumes])."""
        self.n = dwi.shape[0]
        check(lib().csd_state_set(self._h, ctypes.c_void_p(dwi.data_ptr()), self.n, dwi.stride(0), dwi.stride(1),
                                  ctypes.c_void_p(_ptr(mask)) if mask is not None else None,
                                  ctypes.c_void_p(_stream_ptr(stream))))

    def warm(self, negmask, stream=None):
        check(lib().csd_state_warm(self._h, ctypes.c_void_p(negmask.data_ptr()), ctypes.c_void_p(_stream_ptr(stream))))

    def iterate(self, stream=None) -> int:
        """One CSD::iterate() on every active voxel; returns how many remain active."""
        n = ctypes.c_int64()
        check(lib().csd_state_iterate(self._h, ctypes.byref(n), ctypes.c_void_p(_stream_ptr(stream))))
        return n.value

    def stats(self) -> dict:
        """Work and device time since the last set() (csd_state_stats)."""
        out = (ctypes.c_double * 8)()
        check(lib().csd_state_stats(self._h, out))
        keys = ("passes", "projected", "solved", "sum_neg", "ms_set", "ms_project", "ms_solve", "launches")
        d = dict(zip(keys, list(out)))
        r = (ctypes.c_double * 3)()
        check(lib().csd_state_reuse_stats(self._h, r))
        d.update(reuse_solved=r[0], reuse_sum_changes=r[1], ms_reuse=r[2])
        a = (ctypes.c_double * 3)()
        check(lib().csd_state_assembly_stats(self._h, a))
        d.update(asm_launches=a[0], ms_asm=a[1], asm_chunk=a[2])
        return d

    def iterate_all(self, max_passes: int = 0, stream=None) -> int:
        """iterate() until no voxel is active (csd_state_run: passes batched on
        the device, same results); returns how many remain active."""
        n = ctypes.c_int64()
        check(lib().csd_state_run(self._h, int(max_passes), ctypes.byref(n), ctypes.c_void_p(_stream_ptr(stream))))
        return n.value

    def run(self, dwi, mask=None, warm=None, stream=None):
        """The phased method over one volume: set (+ warm sets), then iterate
        until no voxel is active.  Returns the number of passes."""
        self.set(dwi, mask=mask, stream=stream)
        if warm is not None:
            self.warm(warm, stream=stream)
        self.iterate_all(stream=stream)
        return int(self.stats()["passes"])

    def run_async(self, dwi, mask=None, warm=None, passes=None, stream=None):
        """set (+ warm sets) and `passes` passes (default niter + 1, enough for
        every voxel) with no host synchronisation: capturable in a CUDA graph
        (csd_state_run_async).  With warm sets, call warm() once beforehand."""
        self.n = dwi.shape[0]
        if passes is None:
            passes = self.shared.niter + 1
        check(lib().csd_state_run_async(self._h, ctypes.c_void_p(dwi.data_ptr()), self.n, dwi.stride(0),
                                        dwi.stride(1), ctypes.c_void_p(_ptr(mask)) if mask is not None else None,
                                        ctypes.c_void_p(warm.data_ptr()) if warm is not None else None,
                                        int(passes), ctypes.c_void_p(_stream_ptr(stream))))

    def async_result(self, stream=None):
        """(voxels still active, timed out) after run_async (synchronises)."""
        n, e = ctypes.c_int64(), ctypes.c_int()
        check(lib().csd_state_async_result(self._h, ctypes.byref(n), ctypes.byref(e),
                                           ctypes.c_void_p(_stream_ptr(stream))))
        return n.value, bool(e.value)

    def check(self, tol: float = 1e-6, stream=None, counts: bool = True):
        """FP64 residual check of every finished voxel's last solve; voxels with
        max|r| > tol max|b| are re-solved in FP64 (csd_state_check).  Returns
        (checked, re-solved) when ``counts`` (synchronises), else None."""
        if not counts:
            check(lib().csd_state_check(self._h, float(tol), None, None, ctypes.c_void_p(_stream_ptr(stream))))
            return None
        a, b = ctypes.c_int64(), ctypes.c_int64()
        check(lib().csd_state_check(self._h, float(tol), ctypes.byref(a), ctypes.byref(b),
                                    ctypes.c_void_p(_stream_ptr(stream))))
        return a.value, b.value

    def fod(self, stream=None, as_numpy=True):
        import torch
        s = self.shared
        dev = torch.device("cuda", torch.cuda.current_device())
        o = {"fod": torch.empty((self.n, s.nSH()), dtype=torch.float32, device=dev),
             "status": torch.empty(self.n, dtype=torch.uint8, device=dev),
             "iterations": torch.empty(self.n, dtype=torch.uint8, device=dev),
             "negmask": torch.empty((self.n, s.nwords), dtype=torch.int32, device=dev)}
        check(lib().csd_state_fod(self._h, ctypes.c_void_p(o["fod"].data_ptr()), s.nSH(),
                                  ctypes.c_void_p(o["status"].data_ptr()), ctypes.c_void_p(o["iterations"].data_ptr()),
                                  ctypes.c_void_p(o["negmask"].data_ptr()), ctypes.c_void_p(_stream_ptr(stream))))
        if as_numpy:
            torch.cuda.synchronize()
            return {k: v.cpu().numpy() for k, v in o.items()}
        return o

    def close(self):
        if getattr(self, "_h", None) is not None and _LIB is not None:
            _LIB.csd_state_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CSD:
    """The reference's per-voxel object (csd.h:221-271): set(S) takes the
    signals of the selected shell only (``shared.dwis`` order); iterate()
    returns True once the negative set repeats; FOD() returns F.  Each call
    is a batch of one on the GPU -- correct, not fast."""

    def __init__(self, shared: Shared):
        self.shared = shared
        self._state = State(shared, 1)
        self._done = False

    def set(self, DW_signals):
        import torch
        s = self.shared
        rec = np.zeros(s.grad.shape[0], np.float32)
        rec[s.dwis] = np.asarray(DW_signals, np.float32)
        self._state.set(torch.from_numpy(rec[None]).cuda())
        self._done = False

    def iterate(self) -> bool:
        if self._done:
            return True
        self._state.iterate()
        st = int(self._state.fod()["status"][0])
        self._done = (st & 0x0F) == STATUS_CONVERGED
        return self._done

    def FOD(self) -> np.ndarray:
        return self._state.fod()["fod"][0].astype(np.float64)
