"""Learned warm start for CSD: host driver of the csd_mlp_* C ABI.

The network (66 -> 256 -> 256 -> 300, GELU, sigmoid head, BF16 weights,
FP32 accumulation) maps a voxel's normalised signal to the probability that
each of the 300 constraint directions is in the voxel's converged negative
set.  It is trained on the GPU by the library's own forward / backward /
Adam kernels on (signal, negative set) pairs that the plain GPU CSD
produces, and at run time its thresholded prediction replaces only the
first negative set of each voxel (``csd_volume.warm_negmask``): the CSD
iteration still runs to its own stopping rule, and voxels that do not reach
a fixed point are re-solved from the plain start.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import csd
from .csd import check, lib


def _setup(L):
    if getattr(L, "_mlp_ready", False):
        return L
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    L.csd_mlp_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.csd_mlp_destroy.argtypes = [vp]
    L.csd_mlp_destroy.restype = None
    L.csd_mlp_param_count.argtypes = [vp]
    L.csd_mlp_param_count.restype = i64
    L.csd_mlp_get_params.argtypes = [vp, vp, i64]
    L.csd_mlp_set_params.argtypes = [vp, vp, i64]
    L.csd_mlp_set_inputs.argtypes = [vp, vp, ctypes.c_int, vp, vp]
    L.csd_mlp_inputs.argtypes = [vp, vp, i64, i64, i64, vp, vp]
    L.csd_mlp_train_epoch.argtypes = [vp, vp, vp, i64, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_uint64,
                                      ctypes.POINTER(ctypes.c_float), vp]
    L.csd_mlp_predict.argtypes = [vp, vp, i64, i64, i64, vp, ctypes.c_float, vp, vp]
    L.csd_mlp_gradients.argtypes = [vp, vp, vp, i64, vp, vp]
    L.csd_mlp_logits.argtypes = [vp, vp, i64, vp]
    L._mlp_ready = True
    return L


class WarmStartNet:
    """The warm-start MLP on the current CUDA device."""

    def __init__(self, n_in: int = 66, n_hidden: int = 256, n_out: int = 300, seed: int = 0):
        self.L = _setup(lib())
        h = ctypes.c_void_p()
        check(self.L.csd_mlp_create(n_in, n_hidden, n_out, seed, ctypes.byref(h)))
        self._h = h
        self.n_in, self.n_hidden, self.n_out = n_in, n_hidden, n_out
        self.ld_in = (n_in + 15) // 16 * 16
        self.ld_out = (n_out + 7) // 8 * 8
        self.nw = (n_out + 31) // 32
        self.b0_index = None
        self.mean = None
        self.stdev = None
        self.logit_threshold = 0.0

    # ---- parameters ------------------------------------------------------
    @property
    def n_params(self) -> int:
        return int(self.L.csd_mlp_param_count(self._h))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        check(self.L.csd_mlp_get_params(self._h, out.ctypes.data, out.size))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        check(self.L.csd_mlp_set_params(self._h, p.ctypes.data, p.size))

    def layout(self):
        """Offsets of W1 b1 W2 b2 W3 b3 in the flat parameter vector."""
        H, o = self.n_hidden, 0
        out = {}
        for name, size in (("W1", H * self.ld_in), ("b1", H), ("W2", H * H), ("b2", H),
                           ("W3", self.ld_out * H), ("b3", self.ld_out)):
            out[name] = (o, size)
            o += size
        return out

    # ---- inputs ----------------------------------------------------------
    def set_inputs(self, b0_index, mean, stdev):
        self.b0_index = np.ascontiguousarray(b0_index, np.int32)
        self.mean = np.ascontiguousarray(mean, np.float32)
        self.stdev = np.ascontiguousarray(stdev, np.float32)
        check(self.L.csd_mlp_set_inputs(self._h, self.b0_index.ctypes.data, self.b0_index.size,
                                        self.mean.ctypes.data, self.stdev.ctypes.data))

    def fit_inputs(self, grad: np.ndarray, dwi_host: np.ndarray, bzero_threshold: float = 10.0):
        """Per-volume mean / stdev of S / mean(S_b0) over training signals."""
        b0 = np.nonzero(grad[:, 3] <= bzero_threshold)[0]
        s0 = dwi_host[:, b0].mean(axis=1, keepdims=True) if len(b0) else np.ones((len(dwi_host), 1), np.float32)
        x = dwi_host / np.maximum(s0, 1e-6)
        self.set_inputs(b0, x.mean(axis=0), x.std(axis=0) + 1e-6)

    def inputs(self, dwi):
        """Normalised BF16 inputs [n][ld_in] (as an int16 torch tensor) for device signals [n][n_in]."""
        import torch
        x = torch.empty((dwi.shape[0], self.ld_in), dtype=torch.int16, device=dwi.device)
        check(self.L.csd_mlp_inputs(self._h, dwi.data_ptr(), dwi.shape[0], dwi.stride(0), dwi.stride(1), x.data_ptr(),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return x

    # ---- training --------------------------------------------------------
    def train(self, x, negmask, epochs: int = 10, batch: int = 4096, lr: float = 2e-3, weight_decay: float = 0.0,
              seed: int = 0, verbose: bool = False):
        """Adam over shuffled mini-batches; returns the mean BCE of every epoch."""
        import torch
        n = (x.shape[0] // batch) * batch
        losses = []
        for e in range(epochs):
            # cosine decay to 5% of the initial rate
            lr_e = lr * (0.05 + 0.95 * 0.5 * (1 + np.cos(np.pi * e / max(1, epochs))))
            loss = ctypes.c_float()
            check(self.L.csd_mlp_train_epoch(self._h, x.data_ptr(), negmask.data_ptr(), n, batch, lr_e, weight_decay,
                                             seed * 1000 + e, ctypes.byref(loss),
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
            losses.append(loss.value)
            if verbose:
                print(f"epoch {e}: lr {lr_e:.2e} bce {loss.value:.5f}", flush=True)
        return losses

    # ---- inference -------------------------------------------------------
    def predict(self, dwi, mask=None, out=None, stream=None, threshold: float | None = None):
        """Predicted first negative sets [n][nw] (int32 device tensor)."""
        import torch
        n = dwi.shape[0]
        if out is None:
            out = torch.empty((n, self.nw), dtype=torch.int32, device=dwi.device)
        sp = torch.cuda.current_stream().cuda_stream if stream is None else getattr(stream, "cuda_stream", stream)
        thr = self.logit_threshold if threshold is None else threshold
        check(self.L.csd_mlp_predict(self._h, dwi.data_ptr(), n, dwi.stride(0), dwi.stride(1),
                                     None if mask is None else mask.data_ptr(), thr, out.data_ptr(),
                                     ctypes.c_void_p(sp)))
        return out

    def gradients(self, x, negmask):
        g = np.zeros(self.n_params, np.float32)
        loss = np.zeros(1, np.float32)
        check(self.L.csd_mlp_gradients(self._h, x.data_ptr(), negmask.data_ptr(), x.shape[0], g.ctypes.data,
                                       loss.ctypes.data))
        return g, float(loss[0])

    def logits(self, x):
        z = np.zeros((x.shape[0], self.ld_out), np.float32)
        check(self.L.csd_mlp_logits(self._h, x.data_ptr(), x.shape[0], z.ctypes.data))
        return z[:, :self.n_out]

    # ---- persistence -----------------------------------------------------
    def save(self, path: str):
        np.savez_compressed(path, params=self.get_params(), b0_index=self.b0_index, mean=self.mean, stdev=self.stdev,
                            dims=np.array([self.n_in, self.n_hidden, self.n_out]),
                            logit_threshold=np.float32(self.logit_threshold))

    @classmethod
    def load(cls, path: str) -> "WarmStartNet":
        d = np.load(path)
        n_in, n_hidden, n_out = (int(v) for v in d["dims"])
        net = cls(n_in, n_hidden, n_out)
        net.set_params(d["params"])
        net.set_inputs(d["b0_index"], d["mean"], d["stdev"])
        if "logit_threshold" in d:
            net.logit_threshold = float(d["logit_threshold"])
        return net

    def close(self):
        if getattr(self, "_h", None) is not None:
            self.L.csd_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def training_pairs(shared: csd.Shared, dwi, chunk: int = 1 << 20):
    """Label signals [n][n_vol] (device) with the plain GPU CSD's final
    negative sets; returns (negmask [n][nw] int32, converged bool [n])."""
    import torch
    negs, conv = [], []
    for a in range(0, dwi.shape[0], chunk):
        o = csd.dwi2fod_csd(shared, dwi[a:a + chunk], want_negmask=True)
        negs.append(o["negmask"])
        conv.append((o["status"] & 0x0F) == csd.STATUS_CONVERGED)
    return torch.cat(negs), torch.cat(conv)


def train_warm_start(grad, n_train: int = 2_000_000, epochs: int = 12, batch: int = 4096, lr: float = 2e-3,
                     seed: int = 11, verbose: bool = False, signals=None):
    """Generate n_train synthetic voxels on the scheme, label them with the
    plain GPU CSD, fit the input normalisation and train the network."""
    import torch

    from . import synth
    if signals is None:
        rng = np.random.default_rng(seed)
        signals = synth.voxel_signals(rng, grad, n_train, (15.0, 40.0))
    shared = csd.make_shared(grad, synth.RESPONSE)
    dev = torch.device("cuda", torch.cuda.current_device())
    d = torch.from_numpy(signals).to(dev)
    neg, conv = training_pairs(shared, d)
    keep = torch.nonzero(conv).flatten()
    perm = keep[torch.randperm(len(keep), generator=torch.Generator().manual_seed(seed)).to(dev)]
    net = WarmStartNet(grad.shape[0], 256, 300, seed=seed)
    net.fit_inputs(grad, signals[:200_000])
    x = net.inputs(d[perm])
    y = neg[perm].contiguous()
    losses = net.train(x, y, epochs=epochs, batch=batch, lr=lr, seed=seed, verbose=verbose)
    return net, losses
