"""Diffusion tensors on the GPU: ``dwi2tensor`` with the ``tensor2metric``
values that ``dwi2response`` needs (FA and the FA-modulated principal
eigenvector), through csd_dwi2tensor (cmd/dwi2tensor.cpp, cmd/tensor2metric.cpp,
src/dwi/tensor.h)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import csd

DEFAULT_NITER = 2


def bmatrix(grad) -> np.ndarray:
    """-grad2bmatrix (src/dwi/tensor.h:30-56): [volumes][7] rows
    [-b gx^2, -b gy^2, -b gz^2, -2b gx gy, -2b gx gz, -2b gy gz, 1]."""
    g = np.asarray(grad, np.float64)
    x, y, z, b = g[:, 0], g[:, 1], g[:, 2], g[:, 3]
    return -np.stack([b * x * x, b * y * y, b * z * z, 2 * b * x * y, 2 * b * x * z, 2 * b * y * z,
                      -np.ones_like(b)], axis=1)


def dwi2tensor(dwi, grad, mask=None, iter: int = DEFAULT_NITER, ols: bool = False, stream=None):
    """Per row of ``dwi`` (device float32 [n][volumes]): (dt [n][6], b0 [n],
    fa [n], vec [n][3]) device float32 tensors."""
    import torch
    from . import msmt
    g = msmt.normalise_scheme(grad)
    if len(msmt.cluster_shells(g[:, 3])) < 2:
        raise ValueError("Tensor estimation requires at least 2 b-values")
    n, nvol = dwi.shape
    if g.shape[0] != nvol:
        raise ValueError("dwi2tensor: the gradient table does not match the volumes")
    dev = dwi.device
    B = torch.from_numpy(np.ascontiguousarray(bmatrix(g))).to(dev)
    dt = torch.empty((n, 6), dtype=torch.float32, device=dev)
    b0 = torch.empty(n, dtype=torch.float32, device=dev)
    fa = torch.empty(n, dtype=torch.float32, device=dev)
    vec = torch.empty((n, 3), dtype=torch.float32, device=dev)
    m = None if mask is None else mask.to(torch.uint8)
    csd.check(csd.lib().csd_dwi2tensor(ctypes.c_void_p(dwi.data_ptr()), n, dwi.stride(0), dwi.stride(1),
                                       ctypes.c_void_p(B.data_ptr()), nvol,
                                       ctypes.c_void_p(m.data_ptr()) if m is not None else None, int(iter),
                                       int(bool(ols)), ctypes.c_void_p(dt.data_ptr()), 6,
                                       ctypes.c_void_p(b0.data_ptr()), ctypes.c_void_p(fa.data_ptr()),
                                       ctypes.c_void_p(vec.data_ptr()), ctypes.c_void_p(csd._stream_ptr(stream))))
    return dt, b0, fa, vec
