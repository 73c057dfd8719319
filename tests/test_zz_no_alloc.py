"""csd_solve_noalloc: the solve for callers that must not call cudaMalloc.

Some applications own every byte of device memory through their own
allocator, or must keep their footprint fixed once running; they cannot let
a library allocate mid-run.  csd_solve_noalloc keeps all of its device
scratch in one static array of the library instead.  This test calls it
through the C ABI twice in a row (the array keeps the previous call's
contents, so the second call checks that everything that must start from
zero is cleared) and compares each result with csd_solve's, within the
tolerance the other GPU tests use.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from mrtrix3_b200 import csd, synth

pytestmark = pytest.mark.gpu


def _noalloc(shared, dwi, mask, fod, status, iters, negmask):
    L = csd.lib()
    fn = L.csd_solve_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(csd.csd_volume), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    v = csd.csd_volume()
    v.dwi = dwi.data_ptr()
    v.n_voxels = dwi.shape[0]
    v.voxel_stride = dwi.stride(0)
    v.volume_stride = dwi.stride(1)
    v.mask = mask.data_ptr()
    v.warm_negmask = None
    v.fod = fod.data_ptr()
    v.fod_stride = fod.stride(0)
    v.status = status.data_ptr()
    v.iterations = iters.data_ptr()
    v.negmask = negmask.data_ptr()
    import torch
    csd.check(fn(shared.handle, ctypes.byref(v), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))


def test_noalloc_matches_solve_twice(cuda):
    import torch
    v = synth.make_volume((48, 40, 8), 6, 60, (15.0, 40.0), 8, 0.5, 4242)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    dwi = torch.from_numpy(v.dwi).cuda()
    mask = torch.from_numpy(v.mask).cuda()
    ref = csd.dwi2fod_csd(s, dwi, mask=mask, want_negmask=True)
    torch.cuda.synchronize()
    ref = {k: t.cpu().numpy() for k, t in ref.items()}
    n = dwi.shape[0]
    for call in range(2):
        fod = torch.full((n, s.nSH()), float("nan"), dtype=torch.float32, device=cuda)
        status = torch.full((n,), 255, dtype=torch.uint8, device=cuda)
        iters = torch.full((n,), 255, dtype=torch.uint8, device=cuda)
        negmask = torch.full((n, s.nwords), -1, dtype=torch.int32, device=cuda)
        _noalloc(s, dwi, mask, fod, status, iters, negmask)
        torch.cuda.synchronize()
        got = fod.cpu().numpy().astype(np.float64)
        den = np.maximum(np.abs(ref["fod"]).max(axis=1), 1e-30)
        rel = np.abs(got - ref["fod"]).max(axis=1) / den
        rel[np.abs(ref["fod"]).max(axis=1) == 0] = np.abs(got).max(axis=1)[np.abs(ref["fod"]).max(axis=1) == 0]
        assert np.isfinite(got).all(), call
        assert np.percentile(rel, 99) <= 1e-4 and rel.max() <= 1e-3, (call, rel.max())
        assert np.array_equal(status.cpu().numpy(), ref["status"]), call
        assert np.array_equal(iters.cpu().numpy(), ref["iterations"]), call
        assert np.mean(np.all(negmask.cpu().numpy() == ref["negmask"], axis=1)) >= 0.995, call
