"""csd_solve_noalloc: the solve for callers that must not call cudaMalloc.

Some applications own every byte of device memory through their own
allocator, or must keep their footprint fixed once running; they cannot let
a library allocate mid-run.  csd_solve_noalloc keeps all of its device
scratch in one static array of the library instead.  This test calls it
through the C ABI twice in a row (the array keeps the previous call's
contents, so the second call checks that everything that must start from
zero is cleared) and compares each result with csd_solve's and with the FP64
oracle's, within the tolerance the other GPU tests use: at lmax 8, 10 and 12
(at 10 and 12 the array holds fewer blocks' FP64 slots than the GPU has SMs,
so the grid shrinks to fit), and with every factorisation forced through the
FP64 slots.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from mrtrix3_b200 import csd, synth
from oracle import oracle as O

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


CASES = {
    # name: (dims, b=0 volumes, DW directions, lmax, force FP64)
    "lmax8": ((48, 40, 8), 6, 60, 8, False),
    "lmax10": ((40, 24, 8), 8, 90, 10, False),
    "lmax12": ((32, 16, 8), 8, 90, 12, False),
    "lmax8_fp64": ((24, 16, 4), 6, 60, 8, True),
}


@pytest.mark.parametrize("case", list(CASES))
def test_noalloc_matches_solve_twice(cuda, hr_dirs, case):
    import torch
    dims, nb0, ndw, lmax, force64 = CASES[case]
    v = synth.make_volume(dims, nb0, ndw, (15.0, 40.0), lmax, 0.5, 4242 + lmax)
    s = csd.Shared(v.grad)
    s.parse_cmdline_options(lmax=lmax)
    if force64:
        s.fp64_condition = 1.0  # every factorisation goes to the FP64 slots of the static array
    s.set_response(synth.RESPONSE)
    s.init()
    dwi = torch.from_numpy(v.dwi).cuda()
    mask = torch.from_numpy(v.mask).cuda()
    ref = csd.dwi2fod_csd(s, dwi, mask=mask, want_negmask=True)
    torch.cuda.synchronize()
    ref = {k: t.cpu().numpy() for k, t in ref.items()}
    inside = np.nonzero(v.mask)[0]
    o64 = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, lmax=lmax).solve(v.dwi[inside])
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
        st = status.cpu().numpy()
        assert np.array_equal(st, ref["status"]), call
        if force64:
            assert np.all(st[inside] & csd.STATUS_FP64), call
        assert np.array_equal(iters.cpu().numpy(), ref["iterations"]), call
        neg = negmask.cpu().numpy()
        assert np.mean(np.all(neg == ref["negmask"], axis=1)) >= 0.995, call
        # against the FP64 oracle, as the parity tests
        r64 = np.abs(got[inside] - o64["F"]).max(axis=1) / np.abs(o64["F"]).max(axis=1)
        assert np.percentile(r64, 99) <= 1e-4, (call, np.percentile(r64, 99))
        assert np.mean(np.all(neg[inside].view(np.uint32) == o64["negmask"], axis=1)) >= 0.995, call
        assert np.mean((st[inside] & 0x0F) == (o64["status"] & 0x0F)) >= 0.999, call
