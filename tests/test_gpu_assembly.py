"""The phased method's rank-k assembly on tcgen05 (csd_assemble_tc_kernel).

W = Mt_M + H[neg]^T H[neg] (src/dwi/sdeconv/csd.h:255-262) is formed for a
tile of 128 listed voxels at once as a dense product of their 0/1 set masks
with the table of HR_trans products, FP16 hi + lo, FP32 accumulation in
tensor memory; a solve kernel without constraint tables then factorises.
Checked here against the FP64 oracle (p99 rel err <= 1e-4, >= 99.5% of
voxels on the oracle's final set), plain and warm-started, at every
supported lmax, against the mma.sync assembly it replaces (same tolerance),
and across chunkings of the solve list (bit-identical: each voxel's row of
the product does not depend on its tile)."""
import numpy as np
import pytest

from mrtrix3_b200 import autotune, csd, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = {
    # lmax: (dims, b=0 volumes, DW directions)
    2: ((16, 16, 4), 6, 60),
    4: ((24, 16, 6), 6, 60),
    6: ((24, 24, 8), 6, 60),
    8: ((40, 32, 10), 6, 60),
    10: ((32, 24, 8), 8, 90),
    12: ((24, 20, 6), 8, 90),
}


def _run(s, d, m, warm, asm):
    autotune.set_knob(autotune.KNOB_ASSEMBLY, asm)
    try:
        st = csd.State(s, d.shape[0])
        st.run(d, mask=m, warm=warm)
        out = st.fod()
        stats = st.stats()
        st.close()
    finally:
        autotune.set_knob(autotune.KNOB_ASSEMBLY, 0)
    return out, stats


def _rel(a, b):
    den = np.maximum(np.abs(b).max(axis=1), 1e-30)
    return np.abs(a.astype(np.float64) - b).max(axis=1) / den


@pytest.mark.parametrize("lmax", sorted(CASES))
def test_tcgen05_assembly_matches_oracle_and_mma_assembly(cuda, hr_dirs, lmax):
    import torch
    dims, nb0, ndw = CASES[lmax]
    v = synth.make_volume(dims, nb0, ndw, (15.0, 40.0), lmax, 0.5, 700 + lmax)
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=lmax)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    inside = np.nonzero(v.mask)[0]
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, lmax=lmax).solve(v.dwi[inside])
    plain_tc, st_tc = _run(s, d, m, None, 2)
    plain_mma, _ = _run(s, d, m, None, 1)
    # a warm start: the oracle's sets with a few directions flipped
    warm = torch.zeros((v.n_voxels, s.nwords), dtype=torch.int32)
    warm[inside] = torch.from_numpy(ref["negmask"].view(np.int32).copy())
    warm[:, 0] ^= 0x5
    warm = warm.cuda()
    warm_tc, _ = _run(s, d, m, warm, 2)
    for name, out in (("plain", plain_tc), ("warm", warm_tc)):
        rel = _rel(out["fod"][inside], ref["F"])
        assert np.percentile(rel, 99) <= 1e-4, (name, np.percentile(rel, 99))
        match = np.mean(np.all(out["negmask"][inside].view(np.uint32) == ref["negmask"], axis=1))
        assert match >= 0.995, (name, match)
        if name == "plain":
            assert np.mean((out["status"][inside] & 0x0F) == (ref["status"] & 0x0F)) >= 0.999
    outside = np.nonzero(v.mask == 0)[0]
    assert np.all(plain_tc["fod"][outside] == 0)
    # against the mma.sync assembly: the same iteration, FP32 sums in another order
    rel = _rel(plain_tc["fod"][inside], plain_mma["fod"][inside].astype(np.float64))
    assert np.percentile(rel, 99) <= 1e-4
    assert st_tc["solved"] > 0


def test_tcgen05_assembly_chunking_is_bit_identical(cuda, monkeypatch):
    """Lists longer than the assembled-system buffer run chunk by chunk; a
    256-entry chunk (many chunks, a ragged last one) gives the outputs of
    one chunk bit for bit, plain and warm-started."""
    import torch
    v = synth.make_volume((40, 36, 10), 6, 60, (15.0, 40.0), 8, 0.5, 77)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    plain = csd.dwi2fod_csd(s, d, mask=m, want_negmask=True)
    warm = plain["negmask"].clone()
    warm[:, 2] ^= 0x11
    outs = {}
    for chunk in (None, "256"):
        if chunk:
            monkeypatch.setenv("CSD_ASM_CHUNK", chunk)
        else:
            monkeypatch.delenv("CSD_ASM_CHUNK", raising=False)
        for name, w in (("plain", None), ("warm", warm)):
            outs[(chunk, name)] = _run(s, d, m, w, 2)[0]
    for name in ("plain", "warm"):
        a, b = outs[(None, name)], outs[("256", name)]
        for k in ("fod", "negmask", "status", "iterations"):
            assert np.array_equal(a[k], b[k]), (name, k)
