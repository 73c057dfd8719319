"""GPU parity of the CUDA CSD path (through the C ABI) against the FP64 oracle.

Tolerance: per voxel rel = max_i |F_gpu - F_64| /
max_i |F_64| (the reference's own `-voxel` criterion, core/image_diff.h:
92-109); p99 over voxels <= 1e-4, and >= 99.5% of voxels ending on exactly
the oracle's negative set.
"""
import numpy as np
import pytest

from mrtrix3_b200 import csd, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P99_TOL = 1e-4
MATCH_TOL = 0.995


def rel_err(fod, F64):
    den = np.abs(F64).max(axis=1)
    num = np.abs(fod.astype(np.float64) - F64).max(axis=1)
    ok = den > 0
    r = np.zeros(len(F64))
    r[ok] = num[ok] / den[ok]
    r[~ok] = num[~ok]
    return r


def run_gpu(shared, dwi, mask=None, warm=None):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(dwi)).cuda()
    m = None if mask is None else torch.from_numpy(np.ascontiguousarray(mask)).cuda()
    w = None if warm is None else torch.from_numpy(np.ascontiguousarray(warm).view(np.int32)).cuda()
    o = csd.dwi2fod_csd(shared, d, mask=m, warm=w, want_negmask=True)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in o.items()}


def check_parity(out, ref, n_hr=300, p99=P99_TOL, match=MATCH_TOL, iters_frac=0.99):
    r = rel_err(out["fod"], ref["F"])
    assert np.percentile(r, 99) <= p99, (np.percentile(r, 99), r.max())
    m = np.all(out["negmask"].view(np.uint32) == ref["negmask"], axis=1)
    assert m.mean() >= match, m.mean()
    assert (out["iterations"] == ref["iters"]).mean() >= iters_frac
    # outcome per voxel (converged / niter / masked / non-finite); a voxel
    # whose amplitudes sit on a sign change may cycle in one precision only
    assert np.mean((out["status"] & 0x0F) == (ref["status"] & 0x0F)) >= 0.999
    return r, m


def test_config1_full_volume(cuda, hr_dirs):
    """32x32x20, 6 b=0 + 64 DW, SNR 30, lmax 8 -- every voxel."""
    v = synth.config1()
    s = csd.make_shared(v.grad, synth.RESPONSE)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi)
    out = run_gpu(s, v.dwi)
    r, m = check_parity(out, ref)
    assert r.max() < 1e-3
    assert np.mean(out["status"] == 1) >= 0.999


def test_golden_fixtures(cuda):
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "csd_golden.npz"))
    kw = {"l6thr": {"threshold": 0.1}}
    for name in ("c1", "c2", "l10", "l6thr"):
        s = csd.make_shared(g[f"{name}_grad"], synth.RESPONSE, lmax=int(g[f"{name}_lmax"]), **kw.get(name, {}))
        out = run_gpu(s, g[f"{name}_dwi"])
        r = rel_err(out["fod"], g[f"{name}_F"])
        assert np.percentile(r, 99) <= P99_TOL, name
        assert np.mean(np.all(out["negmask"].view(np.uint32) == g[f"{name}_negmask"], axis=1)) >= 0.98, name


@pytest.mark.parametrize("lmax,ndw", [(2, 30), (4, 30), (6, 45), (10, 90), (12, 90)])
def test_other_lmax(cuda, hr_dirs, lmax, ndw):
    v = synth.make_volume((40, 10, 1), 6, ndw, (15.0, 40.0), lmax, None, 20 + lmax)
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=lmax)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, lmax=lmax).solve(v.dwi)
    check_parity(run_gpu(s, v.dwi), ref)


def test_mask_nonfinite_negative(cuda, hr_dirs):
    v = synth.make_volume((64, 1, 1), 6, 60, 30.0, 8, None, 31)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    d = v.dwi.copy()
    dw = s.dwis
    d[1, dw[3]] = np.nan
    d[2, dw[5]] = np.inf
    d[3, dw[7]] = -50.0
    d[4, 0] = np.nan                       # a b=0 volume: not read, so the voxel is solved
    mask = np.ones(64, np.uint8)
    mask[10:20] = 0
    out = run_gpu(s, d, mask=mask)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(d, mask=mask)
    assert np.array_equal(out["status"] & 0x0F, ref["status"] & 0x0F)
    assert np.all(out["fod"][[1, 2]] == 0) and np.all(out["fod"][10:20] == 0)
    assert out["status"][1] == 3 and out["status"][10] == 0 and out["status"][4] == 1
    check_parity(out, ref)


@pytest.mark.parametrize("niter", [0, 1, 2, 3])
def test_niter(cuda, hr_dirs, niter):
    v = synth.make_volume((128, 1, 1), 6, 60, 30.0, 8, None, 40 + niter)
    s = csd.make_shared(v.grad, synth.RESPONSE, niter=niter)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, niter=niter).solve(v.dwi)
    out = run_gpu(s, v.dwi)
    r = rel_err(out["fod"], ref["F"])
    assert np.percentile(r, 99) <= P99_TOL
    assert np.array_equal(out["iterations"], ref["iters"])
    if niter == 0:
        assert r.max() < 1e-6


def test_options(cuda, hr_dirs):
    v = synth.make_volume((128, 1, 1), 6, 60, 30.0, 8, None, 50)
    kw = dict(neg_lambda=0.7, norm_lambda=3.0, threshold=0.05)
    s = csd.make_shared(v.grad, synth.RESPONSE, filter=[1, 1, 1, 0.5], **kw)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, filter=np.array([1, 1, 1, 0.5]), **kw).solve(v.dwi)
    check_parity(run_gpu(s, v.dwi), ref)


def test_custom_direction_set(cuda, hr_dirs):
    v = synth.make_volume((128, 1, 1), 6, 60, 30.0, 8, None, 51)
    dirs = hr_dirs[:200].copy()
    s = csd.make_shared(v.grad, synth.RESPONSE, directions=dirs)
    ref = O.OracleShared(v.grad, synth.RESPONSE, dirs).solve(v.dwi)
    out = run_gpu(s, v.dwi)
    r = rel_err(out["fod"], ref["F"])
    assert np.percentile(r, 99) <= P99_TOL
    assert out["negmask"].shape[1] == 7


def test_fp64_path_forced(cuda, hr_dirs):
    """With the condition threshold at 1 every factorisation runs in FP64."""
    v = synth.make_volume((96, 1, 1), 6, 60, 30.0, 8, None, 52)
    s = csd.Shared(v.grad)
    s.fp64_condition = 1.0
    s.set_response(synth.RESPONSE)
    s.init()
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi)
    out = run_gpu(s, v.dwi)
    assert np.all(out["status"] & csd.STATUS_FP64)
    r, m = check_parity(out, ref, p99=1e-5)
    assert m.mean() >= 0.99


def test_multi_volume_one_launch(cuda, hr_dirs):
    """Uneven volumes with independent random direction sets in one persistent launch."""
    import torch
    vols = [synth.make_volume(dims, 6, 60, (15.0, 40.0), 8, 0.5, 60 + i, random_dirs=True)
            for i, dims in enumerate([(9, 7, 5), (16, 4, 3), (5, 5, 5), (20, 10, 2)])]
    shs = [csd.make_shared(v.grad, synth.RESPONSE) for v in vols]
    outs = csd.solve_volumes(shs, [torch.from_numpy(v.dwi).cuda() for v in vols],
                             masks=[torch.from_numpy(v.mask).cuda() for v in vols], want_negmask=True)
    torch.cuda.synchronize()
    for v, o in zip(vols, outs):
        ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi, mask=v.mask)
        check_parity({k: t.cpu().numpy() for k, t in o.items()}, ref)


def test_warm_start_exact_sets(cuda, hr_dirs):
    """Warm-started from the oracle's final sets, every voxel stops after one solve."""
    v = synth.make_volume((256, 1, 1), 6, 60, (15.0, 40.0), 8, None, 70)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi)
    out = run_gpu(s, v.dwi, warm=ref["negmask"])
    assert (out["iterations"] == 2).mean() >= 0.99
    check_parity(out, ref, iters_frac=0.0)


def test_warm_start_bad_sets_restart(cuda, hr_dirs):
    """Empty first sets still converge; with niter too small to converge the
    voxel is re-solved from the plain start (status flag WARM_RESTART)."""
    v = synth.make_volume((128, 1, 1), 6, 60, (15.0, 40.0), 8, None, 71)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi)
    out = run_gpu(s, v.dwi, warm=np.zeros((128, 10), np.uint32))
    r = rel_err(out["fod"], ref["F"])
    assert np.percentile(r, 99) <= P99_TOL
    s2 = csd.make_shared(v.grad, synth.RESPONSE, niter=1)
    full = np.full((128, 10), 0xFFFFFFFF, np.uint32)
    out2 = run_gpu(s2, v.dwi, warm=full)
    assert np.all(out2["status"] & csd.STATUS_WARM_RESTART)


def test_state_api_matches_oracle(cuda, hr_dirs):
    """csd_state_set / iterate / fod: one CSD::iterate() per call over a batch."""
    import torch
    v = synth.make_volume((300, 1, 1), 6, 60, (15.0, 40.0), 8, None, 80)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi)
    st = csd.State(s, 300)
    st.set(torch.from_numpy(v.dwi).cuda())
    calls = 0
    while True:
        calls += 1
        if st.iterate() == 0:
            break
        assert calls <= 50
    out = st.fod()
    assert calls == ref["iters"].max()
    check_parity(out, ref)


def test_state_run_equals_iterate_loop(cuda):
    """csd_state_run (passes batched on the device, counts read back once per
    batch) gives the same FODs, sets, statuses and iteration counts as
    calling csd_state_iterate until it reports 0, plain and warm-started,
    and max_passes stops it after that many passes."""
    import torch
    v = synth.make_volume((48, 40, 12), 6, 60, (15.0, 40.0), 8, 0.5, 82)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    plain = csd.dwi2fod_csd(s, d, mask=m, want_negmask=True)
    warm = plain["negmask"].clone()
    warm[:, 1] ^= 0x30
    st = csd.State(s, v.n_voxels)
    for w in (None, warm):
        st.set(d, mask=m)
        if w is not None:
            st.warm(w)
        loop = 0
        while st.iterate() > 0:
            loop += 1
        a = st.fod()
        stats_loop = st.stats()
        st.set(d, mask=m)
        if w is not None:
            st.warm(w)
        assert st.iterate_all(max_passes=2) > 0
        assert st.stats()["passes"] == 2
        assert st.iterate_all() == 0
        b = st.fod()
        for k in ("fod", "negmask", "status", "iterations"):
            assert np.array_equal(a[k], b[k]), k
        sb = st.stats()
        for k in ("passes", "projected", "solved", "sum_neg"):
            assert sb[k] == stats_loop[k], k
    st.close()


def test_per_voxel_surface(cuda, hr_dirs):
    """CSD(shared).set(S); while not iterate(); FOD() -- the reference's per-voxel object."""
    v = synth.make_volume((4, 1, 1), 6, 60, 30.0, 8, None, 81)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi)
    c = csd.CSD(s)
    for i in range(4):
        c.set(v.dwi[i][s.dwis])
        n = 0
        while n < s.niter:
            n += 1
            if c.iterate():
                break
        assert n == ref["iters"][i]
        F = c.FOD()
        assert np.abs(F - ref["F"][i]).max() <= P99_TOL * np.abs(ref["F"][i]).max()


def test_host_entry_point_matches_device(cuda):
    import torch
    v = synth.make_volume((200, 4, 1), 6, 60, (15.0, 40.0), 8, 0.6, 90)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    dev = run_gpu(s, v.dwi, mask=v.mask)
    pinned = torch.from_numpy(v.dwi).pin_memory()
    host = csd.dwi2fod_csd_host(s, pinned, v.mask)
    assert np.array_equal(np.asarray(host["fod"]), dev["fod"])
    assert np.array_equal(host["status"], dev["status"])
    host2 = csd.dwi2fod_csd_host(s, v.dwi, v.mask)       # pageable numpy input
    assert np.array_equal(np.asarray(host2["fod"]), dev["fod"])


def test_deterministic(cuda):
    v = synth.make_volume((500, 1, 1), 6, 60, (15.0, 40.0), 8, None, 91)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    a = run_gpu(s, v.dwi)
    b = run_gpu(s, v.dwi)
    assert np.array_equal(a["fod"], b["fod"])


def test_full_size_config2_properties(cuda, hr_dirs):
    """96x96x60 (553k voxels, ~50% mask): every solved voxel is a fixed point
    of its own negative set (checked in FP64), and a random sample of 3000
    voxels matches the oracle."""
    import torch
    v = synth.config2()
    s = csd.make_shared(v.grad, synth.RESPONSE)
    out = run_gpu(s, v.dwi, mask=v.mask)
    st = out["status"]
    assert np.all((st[v.mask == 0] & 0x0F) == 0)
    solved = np.nonzero((st & 0x0F) == 1)[0]
    assert len(solved) >= 0.99 * v.mask.sum()
    H = torch.from_numpy(s.HR_trans).cuda()
    F = torch.from_numpy(out["fod"][solved]).cuda().double()
    neg = (F @ H.T < 0).cpu().numpy()
    got = csd.negmask_to_bool(out["negmask"][solved], 300)
    assert (neg == got).all(axis=1).mean() >= 0.999
    rng = np.random.default_rng(0)
    idx = rng.choice(np.nonzero(v.mask)[0], 3000, replace=False)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi[idx])
    sub = {k: out[k][idx] for k in ("fod", "negmask", "iterations", "status")}
    check_parity(sub, ref)


@pytest.mark.parametrize("lmax", [6, 8, 10])
def test_tiled_set_equals_warp_set(cuda, lmax):
    """The phased set() over tiles of 64 voxels sums in the order of the
    warp-per-voxel set(), so a whole phased run -- with masked voxels,
    non-finite samples, negative samples and a ragged last tile -- ends on
    the same FODs, sets, statuses and iteration counts bit for bit."""
    import torch

    from mrtrix3_b200 import autotune
    ndw, nb0 = (60, 6) if lmax <= 8 else (90, 8)
    v = synth.make_volume((37, 29, 7), nb0, ndw, (15.0, 40.0), lmax, 0.6, 300 + lmax)
    dwi = v.dwi.copy()
    rng = np.random.default_rng(lmax)
    dwi[rng.choice(len(dwi), 20, replace=False), 3] = np.nan
    dwi[rng.choice(len(dwi), 20, replace=False), 7] = -50.0
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=lmax)
    d = torch.from_numpy(dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    outs = []
    try:
        for kind in (1, 2, 2, 2):  # the tiled kernel three times: its result may not depend on timing
            autotune.set_knob(autotune.KNOB_SET_KIND, kind)
            st = csd.State(s, v.n_voxels)
            st.run(d, mask=m)
            outs.append(st.fod())
            st.close()
    finally:
        autotune.set_knob(autotune.KNOB_SET_KIND, 0)
    for o in outs[1:]:
        for k in ("fod", "negmask", "status", "iterations"):
            assert np.array_equal(outs[0][k], o[k]), k
    assert (outs[1]["status"] == csd.STATUS_NONFINITE).sum() > 0


def test_host_phased_after_shared_objects_are_replaced(cuda):
    """The host-buffer entry point caches its device workspace between calls.
    A scheme object destroyed and replaced by a new one (which may reuse the
    address) must get a fresh workspace and uploaded tables: each call equals
    the device-buffer result for its own scheme."""
    import gc

    import torch
    v = synth.make_volume((31, 17, 3), 6, 60, (15.0, 40.0), 8, 0.7, 94)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    for lmax in (8, 6, 8, 4, 8):
        s = csd.make_shared(v.grad, synth.RESPONSE, lmax=lmax)
        host = csd.dwi2fod_csd_host_phased(s, v.dwi, v.mask)
        st = csd.State(s, v.n_voxels)
        st.run(d, mask=m)
        dev = st.fod()
        st.close()
        assert np.array_equal(host["fod"], dev["fod"]), lmax
        assert np.array_equal(host["status"], dev["status"]), lmax
        del s, st
        gc.collect()


@pytest.mark.parametrize("passes", [None, "2"])
def test_host_phased_finishes_slabs_left_iterating(cuda, monkeypatch, passes):
    """The host-buffer entry point enqueues a bounded number of passes per
    slab (16 by default; 2 here to force the case) and finishes any slab
    whose voxels are still iterating with the synchronous run on the same
    state: outputs equal the device-buffer method's bit for bit, plain and
    warm-started by the shipped network, over several slabs."""
    import os

    import torch

    from mrtrix3_b200.warmstart import WarmStartNet
    if passes:
        monkeypatch.setenv("CSD_HOST_PASSES", passes)
    else:
        monkeypatch.delenv("CSD_HOST_PASSES", raising=False)
    net = WarmStartNet.load(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                         "mrtrix3_b200", "data", "warmstart_c5.npz"))
    grad = synth.config5_scheme()
    dwi = synth.voxel_signals(np.random.default_rng(95), grad, 300_000, (15.0, 40.0))
    s = csd.make_shared(grad, synth.RESPONSE)
    d = torch.from_numpy(dwi).cuda()
    st = csd.State(s, len(dwi))
    for w in (None, net):
        host = csd.dwi2fod_csd_host_phased(s, dwi, None, net=w)
        st.run(d, warm=w.predict(d) if w is not None else None)
        dev = st.fod()
        assert np.array_equal(host["fod"], dev["fod"]), w
        assert np.array_equal(host["status"], dev["status"]), w
        assert np.array_equal(host["iterations"], dev["iterations"].astype(np.uint8)), w
    st.close()
