"""GPU parity on the larger workloads: the 140x140x96 lmax-10 volume (8 b=0 +
90 DW) and a batch of uneven volumes with independent direction sets in one
persistent launch, replayed from a captured CUDA graph.  Full-size outputs
are checked by size-independent properties (every solved voxel is a fixed
point of its own negative set, checked in FP64) and a random sample against
the FP64 oracle (p99 rel err <= 1e-4, >= 99.5% same final set)."""
import numpy as np
import pytest

from mrtrix3_b200 import csd, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _check(out, v, s, hr_dirs, lmax, n_sample=1500, seed=0):
    import torch
    st = out["status"]
    solved = np.nonzero((st & 0x0F) == 1)[0]
    inside = np.nonzero(v.mask)[0] if v.mask is not None else np.arange(v.n_voxels)
    assert len(solved) >= 0.999 * len(inside)
    H = torch.from_numpy(s.HR_trans).cuda()
    F = torch.from_numpy(out["fod"][solved]).cuda().double()
    neg = (F @ H.T < 0).cpu().numpy()
    got = csd.negmask_to_bool(out["negmask"][solved], s.n_hr)
    assert (neg == got).all(axis=1).mean() >= 0.999
    idx = np.random.default_rng(seed).choice(inside, min(n_sample, len(inside)), replace=False)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, lmax=lmax).solve(v.dwi[idx])
    den = np.abs(ref["F"]).max(axis=1)
    rel = np.abs(out["fod"][idx].astype(np.float64) - ref["F"]).max(axis=1) / den
    assert np.percentile(rel, 99) <= 1e-4
    assert np.mean(np.all(out["negmask"][idx].view(np.uint32) == ref["negmask"], axis=1)) >= 0.995


def test_config3_lmax10_full_volume(cuda, hr_dirs):
    import torch
    v = synth.config3()
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=10)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    st = csd.State(s, v.n_voxels)
    st.run(d, mask=m)
    _check(st.fod(), v, s, hr_dirs, 10)


def test_uneven_volumes_one_graph_launch(cuda, hr_dirs):
    """Eight uneven volumes (random direction sets) in one persistent launch,
    captured into a CUDA graph and replayed; the replay equals the eager call."""
    import torch
    vols = synth.config4(seed=41, n_volumes=8, scale=0.5)
    shs = [csd.make_shared(v.grad, synth.RESPONSE) for v in vols]
    ds = [torch.from_numpy(v.dwi).cuda() for v in vols]
    ms = [torch.from_numpy(v.mask).cuda() for v in vols]
    eager = csd.solve_volumes(shs, ds, masks=ms, want_negmask=True)
    torch.cuda.synchronize()
    eager = [{k: t.clone() for k, t in o.items()} for o in eager]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        csd.solve_volumes(shs, ds, masks=ms, want_negmask=True, stream=s)  # workspace allocated before capture
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        outs = csd.solve_volumes(shs, ds, masks=ms, want_negmask=True, stream=s)
    for o in outs:
        for t in o.values():
            t.zero_()
    g.replay()
    torch.cuda.synchronize()
    for a, b in zip(eager, outs):
        assert torch.equal(a["fod"], b["fod"])
        assert torch.equal(a["status"], b["status"])
    for i, (v, sh, o) in enumerate(zip(vols, shs, outs)):
        _check({k: t.cpu().numpy() for k, t in o.items()}, v, sh, hr_dirs, 8, n_sample=300, seed=i)


def test_autotuner_picks_valid_shapes_and_results_do_not_change(cuda, tmp_path, monkeypatch):
    import torch

    from mrtrix3_b200 import autotune
    monkeypatch.setenv("CSD_TUNE_CACHE", str(tmp_path / "launch.json"))
    v = synth.make_volume((48, 48, 24), 6, 60, (15.0, 40.0), 8, 0.5, 55)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    before = csd.dwi2fod_csd(s, d, mask=m)["fod"].clone()
    st = csd.State(s, v.n_voxels)
    st.run(d, mask=m)
    before_phased = st.fod()["fod"]
    entry = autotune.tune(s, d, mask=m)
    for k, vals in autotune.CANDIDATES.items():
        assert entry["config"][str(k)] in vals
    after = csd.dwi2fod_csd(s, d, mask=m)["fod"]
    st.run(d, mask=m)
    assert torch.equal(before, after)
    assert np.array_equal(before_phased, st.fod()["fod"])
    again = autotune.tune(s, d, mask=m)          # served from the cache
    assert again["config"] == entry["config"]
    autotune.apply({str(k): 0 for k in autotune.CANDIDATES})


@pytest.mark.parametrize("lmax", [8, 10])
def test_tcgen05_projection_equals_mma_projection(cuda, hr_dirs, lmax):
    """The phased method's tcgen05 projection (accumulators in tensor memory)
    and its mma.sync projection compute the same products in the same FP16
    hi/lo split with FP32 accumulation, so the sets and FODs agree exactly
    on every voxel (plain and warm starts), and both stay on the oracle."""
    import torch

    from mrtrix3_b200 import autotune
    ndw, nb0 = (60, 6) if lmax == 8 else (90, 8)
    v = synth.make_volume((40, 36, 20), nb0, ndw, (15.0, 40.0), lmax, 0.5, 77 + lmax)
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=lmax)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    plain = csd.dwi2fod_csd(s, d, mask=m, want_negmask=True)
    warm = plain["negmask"].clone()
    warm[:, 0] ^= 0x5  # a near-miss first set for every voxel
    outs = {}
    try:
        for kind in (1, 2):
            autotune.set_knob(autotune.KNOB_TC_PROJECTION, kind)
            st = csd.State(s, v.n_voxels)
            st.run(d, mask=m)
            a = st.fod()
            st.run(d, mask=m, warm=warm)
            outs[kind] = (a, st.fod(), st.stats())
            st.close()
    finally:
        autotune.set_knob(autotune.KNOB_TC_PROJECTION, 0)
    for i in range(2):
        for k in ("fod", "negmask", "status", "iterations"):
            assert np.array_equal(outs[1][i][k], outs[2][i][k]), k
    assert outs[1][2]["projected"] == outs[2][2]["projected"]
    _check(outs[2][0], v, s, hr_dirs, lmax, n_sample=800)


@pytest.mark.parametrize("lmax", [4, 6, 8])
def test_grouped_solve_equals_warp_solve(cuda, lmax):
    """The phased solve with 16 or 8 lanes per voxel (2 or 4 voxels per warp)
    performs every voxel's arithmetic in the order of the warp-per-voxel
    solve, so FODs, sets, statuses and iteration counts are identical --
    plain and warm-started, and with every factorisation forced into the
    FP64 fallback."""
    import torch

    from mrtrix3_b200 import autotune
    v = synth.make_volume((40, 36, 20), 6, 60, (15.0, 40.0), lmax, 0.5, 90 + lmax)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=lmax)
    s64 = csd.Shared(v.grad)
    s64.parse_cmdline_options(lmax=lmax)
    s64.fp64_condition = 1.0
    s64.set_response(synth.RESPONSE)
    s64.init()
    plain = csd.dwi2fod_csd(s, d, mask=m, want_negmask=True)
    warm = plain["negmask"].clone()
    warm[:, 0] ^= 0x9
    outs = {}
    try:
        # the grouped kernels assemble with mma.sync: compare with the warp
        # kernel on the same assembly
        autotune.set_knob(autotune.KNOB_ASSEMBLY, 1)
        for kind in (1, 2, 3):
            autotune.set_knob(autotune.KNOB_SOLVE_KIND, kind)
            res = []
            for sh, w in ((s, None), (s, warm), (s64, None)):
                st = csd.State(sh, v.n_voxels)
                st.run(d, mask=m, warm=w)
                res.append(st.fod())
                st.close()
            outs[kind] = res
    finally:
        autotune.set_knob(autotune.KNOB_SOLVE_KIND, 0)
        autotune.set_knob(autotune.KNOB_ASSEMBLY, 0)
    assert np.all(outs[1][2]["status"][v.mask.astype(bool)] & csd.STATUS_FP64)
    for kind in (2, 3):
        for a, b in zip(outs[1], outs[kind]):
            for k in ("fod", "negmask", "status", "iterations"):
                assert np.array_equal(a[k], b[k]), (kind, k)


def test_cycle_jump_equals_full_iteration(cuda):
    """The 140x140x96 benchmark volume (6 b=0 + 60 DW, lmax 8) holds voxels
    that two-cycle until niter.  Jumping such a cycle to its last call once
    it is exactly periodic gives the FODs, sets, statuses and iteration
    counts of running every call -- plain and warm-started -- while the
    number of passes drops.  The warm-started run assembles every solve
    (factor reuse off): its FP32 arithmetic is the one with cycling voxels
    on this volume.  Both assemblies (tcgen05, mma.sync) are run; the
    jump must be exact for each, and the volume must hold a voxel that
    cycles to niter under at least one of them."""
    import os

    import torch

    from mrtrix3_b200 import autotune
    from mrtrix3_b200.warmstart import WarmStartNet
    v = synth.config5(seed=5)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    here = os.path.dirname(os.path.abspath(__file__))
    net = WarmStartNet.load(os.path.join(here, "..", "mrtrix3_b200", "data", "warmstart_c5.npz"))
    warm = net.predict(d, mask=m)
    st = csd.State(s, v.n_voxels)
    outs, passes = {}, {}
    try:
        autotune.set_knob(autotune.KNOB_REUSE, 2)
        for asm in (2, 1):
            autotune.set_knob(autotune.KNOB_ASSEMBLY, asm)
            for knob in (2, 1):
                autotune.set_knob(autotune.KNOB_CYCLE_JUMP, knob)
                for name, w in (("plain", None), ("warm", warm)):
                    st.run(d, mask=m, warm=w)
                    outs[(asm, knob, name)] = st.fod()
                    passes[(asm, knob, name)] = st.stats()["passes"]
    finally:
        autotune.set_knob(autotune.KNOB_CYCLE_JUMP, 0)
        autotune.set_knob(autotune.KNOB_REUSE, 0)
        autotune.set_knob(autotune.KNOB_ASSEMBLY, 0)
    for name in ("plain", "warm"):
        exercised = 0
        for asm in (2, 1):
            a, b = outs[(asm, 2, name)], outs[(asm, 1, name)]
            for k in ("fod", "negmask", "status", "iterations"):
                assert np.array_equal(a[k], b[k]), (asm, name, k)
            cyc = int(((a["status"] & 0x0F) == csd.STATUS_NITER).sum())
            exercised += cyc
            if cyc:
                assert passes[(asm, 1, name)] < passes[(asm, 2, name)]
        assert exercised >= 1  # the case is exercised
    # the persistent kernel's per-voxel loop jumps the same cycles
    pers = {}
    try:
        autotune.set_knob(autotune.KNOB_REUSE, 2)
        for knob in (2, 1):
            autotune.set_knob(autotune.KNOB_CYCLE_JUMP, knob)
            o = csd.dwi2fod_csd(s, d, mask=m, want_negmask=True)
            pers[knob] = {k: t.cpu().numpy() for k, t in o.items()}
    finally:
        autotune.set_knob(autotune.KNOB_CYCLE_JUMP, 0)
    for k in ("fod", "negmask", "status", "iterations"):
        assert np.array_equal(pers[2][k], pers[1][k]), ("persistent", k)
    assert ((pers[1]["status"] & 0x0F) == csd.STATUS_NITER).sum() >= 1


def test_benchmark_volume_shipped_network(cuda, hr_dirs):
    """The configuration bench.py times: the 140x140x96 benchmark volume
    (seed 5, 846,816 masked voxels, 6 b=0 + 60 DW, lmax 8) warm-started by
    the shipped network (data/warmstart_c5.npz) through State.run.  Every
    solved voxel is a fixed point of its own set; 4000 sampled voxels match
    the FP64 oracle (p99 <= 1e-4, >= 99.5% identical final sets); the warm
    start needs fewer solves than the plain start on the same volume."""
    import os

    import torch

    from mrtrix3_b200.warmstart import WarmStartNet
    v = synth.config5(seed=5)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    net = WarmStartNet.load(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                         "mrtrix3_b200", "data", "warmstart_c5.npz"))
    st = csd.State(s, v.n_voxels)
    st.run(d, mask=m, warm=net.predict(d, mask=m))
    warm_solves = st.stats()["solved"]
    _check(st.fod(), v, s, hr_dirs, 8, n_sample=4000, seed=5)
    st.run(d, mask=m)
    plain_solves = st.stats()["solved"]
    assert warm_solves < 0.75 * plain_solves, (warm_solves, plain_solves)


def test_async_phased_run_equals_synchronous_and_replays_from_a_graph(cuda, hr_dirs):
    """csd_state_run_async (no host synchronisation) gives the results of
    csd_state_set + csd_state_warm + csd_state_run bit for bit, plain and
    warm-started; three volumes with their own random direction sets run
    from one captured CUDA graph on three streams and replay to the same
    results."""
    import torch
    vols = synth.config4(seed=43, n_volumes=3, scale=0.4)
    shs = [csd.make_shared(v.grad, synth.RESPONSE) for v in vols]
    ds = [torch.from_numpy(v.dwi).cuda() for v in vols]
    ms = [torch.from_numpy(v.mask).cuda() for v in vols]
    sts = [csd.State(sh, v.n_voxels) for sh, v in zip(shs, vols)]
    refs = []
    for st, d, m in zip(sts, ds, ms):
        st.run(d, mask=m)
        refs.append(st.fod())
    # the same, asynchronous, then with warm sets (the final sets with a bit flipped)
    for st, d, m, ref in zip(sts, ds, ms, refs):
        st.run_async(d, mask=m)
        assert st.async_result() == (0, False)
        out = st.fod()
        for k in ("fod", "negmask", "status", "iterations"):
            assert np.array_equal(out[k], ref[k]), k
        w = torch.from_numpy(ref["negmask"]).cuda()
        w[:, 0] ^= 0x5
        st.run(d, mask=m, warm=w)
        wref = st.fod()
        st.run_async(d, mask=m, warm=w)
        assert st.async_result() == (0, False)
        out = st.fod()
        for k in ("fod", "negmask", "status", "iterations"):
            assert np.array_equal(out[k], wref[k]), k
    # one graph, three streams
    main = torch.cuda.Stream()
    side = [torch.cuda.Stream() for _ in vols]
    g = torch.cuda.CUDAGraph()
    outs = []
    with torch.cuda.graph(g, stream=main):
        for st, d, m, sd in zip(sts, ds, ms, side):
            sd.wait_stream(main)
            with torch.cuda.stream(sd):
                st.run_async(d, mask=m, stream=sd)
                outs.append(st.fod(stream=sd, as_numpy=False))
            main.wait_stream(sd)
    for o in outs:
        o["fod"].zero_()
    g.replay()
    torch.cuda.synchronize()
    for o, ref, v, sh in zip(outs, refs, vols, shs):
        got = {k: t.cpu().numpy() for k, t in o.items()}
        for k in ("fod", "negmask", "status", "iterations"):
            assert np.array_equal(got[k], ref[k]), k
    del g
    for st in sts:
        st.close()
