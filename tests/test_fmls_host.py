"""CPU tests of fod2fixel's FMLS segmenter: the direction set and its tables
(mrtrix3_b200.directions / fmls), and the segmentation core
(csrc/fmls_core.cuh) built for the host and compared with the oracle's
literal restatement of Segmenter::operator() (oracle/fmls_ref.py)."""
import ctypes
import math
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from mrtrix3_b200 import directions, fmls, sh  # noqa: E402
from oracle import fmls_ref  # noqa: E402


@pytest.fixture(scope="module")
def dirset():
    u = directions.unit_vectors(directions.load_tessellation_1281())
    return u, directions.adjacency_1281()


def test_tessellation_and_adjacency(dirset):
    u, adj = dirset
    assert u.shape == (1281, 3)
    np.testing.assert_allclose(np.linalg.norm(u, axis=1), 1.0, atol=1e-12)
    deg = np.array([len(a) for a in adj])
    # a geodesic sphere of 2562 points, antipodes merged: 12 / 2 vertices of
    # degree 5, the rest 6; 7680 / 2 edges
    assert (deg == 5).sum() == 6 and (deg == 6).sum() == 1275 and deg.sum() // 2 == 3840
    for i, a in enumerate(adj):
        assert i not in a and list(a) == sorted(a)
        for j in a:
            assert i in adj[j]


def test_adjacency_file_matches_hull(dirset):
    u, adj = dirset
    again = directions.hull_adjacency(u)
    assert all(np.array_equal(a, b) for a, b in zip(adj, again))


def test_integration_weights(dirset):
    u, _ = dirset
    w = directions.integration_weights(u)
    # a least-squares fit over 1326 basis functions (lmax 50) with 1281 weights
    assert abs(w.sum() - 4.0 * math.pi) < 1e-6
    azel = np.stack([np.arctan2(u[:, 1], u[:, 0]), np.arccos(u[:, 2])], axis=1)
    Y = sh.init_transform(azel, 16)
    integ = w @ Y
    assert abs(integ[0] - 2.0 * math.sqrt(math.pi)) < 1e-6
    assert np.abs(integ[1:]).max() < 1e-6


def test_fast_lookup_matches_exhaustive(dirset):
    u, adj = dirset
    look = directions.FastLookup(u, adj)
    rng = np.random.default_rng(3)
    p = rng.normal(size=(3000, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    for q in p:
        assert look.select_direction(q) == int(np.argmax(np.abs(u @ q)))
    for i in range(0, 1281, 97):  # the set's own directions
        assert look.select_direction(u[i]) == i


def test_precomputed_al_rows():
    tab = directions.precomputed_al(8, 2562)
    el = 100 * math.pi / 2561
    for m in range(9):
        P = sh.plm_sph(8, m, np.array([math.cos(el)]))
        for l in range(m + (m & 1), 9, 2):
            assert abs(tab[100, l * l // 4 + m] - P[l][0]) < 1e-13
    assert np.all(tab[0, [l * l // 4 + m for l in range(0, 9, 2) for m in range(1, l + 1)]] == 0.0)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    from mrtrix3_b200 import build
    build.gen_fmls_inc()
    out = tmp_path_factory.mktemp("fmls") / "libfmls_host.so"
    csrc = os.path.join(ROOT, "mrtrix3_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    os.path.join(ROOT, "tests", "fmls_host_harness.cpp"), os.path.join(csrc, "fmls_tables.cpp"),
                    os.path.join(csrc, "shared_init.cpp")], check=True)
    return ctypes.CDLL(str(out))


def synthetic_fods(n, lmax, seed, noise):
    """Sums of 1-3 truncated delta functions with random weights and
    directions, DC scaled into [0.1, 0.5], plus Gaussian noise on every
    coefficient (which makes small positive and negative lobes)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        k = int(rng.integers(1, 4))
        azel = np.stack([rng.uniform(-np.pi, np.pi, k), np.arccos(rng.uniform(-1, 1, k))], 1)
        c = (rng.uniform(0.3, 1.0, k)[:, None] * sh.init_transform(azel, lmax)).sum(0)
        c = c / c[0] * rng.uniform(0.1, 0.5)
        c = c + rng.normal(0.0, noise, c.shape)
        c[0] = abs(c[0])
        out.append(c)
    return np.array(out)


def host_segment(lib, tables, rows, max_out=64):
    ct = fmls.c_tables(tables)
    rows = np.ascontiguousarray(rows, np.float64)
    counts = np.zeros(len(rows), np.int32)
    fx = np.zeros((len(rows), max_out, 8), np.float32)
    lib.fmls_host_segment(ctypes.byref(ct), ctypes.c_void_p(rows.ctypes.data), len(rows), max_out,
                          ctypes.c_void_p(counts.ctypes.data), ctypes.c_void_p(fx.ctypes.data))
    return counts, fx


def oracle_rows(seg, rows):
    return [seg(r) for r in rows]


def compare(counts, fx, ref, atol=1e-6):
    for v, lobes in enumerate(ref):
        assert counts[v] == len(lobes), f"voxel {v}: {counts[v]} lobes, oracle {len(lobes)}"
        for q, lb in enumerate(lobes[:fx.shape[1]]):
            want = np.concatenate([lb["mean_dir"], lb["peak_dir"], [lb["integral"], lb["max_peak"]]])
            np.testing.assert_allclose(fx[v, q], want.astype(np.float32), rtol=1e-6, atol=atol)


@pytest.mark.parametrize("lmax,noise,merge,integral,peak", [
    (8, 0.01, 1.0, 0.0, 0.1),     # fod2fixel's defaults
    (8, 0.05, 1.0, 0.0, 0.0),     # -fmls_no_thresholds: every positive lobe
    (8, 0.02, 0.5, 0.0, 0.1),     # lobes merged across bridges
    (12, 0.02, 0.3, 0.01, 0.05),
    (6, 0.003, 0.8, 0.0, 0.1),
    (10, 0.03, 0.0, 0.0, 0.1),    # merge ratio 0: every bridge merges
])
def test_core_matches_oracle(harness, lmax, noise, merge, integral, peak):
    T = fmls.FMLSTables(lmax, integral, peak, merge)
    seg = fmls_ref.Segmenter(lmax, integral, peak, merge)
    rows = synthetic_fods(24, lmax, seed=lmax * 100 + int(noise * 1000), noise=noise)
    counts, fx = host_segment(harness, T, rows)
    compare(counts, fx, oracle_rows(seg, rows))
    assert counts.sum() > 0


def test_core_merges_lobes(harness):
    # at merge ratio 0 a lobe holds the peaks of the lobes it absorbed: fewer,
    # larger lobes than with the default ratio 1
    rows = synthetic_fods(16, 8, seed=11, noise=0.03)
    c1, _ = host_segment(harness, fmls.FMLSTables(8, 0.0, 0.0, 1.0), rows)
    c0, _ = host_segment(harness, fmls.FMLSTables(8, 0.0, 0.0, 0.0), rows)
    assert c0.sum() < c1.sum()


def test_core_edge_cases(harness):
    T = fmls.FMLSTables(8)
    seg = fmls_ref.Segmenter(8)
    n = sh.n_for_l(8)
    iso = np.zeros(n)
    iso[0] = 1.0                       # constant amplitude: every direction tied, taken in index order
    neg_dc = synthetic_fods(1, 8, 5, 0.01)[0]
    neg_dc[0] = -neg_dc[0]             # DC not positive: no lobes
    nan_row = synthetic_fods(1, 8, 6, 0.01)[0]
    nan_row[7] = np.nan                # a non-finite coefficient: no lobes
    neg_fod = -synthetic_fods(1, 8, 7, 0.0)[0]
    neg_fod[0] = 1e-3                  # the largest-magnitude amplitude negative: no lobes
    zero = np.zeros(n)
    rows = np.array([iso, neg_dc, nan_row, neg_fod, zero])
    counts, fx = host_segment(harness, T, rows)
    assert list(counts[1:]) == [0, 0, 0, 0]
    # ties break by index, so directions that are not neighbours seed lobes of
    # their own (hundreds of them) and the bridges between them are assigned
    # afterwards: as the reference's ordered multimap does
    ref = seg(iso)
    assert len(ref) > 100
    compare(counts[:1], fx[:1], [ref])
    assert abs(sum(lb["integral"] for lb in ref) - 4.0 * math.pi * sh.init_transform(np.zeros((1, 2)), 8)[0, 0]) < 1e-5


def test_core_max_out_counts_all(harness):
    rows = synthetic_fods(8, 8, seed=9, noise=0.05)
    T = fmls.FMLSTables(8, 0.0, 0.0, 1.0)
    c_all, f_all = host_segment(harness, T, rows, max_out=64)
    c2, f2 = host_segment(harness, T, rows, max_out=2)
    assert np.array_equal(c_all, c2)   # the count is every lobe kept, whatever fits
    np.testing.assert_array_equal(f2, f_all[:, :2])


def test_pack_offsets_and_disp():
    counts = np.array([2, 0, 1])
    fx = np.zeros((3, 2, 8), np.float32)
    fx[0, 0] = [1, 0, 0, 0, 1, 0, 2.0, 4.0]
    fx[0, 1] = [0, 1, 0, 0, 0, 1, 1.0, 3.0]
    fx[2, 0] = [0, 0, 1, 1, 0, 0, 0.5, 0.25]
    c, off, d, afd, pk, disp = fmls.pack(counts, fx)
    assert list(off) == [0, 2, 2] and list(afd) == [2.0, 1.0, 0.5]
    np.testing.assert_array_equal(d[2], [0, 0, 1])
    np.testing.assert_array_equal(disp, np.float32([0.5, 1.0 / 3.0, 2.0]))
    _, _, dp, _, _, _ = fmls.pack(counts, fx, dirpeak=True)
    np.testing.assert_array_equal(dp[2], [1, 0, 0])


def test_cli_argument_errors(tmp_path):
    from mrtrix3_b200 import fod2fixel, mif
    with pytest.raises(SystemExit, match="usage"):
        fod2fixel.run(["only_one"])
    with pytest.raises(SystemExit, match="nii"):
        fod2fixel.run(["a.mif", "b", "-nii"])
    bad = tmp_path / "bad.mif"
    mif.write(str(bad), mif.Image(data=np.zeros((2, 2, 2, 7), np.float32), vox=[1, 1, 1, 1]))
    with pytest.raises(SystemExit, match="SH series"):
        fod2fixel.run([str(bad), str(tmp_path / "out")])
    with pytest.raises(SystemExit, match="merge_ratio"):
        fod2fixel.thresholds({"-fmls_lobe_merge_ratio": "1.5"})
    assert fod2fixel.thresholds({"-fmls_no_thresholds": True, "-fmls_peak_value": "0.3"}) == (0.0, 0.0, 1.0)
    # unambiguous prefixes, as dwi2response's scripts pass "-peak" for -peak_amp
    pos, opt = fod2fixel._parse(["f.mif", "d", "-peak", "p.mif", "-fmls_no_thr"])
    assert pos == ["f.mif", "d"] and opt == {"-peak_amp": "p.mif", "-fmls_no_thresholds": True}
    with pytest.raises(SystemExit, match="unknown option"):
        fod2fixel._parse(["-fmls"])
    # the reference's own test command lines (testing/binaries/tests/fod2fixel)
    pos, opt = fod2fixel._parse("-nthread 1 -fmls_no_thresholds fod.mif tmp-fod2fixel3 -afd afd.mif -peak peak.mif "
                                "-disp disp.mif -force".split())
    assert pos == ["fod.mif", "tmp-fod2fixel3"]
    assert opt == {"-nthreads": "1", "-fmls_no_thresholds": True, "-afd": "afd.mif", "-peak_amp": "peak.mif",
                   "-disp": "disp.mif", "-force": True}
    full = tmp_path / "full"
    full.mkdir()
    (full / "x").write_text("")
    good = tmp_path / "good.mif"
    mif.write(str(good), mif.Image(data=np.zeros((2, 2, 2, 15), np.float32), vox=[1, 1, 1, 1]))
    with pytest.raises(SystemExit, match="not empty"):
        fod2fixel.run([str(good), str(full)])
    with pytest.raises(SystemExit, match="maxnum"):
        fod2fixel.run([str(good), str(tmp_path / "o1"), "-maxnum", "0"])
    small = tmp_path / "small_mask.mif"
    mif.write(str(small), mif.Image(data=np.ones((2, 2, 1), np.float32), vox=[1, 1, 1]))
    with pytest.raises(SystemExit, match="dimensions do not match"):
        fod2fixel.run([str(good), str(tmp_path / "o2"), "-mask", str(small)])
    with pytest.raises(SystemExit, match="non-negative"):
        fod2fixel.run([str(good), str(tmp_path / "o3"), "-fmls_peak_value", "-1"])


def test_c_abi_rejects_bad_tables():
    """csd_fmls_create / csd_fmls_segment check their arguments before any
    device call (no GPU needed)."""
    from mrtrix3_b200 import csd
    L = csd.lib()
    T = fmls.FMLSTables(8)
    h = ctypes.c_void_p()

    def create(**over):
        ct = fmls.c_tables(T)
        for k, v in over.items():
            setattr(ct, k, v)
        return L.csd_fmls_create(ctypes.byref(ct), ctypes.byref(h))

    assert L.csd_fmls_create(None, ctypes.byref(h)) == csd.CSD_ERR_INVALID
    assert create(lmax=7) == csd.CSD_ERR_INVALID          # odd lmax
    assert create(nsh=44) == csd.CSD_ERR_INVALID          # nsh not NforL(lmax)
    assert create(ndir=4096) == csd.CSD_ERR_INVALID       # more directions than the sort's width
    assert create(n_al=10) == csd.CSD_ERR_INVALID         # PrecomputedAL rows of another lmax
    assert create(n_adj=T.adj_off[-1] - 1) == csd.CSD_ERR_INVALID  # offsets and list disagree
    bad = T.adj.copy()
    bad[5] = 1281                                          # a neighbour out of range
    keep = T.adj
    T.adj = bad
    assert create() == csd.CSD_ERR_INVALID
    T.adj = keep
    assert b"neighbour" in L.csd_last_error()
    assert create(merge_ratio=-0.5) == csd.CSD_ERR_INVALID
    assert L.csd_fmls_create_default(7, 0.0, 0.1, 1.0, ctypes.byref(h)) == csd.CSD_ERR_INVALID
    assert b"lmax" in L.csd_last_error()
    assert L.csd_fmls_create_default(8, 0.0, 0.1, 1.0, None) == csd.CSD_ERR_INVALID
    assert h.value is None
    assert L.csd_fmls_segment(None, None, 0, 45, 1, None, 16, None, None, None) == csd.CSD_ERR_INVALID


def test_precomputed_al_matches_exact_values():
    """The reference's own known-answer test for SH::PrecomputedAL
    (testing/cmd/testing_unit_tests_sh_precomputer.cpp): random lmax-8
    coefficients in [-1, 1], 10,000 random unit directions, the value
    through the 512-elevation table within 1e-3 of the exact one.  Here with
    the oracle's interpolation (fmls_ref._AL, SH.h:435-460) on the host
    table (directions.precomputed_al)."""
    lmax = 8
    rng = np.random.default_rng(2)
    coefs = rng.uniform(-1.0, 1.0, sh.n_for_l(lmax))
    al = fmls_ref._AL(directions.precomputed_al(lmax, 512))
    p = rng.uniform(-1.0, 1.0, (10000, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    az = np.arctan2(p[:, 1], p[:, 0])
    el = np.arccos(p[:, 2])
    exact = sh.init_transform(np.stack([az, el], axis=1), lmax) @ coefs
    for i in range(len(p)):
        A = al.get(el[i])
        v = 0.0
        for l in range(0, lmax + 1, 2):
            v += A[l * l // 4] * coefs[l * (l + 1) // 2]
        for m in range(1, lmax + 1):
            c, s = math.cos(m * az[i]), math.sin(m * az[i])
            for l in range(m + (m & 1), lmax + 1, 2):
                v += A[l * l // 4 + m] * math.sqrt(2.0) * (c * coefs[l * (l + 1) // 2 + m] +
                                                          s * coefs[l * (l + 1) // 2 - m])
        assert abs(v - exact[i]) <= 1e-3


@pytest.mark.parametrize("lmax", [8, 12])
def test_cpp_default_tables_equal_host_tables(harness, lmax):
    """csd_fmls_create_default's C++ tables (fmls_tables.cpp) against the
    Python host tables the GPU tests use (mrtrix3_b200.fmls.FMLSTables)."""
    T = fmls.FMLSTables(lmax)
    dims = np.zeros(7, np.int32)
    steps = np.zeros(5)
    assert harness.fmls_host_default_tables(lmax, ctypes.c_void_p(dims.ctypes.data),
                                            ctypes.c_void_p(steps.ctypes.data), *([None] * 8)) == 0
    nd, nsh, al_ndir, n_al, num_az, num_el, n_grid = (int(v) for v in dims)
    assert (nd, nsh, al_ndir, n_al, num_az, num_el, n_grid) == (T.ndir, T.nsh, T.al_ndir, T.n_al, T.num_az,
                                                                T.num_el, len(T.grid))
    np.testing.assert_allclose(steps, [T.al_inc, T.az_begin, T.el_begin, T.az_step, T.el_step], rtol=1e-15)
    unit, weight = np.zeros((nd, 3)), np.zeros(nd)
    sh2amp, al = np.zeros((nd, nsh)), np.zeros((al_ndir, n_al))
    adj_off, adj = np.zeros(nd + 1, np.int32), np.zeros(len(T.adj), np.int32)
    grid_off, grid = np.zeros(num_az * num_el + 1, np.int32), np.zeros(n_grid, np.int32)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    assert harness.fmls_host_default_tables(lmax, p(dims), p(steps), p(unit), p(weight), p(sh2amp), p(al), p(adj_off),
                                            p(adj), p(grid_off), p(grid)) == 0
    np.testing.assert_allclose(unit, T.unit, rtol=0, atol=1e-15)
    np.testing.assert_array_equal(weight, T.weight)
    np.testing.assert_allclose(sh2amp, T.sh2amp, rtol=0, atol=1e-13)
    np.testing.assert_allclose(al, T.al, rtol=0, atol=1e-13)
    np.testing.assert_array_equal(adj_off, T.adj_off)
    np.testing.assert_array_equal(adj, T.adj)
    np.testing.assert_array_equal(grid_off, T.grid_off)
    np.testing.assert_array_equal(grid, T.grid)
    assert harness.fmls_host_default_tables(7, p(dims), p(steps), *([None] * 8)) == -1


GOLDEN = os.path.join(ROOT, "tests", "golden", "fmls_golden.npz")
GOLDEN_CASES = {"default": (0.0, 0.1, 1.0), "no_thresholds": (0.0, 0.0, 1.0), "merge_0.5": (0.0, 0.1, 0.5)}


@pytest.mark.parametrize("case", sorted(GOLDEN_CASES))
def test_core_reproduces_golden(harness, case):
    """The host-built core against the committed oracle fixtures
    (tests/golden/make_fmls_golden.py), bit for bit in float32."""
    g = np.load(GOLDEN)
    counts, fx = host_segment(harness, fmls.FMLSTables(8, *GOLDEN_CASES[case]), g["rows"].astype(np.float64),
                              max_out=24)
    np.testing.assert_array_equal(counts, g[case + "_counts"])
    np.testing.assert_array_equal(fx, g[case + "_fixels"])


def test_oracle_reproduces_golden():
    g = np.load(GOLDEN)
    seg = fmls_ref.Segmenter(8, *GOLDEN_CASES["merge_0.5"])
    for v in range(0, 48, 12):
        lobes = seg(g["rows"][v].astype(np.float64))
        assert len(lobes) == g["merge_0.5_counts"][v]
        for q, lb in enumerate(lobes[:24]):
            want = np.concatenate([lb["mean_dir"], lb["peak_dir"], [lb["integral"], lb["max_peak"]]]).astype(np.float32)
            np.testing.assert_array_equal(g["merge_0.5_fixels"][v, q], want)


@pytest.mark.parametrize("case", sorted(GOLDEN_CASES))
def test_c_oracle_reproduces_golden(case):
    """The C restatement (oracle/fmls_oracle.c: the reference's vector of
    lobes with masks, erased on merges) against the same fixtures, threaded."""
    g = np.load(GOLDEN)
    seg = fmls_ref.Segmenter(8, *GOLDEN_CASES[case])
    counts, fx = fmls_ref.segment_batch_c(seg, g["rows"].astype(np.float64), max_out=24, nthreads=4)
    np.testing.assert_array_equal(counts, g[case + "_counts"])
    np.testing.assert_array_equal(fx, g[case + "_fixels"])


def test_c_oracle_matches_host_core(harness):
    rows = synthetic_fods(64, 10, seed=31, noise=0.03)
    kw = (0.0, 0.0, 0.3)
    c1, f1 = fmls_ref.segment_batch_c(fmls_ref.Segmenter(10, *kw), rows, max_out=32, nthreads=2)
    c2, f2 = host_segment(harness, fmls.FMLSTables(10, *kw), rows, max_out=32)
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_allclose(f1, f2, rtol=1e-6, atol=1e-6)


def test_cli_writes_the_fixel_directory(tmp_path, monkeypatch):
    """fod2fixel's command line end to end on the CPU, the device segmenter
    replaced by the C restatement: index (count, offset), directions and the
    metric images in voxel order, x fastest; offset 0 where a voxel has no
    fixels (the reference leaves those index entries unwritten)."""
    import torch

    from mrtrix3_b200 import fod2fixel, mif

    class HostSegmenter:
        def __init__(self, lmax, integral, peak, merge):
            self.ref = fmls_ref.Segmenter(lmax, integral, peak, merge)

        def segment(self, fod, mask=None, max_fixels=0):
            rows = fod.numpy().astype(np.float64)
            c, f = fmls_ref.segment_batch_c(self.ref, rows, max_out=64, nthreads=2)
            if mask is not None:
                c = np.where(mask.numpy() != 0, c, 0)
            if max_fixels:
                c = np.minimum(c, max_fixels)
            return torch.from_numpy(c), torch.from_numpy(f)

    monkeypatch.setattr(fmls, "Segmenter", HostSegmenter)
    monkeypatch.setattr(torch.cuda, "current_device", lambda: 0)
    monkeypatch.setattr(torch.Tensor, "to", lambda self, *a, **k: self)
    nx, ny, nz = 3, 2, 2
    rows = synthetic_fods(nx * ny * nz, 8, seed=41, noise=0.01).astype(np.float32)
    rows[5] = 0.0  # no lobes
    data = rows.reshape(nz, ny, nx, -1).transpose(2, 1, 0, 3)
    src = tmp_path / "fod.mif"
    mif.write(str(src), mif.Image(data=data, vox=[2.0, 2.0, 2.0, 1.0], keyval={"comments": "x"}))
    out = tmp_path / "fixels"
    assert fod2fixel.run([str(src), str(out), "-afd", "afd.mif", "-peak", "pk.mif", "-disp", "disp.mif",
                          "-maxnum", "3"]) == 0
    index = mif.read(str(out / "index.mif"))
    dirs = mif.read(str(out / "directions.mif")).data
    afd = mif.read(str(out / "afd.mif")).data.reshape(-1)
    pk = mif.read(str(out / "pk.mif")).data.reshape(-1)
    c, f = fmls_ref.segment_batch_c(fmls_ref.Segmenter(8), rows.astype(np.float64), max_out=64, nthreads=2)
    c = np.minimum(c, 3)
    assert int(index.keyval["nfixels"]) == c.sum() == len(afd)
    assert index.keyval["comments"] == "x"
    off = 0
    for v in range(nx * ny * nz):
        z, r = divmod(v, nx * ny)
        y, x = divmod(r, nx)
        cnt, o = index.data[x, y, z]
        assert cnt == c[v] and o == (off if c[v] else 0)
        for q in range(c[v]):
            np.testing.assert_array_equal(dirs[off + q, :, 0], f[v, q, 0:3])
            assert afd[off + q] == f[v, q, 6] and pk[off + q] == f[v, q, 7]
        off += c[v]
    np.testing.assert_array_equal(mif.read(str(out / "disp.mif")).data.reshape(-1), (afd / pk).astype(np.float32))
