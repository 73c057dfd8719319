"""GPU parity of fod2fixel's FMLS segmenter (csd_fmls_segment through the C
ABI) against the oracle's restatement of Segmenter::operator()
(oracle/fmls_ref.py): per voxel the same lobes in the same order.  The
amplitudes are FP64 on both sides but summed in another order, so a lobe
boundary may move where two amplitudes tie to rounding: counts must agree
on at least 98% of voxels and the values of agreeing voxels to 1e-4."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

pytestmark = pytest.mark.gpu


def _fods(n, lmax, seed, noise):
    from test_fmls_host import synthetic_fods
    return synthetic_fods(n, lmax, seed, noise)


def _segment(rows, lmax, mask=None, max_fixels=0, **kw):
    import torch

    from mrtrix3_b200 import fmls
    seg = fmls.Segmenter(lmax, **kw)
    c, f = seg.segment(torch.from_numpy(np.ascontiguousarray(rows, np.float32)).cuda(),
                       None if mask is None else torch.from_numpy(mask.astype(np.uint8)).cuda(),
                       max_fixels=max_fixels)
    torch.cuda.synchronize()
    return c.cpu().numpy(), f.cpu().numpy()


def _check(counts, fx, rows, lmax, atol=1e-4, min_agree=0.98, **kw):
    from oracle import fmls_ref
    seg = fmls_ref.Segmenter(lmax, **{k: v for k, v in kw.items()})
    agree = 0
    for v, r in enumerate(rows.astype(np.float32).astype(np.float64)):
        lobes = seg(r)
        if len(lobes) != counts[v]:
            continue
        agree += 1
        for q, lb in enumerate(lobes[:fx.shape[1]]):
            want = np.concatenate([lb["mean_dir"], lb["peak_dir"], [lb["integral"], lb["max_peak"]]])
            np.testing.assert_allclose(fx[v, q], want, rtol=1e-4, atol=atol)
    assert agree >= min_agree * len(rows), f"{agree} of {len(rows)} voxels agree"


@pytest.mark.parametrize("lmax,noise", [(8, 0.01), (8, 0.04), (6, 0.02), (10, 0.02)])
def test_segment_matches_oracle(lmax, noise):
    rows = _fods(60, lmax, seed=lmax + int(noise * 100), noise=noise)
    counts, fx = _segment(rows, lmax)
    assert counts.sum() > 0
    _check(counts, fx, rows, lmax)


def test_segment_thresholds_and_merging():
    rows = _fods(40, 8, seed=21, noise=0.03)
    kw = dict(integral_threshold=0.01, peak_value_threshold=0.05, merge_ratio=0.4)
    counts, fx = _segment(rows, 8, **kw)
    _check(counts, fx, rows, 8, **kw)


def test_segment_mask_layout_and_invalid_rows():
    import torch

    from mrtrix3_b200 import fmls, sh
    n = sh.n_for_l(8)
    rows = _fods(30, 8, seed=4, noise=0.01).astype(np.float32)
    rows[3, 0] = -1.0
    rows[5, 9] = np.nan
    mask = np.ones(30, bool)
    mask[[1, 7]] = False
    c_ref, f_ref = _segment(rows, 8, mask=mask)
    assert c_ref[1] == 0 and c_ref[7] == 0 and c_ref[3] == 0 and c_ref[5] == 0
    # coefficient-major storage ([nsh][n], coefficients n apart)
    t = torch.from_numpy(np.ascontiguousarray(rows.T)).cuda().t()
    seg = fmls.Segmenter(8)
    c2, f2 = seg.segment(t, torch.from_numpy(mask.astype(np.uint8)).cuda())
    np.testing.assert_array_equal(c2.cpu().numpy(), c_ref)
    np.testing.assert_array_equal(f2.cpu().numpy(), f_ref)
    assert t.shape[1] == n


def test_segment_overflow_and_maxnum():
    # an isotropic FOD (every amplitude tied: hundreds of lobes) among others
    rows = _fods(12, 8, seed=8, noise=0.06)
    rows[4] = 0.0
    rows[4, 0] = 0.5
    kw = dict(integral_threshold=0.0, peak_value_threshold=0.0)
    counts, fx = _segment(rows, 8, **kw)
    assert counts.max() > 16        # voxels run again with room for all their lobes
    assert fx.shape[1] == counts.max()
    _check(counts, fx, rows, 8, **kw)
    c3, f3 = _segment(rows, 8, max_fixels=3, **kw)
    np.testing.assert_array_equal(c3, np.minimum(counts, 3))
    np.testing.assert_array_equal(f3, fx[:, :3])


def test_fod2fixel_cli(tmp_path):
    from mrtrix3_b200 import fmls, fod2fixel, mif
    from oracle import fmls_ref
    nx, ny, nz = 4, 3, 2
    rows = _fods(nx * ny * nz, 8, seed=31, noise=0.01).astype(np.float32)
    data = rows.reshape(nz, ny, nx, -1).transpose(2, 1, 0, 3)
    src = tmp_path / "fod.mif"
    mif.write(str(src), mif.Image(data=data, vox=[2.0, 2.0, 2.0, 1.0]))
    out = tmp_path / "fixels"
    assert fod2fixel.run([str(src), str(out), "-afd", "afd.mif", "-peak_amp", "peak.mif", "-disp", "disp.mif"]) == 0
    index = mif.read(str(out / "index.mif"))
    dirs = mif.read(str(out / "directions.mif")).data
    afd = mif.read(str(out / "afd.mif")).data.reshape(-1)
    peak = mif.read(str(out / "peak.mif")).data.reshape(-1)
    disp = mif.read(str(out / "disp.mif")).data.reshape(-1)
    assert index.data.shape == (nx, ny, nz, 2) and int(index.keyval["nfixels"]) == len(afd)
    assert dirs.shape == (len(afd), 3, 1)
    np.testing.assert_array_equal(disp, (afd / peak).astype(np.float32))
    seg = fmls_ref.Segmenter(8)
    agree = 0
    for x in range(nx):
        for y in range(ny):
            for z in range(nz):
                cnt, off = index.data[x, y, z]
                lobes = seg(data[x, y, z].astype(np.float64))
                if len(lobes) != cnt:
                    continue
                agree += 1
                for q, lb in enumerate(lobes):
                    np.testing.assert_allclose(dirs[off + q, :, 0], lb["mean_dir"], atol=1e-4)
                    np.testing.assert_allclose(afd[off + q], lb["integral"], rtol=1e-4)
    assert agree >= 0.9 * nx * ny * nz
    assert fmls.FIXEL_FIELDS == 8


def test_builtin_tables_give_the_same_lobes():
    """csd_fmls_create_default (tables built by the library) against the
    host tables: the same lobes, values to 1e-5 (the SH transform and
    Legendre table agree to 1e-13)."""
    import torch

    from mrtrix3_b200 import fmls
    rows = _fods(80, 8, seed=77, noise=0.02).astype(np.float32)
    d = torch.from_numpy(rows).cuda()
    c1, f1 = fmls.Segmenter(8).segment(d, max_fixels=16)
    c2, f2 = fmls.Segmenter(8, builtin=True).segment(d, max_fixels=16)
    c1, f1, c2, f2 = (t.cpu().numpy() for t in (c1, f1, c2, f2))
    same = c1 == c2
    assert same.mean() >= 0.98
    np.testing.assert_allclose(f2[same], f1[same], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("case,kw", [("default", {}),
                                     ("no_thresholds", dict(integral_threshold=0.0, peak_value_threshold=0.0)),
                                     ("merge_0.5", dict(merge_ratio=0.5))])
def test_segment_matches_golden(case, kw):
    """Against the committed oracle fixtures (tests/golden/fmls_golden.npz):
    counts equal on >= 98% of voxels, values of those to 1e-4."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "fmls_golden.npz"))
    counts, fx = _segment(g["rows"], 8, max_fixels=24, **kw)
    want_c = np.minimum(g[case + "_counts"], 24)
    same = counts == want_c
    assert same.mean() >= 0.98
    np.testing.assert_allclose(fx[same], g[case + "_fixels"][same], rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("kw", [{}, dict(integral_threshold=0.0, peak_value_threshold=0.0, merge_ratio=0.6)])
def test_segment_matches_c_oracle_large(kw):
    """4096 voxels against the threaded C restatement (oracle/fmls_oracle.c):
    counts equal on >= 99%, values of those to 1e-4."""
    import os as _os

    from oracle import fmls_ref
    rows = _fods(4096, 8, seed=123, noise=0.015).astype(np.float32)
    counts, fx = _segment(rows, 8, max_fixels=16, **kw)
    rc, rf = fmls_ref.segment_batch_c(fmls_ref.Segmenter(8, **kw), rows.astype(np.float64), max_out=16,
                                      nthreads=_os.cpu_count() or 1)
    same = np.minimum(rc, 16) == counts
    assert same.mean() >= 0.99
    np.testing.assert_allclose(fx[same], rf[same], rtol=1e-4, atol=1e-4)


def test_segment_rounds_match_c_oracle():
    """40,000 voxels: three rounds of the growing / peak / finishing kernels
    (16,384 voxels a round, the last one partial), masked voxels among them;
    every 8th voxel against the C restatement."""
    import os as _os

    from oracle import fmls_ref
    rows = _fods(40000, 8, seed=321, noise=0.01).astype(np.float32)
    mask = np.ones(len(rows), np.uint8)
    mask[::7] = 0
    counts, fx = _segment(rows, 8, mask=mask, max_fixels=16)
    assert not counts[mask == 0].any()
    idx = np.nonzero(mask)[0][::8]
    rc, rf = fmls_ref.segment_batch_c(fmls_ref.Segmenter(8), rows[idx].astype(np.float64), max_out=16,
                                      nthreads=_os.cpu_count() or 1)
    same = np.minimum(rc, 16) == counts[idx]
    assert same.mean() >= 0.99
    np.testing.assert_allclose(fx[idx][same], rf[same], rtol=1e-4, atol=1e-4)
