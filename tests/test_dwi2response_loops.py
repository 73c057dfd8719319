"""CPU tests of dwi2response tournier / tax's control flow
(lib/mrtrix3/dwi2response/tournier.py:53-150, tax.py:53-160) with fake
CSD + segmentation steps, and of the voxel tools they use (mrthreshold -top,
maskfilter dilate, mrstats' masked mean / std as printed)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from mrtrix3_b200 import dwi2response as D  # noqa: E402


def test_dilate_six_neighbourhood():
    m = np.zeros((5, 5, 5), bool)
    m[2, 2, 2] = True
    d1 = D.dilate(m, 1)
    assert d1.sum() == 7 and d1[1, 2, 2] and d1[2, 2, 3] and not d1[1, 1, 2]
    d2 = D.dilate(m, 2)
    assert d2.sum() == 25  # the L1 ball of radius 2
    edge = np.zeros((3, 3, 3), bool)
    edge[0, 0, 0] = True
    assert D.dilate(edge, 1).sum() == 4  # clipped at the image border


def test_masked_mean_std_as_printed():
    vals = np.array([[1.0, 2.0], [3.0, np.nan], [100.0, 100.0]])
    mean, std = D.masked_mean_std(vals, np.array([True, True, False]))
    assert mean == 2.0 and std == float(f"{np.std([1.0, 2.0, 3.0], ddof=1):.6g}")
    m2, _ = D.masked_mean_std(np.array([[1.0 / 3.0, 1.0 / 3.0]]), np.array([True]))
    assert m2 == 0.333333


class FakeSteps:
    """A fixed field of first / second peak amplitudes: each call records the
    response it got and the voxels it was asked for."""

    def __init__(self, p1, p2, rf_fn=None):
        self.p1, self.p2 = np.asarray(p1, np.float32), np.asarray(p2, np.float32)
        self.calls, self.fits = [], []
        self.rf_fn = rf_fn or (lambda it, sf: np.array([10.0 + sf.sum(), -3.0, 1.0]))

    def step(self, rf, voxels):
        self.calls.append((np.array(rf), np.array(voxels)))
        v = np.asarray(voxels, bool)
        p1 = np.where(v, self.p1, 0.0).astype(np.float32)
        p2 = np.where(v, self.p2, 0.0).astype(np.float32)
        return p1, p2, np.zeros((len(v), 3), np.float32)

    def fit(self, sf, first_dir, lmax):
        self.fits.append((np.array(sf), lmax))
        return self.rf_fn(len(self.fits) - 1, sf)


def test_tournier_converges_when_no_voxel_is_added():
    rng = np.random.default_rng(0)
    dims = (6, 5, 4)
    n = 120
    p1 = rng.uniform(0.2, 1.0, n)
    p2 = rng.uniform(0.0, 0.5, n) * p1
    mask = np.ones(n, bool)
    mask[:10] = False
    f = FakeSteps(p1, p2)
    rf, sf, iters = D.tournier_loop(f.step, f.fit, mask, dims, number=8, iter_voxels=20, dilate_passes=1,
                                    max_iters=10, lmax=6)
    # iteration 0 on the whole mask with "1 -1 1" at lmax 4, then the dilated
    # top-20 voxels (inside the mask) with the user's lmax
    np.testing.assert_array_equal(f.calls[0][0], [1.0, -1.0, 1.0])
    np.testing.assert_array_equal(f.calls[0][1], mask)
    assert f.fits[0][1] == 4 and f.fits[1][1] == 6
    with np.errstate(divide="ignore", invalid="ignore"):
        cf = (np.sqrt(np.where(mask, p1, 0.0).astype(np.float32).astype(np.float64)) *
              (1.0 - np.where(mask, p2, 0.0).astype(np.float32) / np.where(mask, p1, 0.0).astype(np.float32)) ** 2)
    cf = cf.astype(np.float32)
    top20 = cf >= D.top_threshold(cf, 20)
    want_mask = mask & D.dilate(top20.reshape(4, 5, 6), 1).reshape(-1)
    np.testing.assert_array_equal(f.calls[1][1], want_mask)
    assert iters == 2 and sf.sum() == 8
    np.testing.assert_array_equal(rf, f.rf_fn(1, sf))


def test_tournier_runs_out_of_iterations_and_subset_counts_as_converged():
    # the single-fibre set only ever gains voxels when the field shifts: a
    # field where iteration k favours voxels never chosen before never
    # converges; a shrinking set converges (the script tests max(SF - SF_prev) == 0)
    n, dims = 60, (5, 4, 3)
    mask = np.ones(n, bool)

    class Shifting(FakeSteps):
        def step(self, rf, voxels):
            k = len(self.calls)
            self.calls.append((np.array(rf), np.array(voxels)))
            p1 = np.full(n, 0.5, np.float32)
            p1[(np.arange(n) + 7 * k) % n < 3] = 1.0
            return p1, np.zeros(n, np.float32), np.zeros((n, 3), np.float32)

    f = Shifting(np.ones(n), np.zeros(n))
    rf, sf, iters = D.tournier_loop(f.step, f.fit, mask, dims, number=3, iter_voxels=n, max_iters=4)
    assert iters == 4 and len(f.calls) == 4
    np.testing.assert_array_equal(sf, f.fits[-1][0])
    with pytest.raises(SystemExit, match="at least 2"):
        D.tournier_loop(f.step, f.fit, mask, dims, max_iters=1)
    with pytest.raises(SystemExit, match="iter_voxels"):
        D.tournier_loop(f.step, f.fit, mask, dims, number=10, iter_voxels=5)


def test_tax_convergence_rule():
    n = 50
    rng = np.random.default_rng(1)
    p1 = rng.uniform(0.5, 1.0, n)
    p2 = p1 * np.where(np.arange(n) % 3 == 0, 0.05, 0.5)
    mask = np.ones(n, bool)
    # coefficients: a positive one converging, a negative one jumping (its
    # "ratio" is negative, so the script never re-iterates for it)
    seq = [np.array([100.0, -40.0]), np.array([110.0, -10.0]), np.array([110.2, -80.0]), np.array([110.2, -5.0])]
    f = FakeSteps(p1, p2, rf_fn=lambda it, sf: seq[min(it, len(seq) - 1)])
    rf, sf, iters = D.tax_loop(f.step, f.fit, mask, [90.0, -45.0, 5.0], peak_ratio=0.1, max_iters=20,
                               convergence=0.5)
    assert iters == 3
    np.testing.assert_array_equal(rf, seq[2])
    np.testing.assert_array_equal(sf, (np.arange(n) % 3 == 0))
    # the mask of each iteration is the previous single-fibre set
    np.testing.assert_array_equal(f.calls[1][1], sf)
    np.testing.assert_array_equal(f.calls[0][0], [90.0, -45.0, 5.0])
    # a coefficient whose old and new values cancel: the script divides by zero
    fz = FakeSteps(p1, p2, rf_fn=lambda it, sf: [np.array([100.0, 0.0]), np.array([110.0, 0.0])][min(it, 1)])
    with pytest.raises(ZeroDivisionError):
        D.tax_loop(fz.step, fz.fit, mask, [90.0, -45.0, 5.0])
    f0 = FakeSteps(np.zeros(n), np.zeros(n))
    with pytest.raises(SystemExit, match="excluded"):
        D.tax_loop(f0.step, f0.fit, mask, [1.0, 0.0, 0.0])


def test_iterative_cli_argument_errors(tmp_path):
    with pytest.raises(SystemExit, match="-mask is required"):
        D.run(["tournier", "dwi.mif", str(tmp_path / "out.txt")])
    with pytest.raises(SystemExit, match="single lmax"):
        D.run(["tax", "dwi.mif", str(tmp_path / "out.txt"), "-mask", "m.mif", "-lmax", "8,8"])
    with pytest.raises(SystemExit, match="single b-value"):
        D.run(["tournier", "dwi.mif", str(tmp_path / "out.txt"), "-mask", "m.mif", "-shells", "1000,2000"])
    with pytest.raises(SystemExit, match="tournier and tax only"):
        D.run(["fa", "dwi.mif", str(tmp_path / "out.txt"), "-mask", "m.mif", "-shells", "1000"])
    with pytest.raises(SystemExit, match="wrong number"):
        D.run(["tax", "dwi.mif", "x", str(tmp_path / "out.txt")])


@pytest.mark.parametrize("algo,kw", [("tournier", dict(number=10, iter_voxels=30)), ("tax", dict(max_iters=4))])
def test_loops_on_the_restatements_recover_the_response(algo, kw):
    """The loops over the FP64 restatements of CSD, FMLS and amp2response
    (oracle/dwi2response_ref.py, the reference side of the GPU parity test)
    on a 60-voxel phantom made with synth.RESPONSE."""
    from mrtrix3_b200 import msmt, synth
    from oracle import dwi2response_ref as R
    rng = np.random.default_rng(5)
    grad = synth.grad_table(6, synth.fibonacci_hemisphere(60))
    dwi = synth.voxel_signals(rng, grad, 60, 50.0)
    g = msmt.normalise_scheme(grad)
    vols = msmt.cluster_shells(g[:, 3])[-1]
    rf, sf, it = R.iterative_ref(algo, g[vols], dwi[:, vols], np.ones(60, bool), (5, 4, 3), synth.load_hr_dirs(),
                                 lmax=8, **kw)
    assert 2 <= it <= 4 and sf.sum() >= 10
    assert np.abs(rf - synth.RESPONSE).max() <= 0.1 * synth.RESPONSE[0]
