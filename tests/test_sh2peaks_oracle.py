"""The sh2peaks restatement (oracle/sh2peaks_ref.py) on the CPU: its Legendre
functions agree with the oracle's (pinned bit for bit against the
reference's legendre.h), its analytic derivatives agree with finite
differences of the amplitude, and it recovers the fibre directions of
sums of delta FODs, in amplitude order, with duplicates merged."""
import numpy as np
import pytest

from mrtrix3_b200 import csd
from oracle import oracle as O
from oracle import sh2peaks_ref as S


def test_legendre_matches_pinned_oracle():
    x = np.linspace(-0.99, 0.99, 37)
    for m in range(0, 9):
        a = S.plm_sph(8, m, x, np.sqrt(1 - x * x))
        for i, xv in enumerate(x):
            b = O.plm_sph(8, m, xv)
            np.testing.assert_allclose(a[m:, i], b[m:], rtol=1e-12, atol=1e-14)


def test_derivatives_match_finite_differences():
    rng = np.random.default_rng(0)
    sh = rng.normal(size=45)
    el, az, h = np.array([0.9]), np.array([0.4]), 1e-6
    amp, d_el, d_az, d2_el, d2_elaz, d2_az = S.derivatives(sh, 8, el, az)
    f = lambda e, a: S.derivatives(sh, 8, np.array([e]), np.array([a]))[0][0]
    assert abs(d_el[0] - (f(0.9 + h, 0.4) - f(0.9 - h, 0.4)) / (2 * h)) < 1e-5
    assert abs(d_az[0] * np.sin(0.9) - (f(0.9, 0.4 + h) - f(0.9, 0.4 - h)) / (2 * h)) < 1e-5
    g = lambda e: S.derivatives(sh, 8, np.array([e]), az)[1][0]
    assert abs(d2_el[0] - (g(0.9 + h) - g(0.9 - h)) / (2 * h)) < 1e-4


def _delta(az, el):
    return O.init_transform(np.array([[az, el]]), 8)[0]


@pytest.mark.parametrize("fibres", [[(0.3, 0.4, 1.0)], [(0.7, 1.1, 1.0), (2.6, 1.3, 0.6)],
                                    [(0.0, 1.5707963, 1.0), (1.5707963, 1.5707963, 0.8), (0.0, 0.0, 0.6)]])
def test_recovers_fibres(fibres):
    f = sum(w * _delta(az, el) for az, el, w in fibres)
    seeds = csd.default_peak_seeds().astype(np.float64)
    p = S.voxel_peaks(f, 8, seeds, npeaks=4)
    amps = np.linalg.norm(p, axis=1)
    n = len(fibres)
    assert np.isfinite(amps[:n]).all()
    assert (np.diff(amps[:n]) <= 0).all()
    for az, el, w in fibres:
        u = S.seed_vectors(np.array([[az, el]]))[0]
        best = max(abs(np.dot(u, p[i] / amps[i])) for i in range(n))
        assert best > 0.995


def test_isotropic_and_nan_give_no_peaks():
    f = np.zeros(45)
    f[0] = 1.0
    seeds = csd.default_peak_seeds().astype(np.float64)
    assert np.isnan(S.voxel_peaks(f, 8, seeds)).all()
    f[3] = np.nan
    assert np.isnan(S.voxel_peaks(f, 8, seeds)).all()
