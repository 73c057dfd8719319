"""CPU tests of the FP64 oracle: pins, known answers and golden fixtures."""
import ctypes
import math
import os

import numpy as np
import pytest
import scipy.special as sps

from mrtrix3_b200 import synth
from oracle import np_ref
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LEGENDRE = os.path.join(ROOT, "oracle", "_ref", "libref_legendre.so")


def test_legendre_bit_exact_vs_reference_source():
    """The restated Plm_sph equals the reference's own legendre.h:101-123, compiled from its source."""
    if not os.path.exists(REF_LEGENDRE):
        pytest.skip("oracle/_ref not built (reference tree absent)")
    ref = ctypes.CDLL(REF_LEGENDRE)
    ref.ref_plm_sph.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int, ctypes.c_double]
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-1, 1, 200), [-1.0, 0.0, 1.0, 1e-12, -0.999999]])
    for lmax in (0, 2, 8, 10, 12, 16):
        for m in range(0, lmax + 1):
            for x in xs:
                a = np.zeros(lmax + 1)
                b = np.zeros(lmax + 1)
                ref.ref_plm_sph(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), lmax, m, float(x))
                b[:] = O.plm_sph(lmax, m, float(x))
                assert np.array_equal(a[m:], b[m:]), (lmax, m, x)


def test_legendre_vs_scipy():
    """AL[l] = sqrt((2l+1)/4pi (l-m)!/(l+m)!) P_l^m(x) with the Condon-Shortley phase."""
    for lmax in (8, 12):
        for m in range(0, lmax + 1):
            for x in (-0.9, -0.3, 0.0, 0.42, 0.97):
                a = O.plm_sph(lmax, m, x)
                for l in range(m, lmax + 1):
                    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - m) / math.factorial(l + m))
                    assert a[l] == pytest.approx(norm * sps.lpmv(m, l, x), rel=1e-10, abs=1e-12)


def test_sh_transform_vs_scipy(hr_dirs):
    for lmax in (2, 8, 10):
        A = O.init_transform(hr_dirs, lmax)
        B = np_ref.sh_basis(hr_dirs, lmax)
        assert np.abs(A - B).max() < 1e-12


def test_sh_orthonormal():
    """Gauss-Legendre x uniform-azimuth quadrature of Y_i Y_j is the identity."""
    lmax = 10
    nz, nphi = 24, 48
    z, wz = np.polynomial.legendre.leggauss(nz)
    phi = (np.arange(nphi) + 0.5) * 2 * math.pi / nphi
    Z, P = np.meshgrid(z, phi, indexing="ij")
    dirs = np.stack([P.ravel(), np.arccos(Z.ravel())], 1)
    w = (wz[:, None] * np.full(nphi, 2 * math.pi / nphi)[None, :]).ravel()
    Y = O.init_transform(dirs, lmax)
    G = (Y * w[:, None]).T @ Y
    assert np.abs(G - np.eye(Y.shape[1])).max() < 1e-10


def _vol(n=256, seed=7, ndw=60, lmax=8):
    return synth.make_volume((n, 1, 1), 6, ndw, (15.0, 40.0), lmax, None, seed)


def test_oracle_matches_independent_numpy(hr_dirs):
    v = _vol(200)
    sh = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs)
    r = sh.solve(v.dwi, nthreads=2)
    ns = np_ref.shared(v.grad, synth.RESPONSE, hr_dirs)
    for i in range(200):
        F, it, neg = np_ref.solve_voxel(ns, v.dwi[i])
        assert np.abs(F - r["F"][i]).max() <= 1e-10 * np.abs(F).max()
        assert it == r["iters"][i]
        m = np.zeros(300, bool)
        m[neg] = True
        got = np.unpackbits(r["negmask"][i].view(np.uint8), bitorder="little")[:300].astype(bool)
        assert np.array_equal(m, got)


def test_shared_tables_match_numpy(hr_dirs):
    v = _vol(4, ndw=90)
    for lmax in (0, 6, 10):
        sh = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, lmax=lmax)
        ns = np_ref.shared(v.grad, synth.RESPONSE, hr_dirs, lmax=lmax)
        assert np.abs(sh.rconv - ns["rconv"]).max() < 1e-12 * np.abs(ns["rconv"]).max()
        assert np.abs(sh.M - ns["M"]).max() < 1e-12 * np.abs(ns["M"]).max()
        assert np.abs(sh.HR_trans - ns["H"]).max() < 1e-12 * np.abs(ns["H"]).max()
        assert np.abs(sh.Mt_M - ns["MtM"]).max() < 1e-12 * np.abs(ns["MtM"]).max()


def test_defaults_and_scaling(hr_dirs):
    """csd.h:127,175-180,192-195: lmax 8, c = 50*r0/300, norm_lambda = 2e-4*MtM(0,0)."""
    v = _vol(4)
    sh = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, threshold=0.2)
    assert sh.lmax == 8 and sh.n == 45 and sh.nr == 45 and sh.ndw == 60 and sh.nhr == 300
    c = 50.0 * 1700.0 / 300.0
    assert sh.scalars["threshold"] == pytest.approx(0.2 * c)
    ns = np_ref.shared(v.grad, synth.RESPONSE, hr_dirs, norm_lambda=0.0)
    assert sh.scalars["norm_lambda"] == pytest.approx(2e-4 * ns["MtM"][0, 0], rel=1e-12)


def test_lmax_above_response_zero_columns(hr_dirs):
    """csd.h:140-142: with lmax 10 and a response to l=8 the l=10 columns of M are zero."""
    v = _vol(4, ndw=90)
    sh = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, lmax=10)
    assert sh.n == 66 and sh.nr == 45
    assert np.all(sh.M[:, 45:] == 0.0)


def test_niter0_is_linear_init(hr_dirs):
    v = _vol(16)
    sh = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, niter=0)
    r = sh.solve(v.dwi, nthreads=1)
    S = np.maximum(v.dwi[:, sh.dwis].astype(np.float64), 0)
    F0 = S @ sh.rconv.T
    assert np.allclose(r["F"][:, :sh.nr], F0, rtol=1e-13, atol=1e-9)
    assert np.all(r["F"][:, sh.nr:] == 0)
    assert np.all(r["iters"] == 0)


def test_single_fibre_peak(hr_dirs):
    """A noiseless single fibre deconvolves to an FOD peaking at the fibre."""
    rng = np.random.default_rng(3)
    grad = synth.grad_table(6, synth.fibonacci_hemisphere(60))
    sh = O.OracleShared(grad, synth.RESPONSE, hr_dirs)
    dense = np.stack([rng.uniform(-np.pi, np.pi, 20000), np.arccos(rng.uniform(-1, 1, 20000))], 1)
    Y = O.init_transform(dense, 8)
    xyz = np.stack([np.sin(dense[:, 1]) * np.cos(dense[:, 0]), np.sin(dense[:, 1]) * np.sin(dense[:, 0]),
                    np.cos(dense[:, 1])], 1)
    for _ in range(5):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        x = grad[:, :3] @ u
        s = np.zeros(grad.shape[0])
        for k, r in enumerate(synth.RESPONSE):
            s += r * math.sqrt((4 * k + 1) / (4 * math.pi)) * sps.eval_legendre(2 * k, x)
        s[grad[:, 3] == 0] = 1500.0
        F = sh.solve(s[None].astype(np.float32), nthreads=1)["F"][0]
        peak = xyz[np.argmax(Y @ F)]
        assert abs(peak @ u) > math.cos(math.radians(5.0))


def test_warm_start_with_final_set(hr_dirs):
    """Starting from the converged negative set, the iteration stops after one solve."""
    v = _vol(64)
    sh = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs)
    r = sh.solve(v.dwi, nthreads=2)
    w = sh.solve(v.dwi, warm=r["negmask"], nthreads=2)
    assert np.all(w["iters"] == 2)
    assert np.array_equal(w["negmask"], r["negmask"])
    assert np.abs(w["F"] - r["F"]).max() <= 1e-9 * np.abs(r["F"]).max()


def test_mask_nonfinite_negative(hr_dirs):
    """dwi2fod.cpp:158-170: masked and non-finite voxels give zeros; negatives are clamped."""
    v = _vol(6)
    sh = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs)
    d = v.dwi.copy()
    d[1, sh.dwis[3]] = np.nan
    d[2, sh.dwis[5]] = np.inf
    d[3, sh.dwis[7]] = -50.0
    d[4] = d[3]
    d[4, sh.dwis[7]] = 0.0
    mask = np.array([1, 1, 1, 1, 1, 0], np.uint8)
    r = sh.solve(d, mask=mask, nthreads=1)
    assert list(r["status"]) == [1, 3, 3, 1, 1, 0]
    assert np.all(r["F"][[1, 2, 5]] == 0)
    assert np.array_equal(r["F"][3], r["F"][4])


def test_b0_in_table_is_ignored_and_b_value_scaling(hr_dirs):
    """Only the DW shell is used; unnormalised gradient rows are normalised with b scaled (gradient.cpp:286-310)."""
    v = _vol(8)
    g2 = v.grad.copy()
    dw = g2[:, 3] > 0
    g2[dw, :3] *= 1.0 / math.sqrt(2.0)      # |g|^2 = 0.5 -> b scaled to 1500, one shell all the same
    a = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs)
    b = O.OracleShared(g2, synth.RESPONSE, hr_dirs)
    assert np.array_equal(a.dwis, b.dwis)
    assert np.abs(a.M - b.M).max() < 1e-12


def test_multishell_picks_largest(hr_dirs):
    d1 = synth.fibonacci_hemisphere(30)
    d3 = synth.fibonacci_hemisphere(60)
    g = np.concatenate([synth.grad_table(4, d1, 1000.0), synth.grad_table(2, d3, 3000.0)])
    g[np.arange(len(g)) % 7 == 3, 3] += 15.0  # jitter within BValueEpsilon
    sh = O.OracleShared(g, synth.RESPONSE, hr_dirs)
    assert sh.ndw == 60
    assert np.all(g[sh.dwis, 3] > 2000)


def test_init_errors(hr_dirs):
    g = synth.grad_table(2, synth.fibonacci_hemisphere(5))
    with pytest.raises(RuntimeError, match="too few directions"):
        O.OracleShared(g, synth.RESPONSE, hr_dirs)
    g = synth.grad_table(2, synth.fibonacci_hemisphere(30))
    with pytest.raises(RuntimeError, match="anisotropic"):
        O.OracleShared(g, synth.RESPONSE[:1], hr_dirs)
    with pytest.raises(RuntimeError, match="positive even"):
        O.OracleShared(g, synth.RESPONSE, hr_dirs, lmax=7)
    with pytest.raises(RuntimeError, match="non b=0"):
        O.OracleShared(np.zeros((6, 4)), synth.RESPONSE, hr_dirs)


def test_golden_fixtures(hr_dirs):
    """The oracle reproduces the committed fixtures (cross-validated at generation)."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "csd_golden.npz"))
    kw = {"l6thr": {"threshold": 0.1}}
    for name in ("c1", "c2", "l10", "l6thr"):
        sh = O.OracleShared(g[f"{name}_grad"], synth.RESPONSE, hr_dirs, lmax=int(g[f"{name}_lmax"]),
                            **kw.get(name, {}))
        r = sh.solve(g[f"{name}_dwi"], nthreads=2)
        F = g[f"{name}_F"]
        assert np.abs(r["F"] - F).max() <= 1e-12 * np.abs(F).max()
        assert np.array_equal(r["iters"], g[f"{name}_iters"])
        assert np.array_equal(r["negmask"], g[f"{name}_negmask"])
