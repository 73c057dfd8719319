"""Host-side SH set-up of amp2sh (mrtrix3_b200/sh.py) against the FP64 oracle
and the rules of DWI::compute_SH2amp_mapping (core/dwi/gradient.h:326-374).
CPU only."""
import numpy as np
import pytest

from mrtrix3_b200 import sh


def _fib_dirs(n, seed=0):
    i = np.arange(n) + 0.5
    el = np.arccos(1.0 - 2.0 * i / n)
    az = np.pi * (1.0 + 5.0 ** 0.5) * i
    rng = np.random.default_rng(seed)
    return np.stack([az + rng.normal(0, 1e-3, n), el], axis=1)


@pytest.mark.parametrize("lmax", [0, 2, 4, 8, 10, 12])
def test_init_transform_matches_oracle(lmax):
    from oracle import oracle as O
    dirs = _fib_dirs(97, seed=lmax)
    dirs = np.vstack([dirs, [[0.3, 0.0], [1.0, np.pi], [2.0, np.pi / 2]]])  # poles and the equator
    got = sh.init_transform(dirs, lmax)
    want = O.init_transform(dirs, lmax)
    assert got.shape == want.shape == (len(dirs), sh.n_for_l(lmax))
    assert np.max(np.abs(got - want)) <= 1e-12


def test_l_for_n():
    # SH::LforN: 2 floor((sqrt(1 + 8N) - 3) / 4)
    cases = {0: 0, 1: 0, 5: 0, 6: 2, 14: 2, 15: 4, 27: 4, 28: 6, 44: 6, 45: 8, 60: 8, 66: 10, 300: 22}
    for n, l in cases.items():
        assert sh.l_for_n(n) == l, n
    for l in range(0, 20, 2):
        assert sh.l_for_n(sh.n_for_l(l)) == l


def test_sh2amp_mapping_lmax_rules():
    d60 = _fib_dirs(60)
    m, l = sh.sh2amp_mapping(d60)
    assert l == 8 and m.shape == (60, 45)            # default cap of 8
    m, l = sh.sh2amp_mapping(d60, lmax=4)
    assert l == 4 and m.shape == (60, 15)
    m, l = sh.sh2amp_mapping(d60, lmax=12)
    assert l == 8                                     # capped by the direction count
    m, l = sh.sh2amp_mapping(_fib_dirs(20))
    assert l == 4                                     # LforN(20) = 4
    with pytest.raises(ValueError):
        sh.sh2amp_mapping(d60, lmax=3)
    with pytest.raises(ValueError):
        sh.sh2amp_mapping(d60, lmax=-2)


def _cond(m):
    s = np.linalg.svd(m, compute_uv=False)
    return s[0] / s[-1]


def test_sh2amp_mapping_drops_lmax_when_poorly_conditioned():
    # directions in a cap of the sphere: lmax 8 is ill-conditioned
    rng = np.random.default_rng(3)
    n = 60
    dirs = np.stack([rng.uniform(0, 2 * np.pi, n), np.arccos(rng.uniform(0.55, 1.0, n))], axis=1)
    m, l = sh.sh2amp_mapping(dirs)
    assert l < 8
    assert _cond(m) < 100.0 or l == 0
    assert _cond(sh.init_transform(dirs, l + 2)) >= 100.0
    # a requested lmax is kept however poor the conditioning
    m, l = sh.sh2amp_mapping(dirs, lmax=8)
    assert l == 8 and _cond(m) >= 100.0


def test_pinv_is_left_inverse():
    m = sh.init_transform(_fib_dirs(60), 8)
    p = sh.pinv(m)
    assert p.shape == (45, 60)
    assert np.max(np.abs(p @ m - np.eye(45))) < 1e-10
    # the least-squares fit of amplitudes sampled from a known function
    c = np.random.default_rng(1).normal(size=45)
    assert np.allclose(p @ (m @ c), c, atol=1e-10)


def test_cartesian_to_azel_round_trip():
    d = _fib_dirs(50)
    xyz = np.stack([np.cos(d[:, 0]) * np.sin(d[:, 1]), np.sin(d[:, 0]) * np.sin(d[:, 1]), np.cos(d[:, 1])], axis=1)
    back = sh.cartesian_to_azel(3.0 * xyz)
    assert np.allclose(np.cos(back[:, 0]), np.cos(d[:, 0])) and np.allclose(np.sin(back[:, 0]), np.sin(d[:, 0]))
    assert np.allclose(back[:, 1], d[:, 1])


def test_amp2sh_cli_rejects_options_before_any_device_work(tmp_path):
    from mrtrix3_b200 import amp2sh, mif
    img = mif.Image(data=np.ones((2, 2, 1, 6), np.float32), vox=[2.0, 2.0, 2.0, 1.0])
    p = str(tmp_path / "amp.mif")
    mif.write(p, img)
    dirs = str(tmp_path / "dirs.txt")
    np.savetxt(dirs, _fib_dirs(6))
    with pytest.raises(SystemExit, match="normalise"):
        amp2sh.run([p, str(tmp_path / "o.mif"), "-directions", dirs, "-normalise"])
    with pytest.raises(SystemExit, match="directions or diffusion encoding"):
        amp2sh.run([p, str(tmp_path / "o.mif")])
    with pytest.raises(SystemExit, match="does not match"):
        np.savetxt(dirs, _fib_dirs(7))
        amp2sh.run([p, str(tmp_path / "o.mif"), "-directions", dirs])
    open(str(tmp_path / "o.mif"), "w").close()
    with pytest.raises(SystemExit, match="already exists"):
        amp2sh.run([p, str(tmp_path / "o.mif"), "-directions", dirs])
