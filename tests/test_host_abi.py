"""CPU tests of the C ABI library: it loads, exports every declared symbol, and
its host FP64 precompute (CSD::Shared::init, csd.h:117-198) equals the oracle.
No device compute runs here."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from mrtrix3_b200 import csd, synth
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = []
    for f in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            syms += re.findall(r"^\s*(?:[\w\s\*]+?)\b(csd_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(syms))


def test_library_exports_every_declared_symbol():
    L = csd.lib()
    syms = declared_symbols()
    assert len(syms) >= 16
    for s in syms:
        assert hasattr(L, s), s
    assert set(csd.EXPORTED) <= set(syms)


@pytest.mark.parametrize("lmax,ndw", [(0, 60), (8, 64), (10, 90), (6, 45), (12, 90), (2, 12)])
def test_host_precompute_equals_oracle(hr_dirs, lmax, ndw):
    v = synth.make_volume((2, 1, 1), 6, ndw, 30.0, 8, None, 5)
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=lmax or None)
    o = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, lmax=lmax)
    assert (s.lmax, s.nSH(), s.n_init, s.n_dw, s.n_hr) == (o.lmax, o.n, o.nr, o.ndw, o.nhr)
    assert np.array_equal(s.dwis, o.dwis)
    for k in ("rconv", "M", "HR_trans", "Mt_M"):
        a, b = getattr(s, k), getattr(o, k)
        assert np.abs(a - b).max() <= 1e-14 * max(np.abs(b).max(), 1.0), k


def test_options_pass_through(hr_dirs):
    v = synth.make_volume((2, 1, 1), 6, 60, 30.0, 8, None, 5)
    s = csd.Shared(v.grad)
    s.parse_cmdline_options(lmax=[6], neg_lambda=0.5, norm_lambda=2.0, threshold=0.1, niter=7,
                            filter=[1, 1, 0.5, 0.25])
    s.set_response(synth.RESPONSE)
    s.init()
    o = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs, lmax=6, neg_lambda=0.5, norm_lambda=2.0, threshold=0.1,
                       niter=7, filter=np.array([1, 1, 0.5, 0.25]))
    assert s.niter == 7 and s.lmax == 6
    for k in ("rconv", "HR_trans", "Mt_M"):
        assert np.abs(getattr(s, k) - getattr(o, k)).max() <= 1e-13 * np.abs(getattr(o, k)).max()


def test_custom_directions(hr_dirs):
    v = synth.make_volume((2, 1, 1), 6, 60, 30.0, 8, None, 5)
    dirs = hr_dirs[:129].copy()
    s = csd.make_shared(v.grad, synth.RESPONSE, directions=dirs)
    o = O.OracleShared(v.grad, synth.RESPONSE, dirs)
    assert s.n_hr == 129
    assert np.abs(s.HR_trans - o.HR_trans).max() <= 1e-13 * np.abs(o.HR_trans).max()


def test_response_file(tmp_path):
    v = synth.make_volume((2, 1, 1), 6, 60, 30.0, 8, None, 5)
    p = tmp_path / "response.txt"
    p.write_text(" ".join(str(x) for x in synth.RESPONSE) + "\n")
    s = csd.Shared(v.grad)
    s.set_response(str(p))
    s.init()
    assert s.nSH() == 45


def test_errors_follow_reference_messages():
    g = synth.grad_table(2, synth.fibonacci_hemisphere(5))
    with pytest.raises(csd.CSDError, match="too few directions"):
        csd.make_shared(g, synth.RESPONSE)
    g = synth.grad_table(2, synth.fibonacci_hemisphere(30))
    with pytest.raises(csd.CSDError, match="anisotropic"):
        csd.make_shared(g, synth.RESPONSE[:1])
    with pytest.raises(csd.CSDError, match="positive even"):
        csd.make_shared(g, synth.RESPONSE, lmax=5)
    with pytest.raises(csd.CSDError, match="compiled maximum"):
        csd.make_shared(g, synth.RESPONSE, lmax=14)
    with pytest.raises(csd.CSDError, match="single lmax"):
        s = csd.Shared(g)
        s.parse_cmdline_options(lmax=[6, 8])
    L = csd.lib()
    assert L.csd_shared_nsh(None) == csd.lib().csd_shared_nsh(None) < 0


def test_state_queries_and_launch_knobs_reject_bad_arguments():
    """The state queries refuse NULL arguments and the launch knobs refuse
    values out of range (no device work: both checks come first)."""
    L = csd.lib()
    out = (ctypes.c_double * 8)()
    for name in ("csd_state_stats", "csd_state_reuse_stats", "csd_state_assembly_stats"):
        fn = getattr(L, name)
        fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        assert fn(None, out) == csd.CSD_ERR_INVALID, name
    L.csd_set_launch_config.argtypes = [ctypes.c_int, ctypes.c_int]
    assert L.csd_set_launch_config(12, 3) == csd.CSD_ERR_INVALID   # assembly: 0, 1 or 2
    assert L.csd_set_launch_config(13, 17) == csd.CSD_ERR_INVALID  # at most 16 slabs at once
    assert L.csd_set_launch_config(14, 0) == csd.CSD_ERR_INVALID   # no such knob
    assert L.csd_set_launch_config(12, 0) == csd.CSD_OK and L.csd_set_launch_config(13, 0) == csd.CSD_OK


def test_cpp_shim_compiles():
    """The C++ drop-in headers (CSD::Shared / CSD, csd.h:46-271; ICLS::Problem
    / Solver, constrained_least_squares.h:71-370; FMLS::Segmenter, fmls.h:60-291)
    and their examples compile against the C ABI."""
    ex = os.path.join(ROOT, "mrtrix3_b200", "csrc", "examples", "dwi2fod_csd_example.cpp")
    if not os.path.exists(ex):
        pytest.skip("C++ shim example not present")
    for src in (ex, os.path.join(ROOT, "mrtrix3_b200", "csrc", "examples", "icls_example.cpp"),
                os.path.join(ROOT, "mrtrix3_b200", "csrc", "examples", "fod2fixel_example.cpp"),
                os.path.join(ROOT, "mrtrix3_b200", "csrc", "examples", "fmls_segmenter_example.cpp")):
        r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
                            os.path.join(ROOT, "mrtrix3_b200", "csrc"), "-I", "/usr/local/cuda/include", src],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def _two_shell_grad(jitter=False):
    """6 b=0, 60 directions at b=1000 and 45 at b=3000, the shells interleaved."""
    d1 = synth.fibonacci_hemisphere(60)
    d3 = synth.fibonacci_hemisphere(45)
    rows = [[0, 0, 0, 0]] * 6
    rows += [[*d1[i], 1000.0 + (5.0 * ((i % 3) - 1) if jitter else 0.0)] for i in range(60)]
    rows += [[*d3[i], 3000.0] for i in range(45)]
    g = np.array(rows, np.float64)
    order = np.random.default_rng(3).permutation(len(g))
    return g[order]


@pytest.mark.parametrize("want,b", [([1000], 1000.0), ([3000], 3000.0), ([1000.5], 1000.0), ([2990], 3000.0),
                                    (None, 3000.0)])
def test_shells_option_selects_one_shell(hr_dirs, want, b):
    """-shells picks the one non-b=0 shell (shells.cpp:111-239 under
    select_shells(true, false, true), csd.h:64); the tables then equal the
    oracle's on the scheme holding only that shell."""
    g = _two_shell_grad()
    s = csd.Shared(g)
    s.parse_cmdline_options(shells=want)
    s.set_response(synth.RESPONSE)
    s.init()
    expect = np.nonzero(g[:, 3] == b)[0]
    assert np.array_equal(np.asarray(s.dwis), expect)
    keep = np.nonzero((g[:, 3] == 0) | (g[:, 3] == b))[0]
    o = O.OracleShared(g[keep], synth.RESPONSE, hr_dirs)
    assert np.array_equal(keep[o.dwis], expect)
    for k in ("rconv", "M", "HR_trans", "Mt_M"):
        a, r = getattr(s, k), getattr(o, k)
        assert np.abs(a - r).max() <= 1e-14 * max(np.abs(r).max(), 1.0), k


def test_shells_option_range_and_errors():
    g = _two_shell_grad(jitter=True)
    # within the shell's [min, max] range (995..1005)
    s = csd.make_shared(g, synth.RESPONSE, shells=[1003])
    assert np.array_equal(np.asarray(s.dwis), np.nonzero(np.abs(g[:, 3] - 1000) <= 5)[0])
    cases = [([-5], "negative b-values"),
             ([0], "User selected 0 non b=0 shells"),
             ([1000, 3000], "User selected 2 non b=0 shells"),
             ([1000, 0], "not compatible with b=0 data"),
             ([1000, 1001], "more than once"),
             ([2000], "Unable to robustly select desired shell b=2000")]
    for want, msg in cases:
        with pytest.raises(csd.CSDError, match=msg):
            csd.make_shared(g, synth.RESPONSE, shells=want)
    # no b=0 volumes: a requested b=0 shell is an error of its own
    with pytest.raises(csd.CSDError, match="no such data was found"):
        csd.make_shared(g[g[:, 3] > 0], synth.RESPONSE, shells=[0, 1000])
