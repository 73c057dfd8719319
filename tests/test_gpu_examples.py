"""The C and C++ examples built against libcsd_b200.so and run on the GPU.

Each example is what an MRtrix3 maintainer would write against the drop-in
surfaces: dwi2fod's csd branch over csd.hpp (CSD::Shared / CSD,
cmd/dwi2fod.cpp:256-281), a batch of ICLS problems over icls.hpp
(constrained_least_squares.h:71-370), fod2fixel's segmentation over the C
ABI (cmd/fod2fixel.cpp:288-330) and over fmls.hpp (FMLS::Segmenter,
src/dwi/fmls.cpp:118-311).  The tests compile them with g++, run them, and
check their output (the dwi2fod example's FODs against the FP64 oracle).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from mrtrix3_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mrtrix3_b200", "csrc")
LIBDIR = os.path.join(ROOT, "mrtrix3_b200")


def _build(name, tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / name)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-I",
                    "/usr/local/cuda/include", os.path.join(CSRC, "examples", name + ".cpp"), "-L", LIBDIR,
                    "-lcsd_b200", "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{LIBDIR}", "-o", exe],
                   check=True)
    return exe


def _run(args):
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def test_fod2fixel_example(cuda, tmp_path):
    out = _run([_build("fod2fixel_example", tmp_path)])
    # voxel 0: one lobe along z; voxel 1: a negative DC term, no lobes
    assert "voxel 0: 1 fixel(s)" in out and "voxel 1: 0 fixel(s)" in out, out


def test_fmls_segmenter_example(cuda, tmp_path):
    out = _run([_build("fmls_segmenter_example", tmp_path)])
    assert "lobe:" in out and "voxel 0:" in out, out


def test_icls_example(cuda, tmp_path):
    out = _run([_build("icls_example", tmp_path)])
    # min ||H x - b|| subject to x >= 0 on a 2-parameter problem: x[0] = 0.75
    x0 = float(out.split("x = [")[1].split()[0])
    assert abs(x0 - 0.75) < 1e-5, out


def test_dwi2fod_csd_example(cuda, tmp_path, hr_dirs):
    v = synth.make_volume((24, 10, 2), 6, 60, (15.0, 40.0), 8, None, 123)
    np.savetxt(tmp_path / "grad.txt", v.grad)
    np.savetxt(tmp_path / "response.txt", synth.RESPONSE[None])
    v.dwi.astype(np.float32).tofile(tmp_path / "dwi.f32")
    out = _run([_build("dwi2fod_csd_example", tmp_path), str(tmp_path / "grad.txt"), str(tmp_path / "response.txt"),
                str(tmp_path / "dwi.f32"), str(v.n_voxels), str(tmp_path / "fod.f32"), "-per_voxel", "8"])
    assert "nSH 45" in out, out
    fod = np.fromfile(tmp_path / "fod.f32", np.float32).reshape(v.n_voxels, 45).astype(np.float64)
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi)
    rel = np.abs(fod - ref["F"]).max(axis=1) / np.abs(ref["F"]).max(axis=1)
    assert np.percentile(rel, 99) <= 1e-4, np.percentile(rel, 99)
    worst = float(out.split("per_voxel_max_rel_diff")[1].split()[0])
    assert worst <= 1e-4, out
