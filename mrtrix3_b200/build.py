"""Builds libcsd_b200.so in-tree for sm_100a (nvcc + g++, no JIT cache).

    python -m mrtrix3_b200.build [--force]

Sources: csrc/shared_init.cpp (host FP64 precompute), csrc/csd_solver.cu
(kernels + C ABI), csrc/csd_tc.cu (tensor-core phases), csrc/mlp.cu (warm-start
network).  The built-in constraint directions are compiled in from
data/electrostatic_repulsion_300.txt.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("CSD_BUILD_DIR", os.path.join(HERE, "_build"))
LIB = os.environ.get("CSD_LIB_OUT", os.path.join(HERE, "libcsd_b200.so"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-Xptxas", "-warn-spills"] + os.environ.get("CSD_EXTRA_NVFLAGS", "").split()
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall"]


def _inc_path():
    return os.path.join(CSRC, "hr_dirs_builtin.inc")


def gen_hr_inc():
    src = os.path.join(HERE, "data", "electrostatic_repulsion_300.txt")
    dst = _inc_path()
    if os.path.exists(dst) and os.path.getmtime(dst) >= os.path.getmtime(src):
        return
    vals = []
    for line in open(src):
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        vals.extend(line.split())
    with open(dst, "w") as f:
        f.write("// generated by mrtrix3_b200/build.py from data/electrostatic_repulsion_300.txt\n")
        f.write("static const double kBuiltinHR[%d] = {\n" % len(vals))
        for i in range(0, len(vals), 2):
            f.write("  %s, %s,\n" % (vals[i], vals[i + 1]))
        f.write("};\n")
        f.write("static std::vector<double> builtin_hr_dirs() {\n"
                "  return std::vector<double>(kBuiltinHR, kBuiltinHR + %d);\n}\n" % len(vals))


def gen_fmls_inc():
    """fmls_builtin.inc: the 1281 tessellation directions (verbatim text),
    their hull neighbours and the integration weights (least squares, numpy
    FP64, printed with 17 significant digits) for csd_fmls_create_default."""
    src = [os.path.join(HERE, "data", f) for f in ("tessellation_1281.txt", "tessellation_1281_adjacency.txt")]
    dst = os.path.join(CSRC, "fmls_builtin.inc")
    if os.path.exists(dst) and all(os.path.getmtime(dst) >= os.path.getmtime(f) for f in src):
        return
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from mrtrix3_b200 import directions
    azel = [line.split() for line in open(src[0]) if line.strip() and not line.startswith("#")]
    adj = directions.adjacency_1281()
    w = directions.integration_weights(directions.unit_vectors(directions.load_tessellation_1281()))
    off = [0]
    for a in adj:
        off.append(off[-1] + len(a))
    with open(dst, "w") as f:
        f.write("// generated by mrtrix3_b200/build.py from data/tessellation_1281*.txt\n")
        f.write("static const double kTess1281AzEl[%d] = {\n" % (2 * len(azel)))
        for a, e in azel:
            f.write("  %s, %s,\n" % (a, e))
        f.write("};\n")
        f.write("static const int kTess1281AdjOff[%d] = {%s};\n" % (len(off), ", ".join(str(v) for v in off)))
        f.write("static const int kTess1281Adj[%d] = {%s};\n" % (off[-1], ", ".join(str(int(v)) for a in adj for v in a)))
        f.write("static const double kTess1281Weight[%d] = {\n" % len(w))
        for v in w:
            f.write("  %.17g,\n" % v)
        f.write("};\n")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def sources():
    cu = [f for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]
    cpp = [f for f in sorted(os.listdir(CSRC)) if f.endswith(".cpp")]
    return cu, cpp


def build(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    gen_hr_inc()
    gen_fmls_inc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".inc", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "csd_b200.h"))
    cu, cpp = sources()
    objs = []
    for f in cpp:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if force or _stale(obj, [src] + headers):
            _run(["g++"] + CXXFLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    for f in cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if force or _stale(obj, [src] + headers):
            _run([NVCC] + ARCH + NVFLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
