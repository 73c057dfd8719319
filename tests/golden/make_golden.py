"""Generates tests/golden/csd_golden.npz: small seeded CSD cases with FP64 outputs.

The reference ships no golden data for `dwi2fod csd` in this tree (its
test_data submodule is absent), so these fixtures are produced by the FP64
oracle (oracle/csd_oracle.c) and accepted only when the independent
numpy/scipy implementation (oracle/np_ref.py) agrees to 1e-10 on every voxel
with identical iteration counts and negative sets.  They anchor the oracle
against regressions and give the GPU tests fixed inputs.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mrtrix3_b200 import synth  # noqa: E402
from oracle import np_ref  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csd_golden.npz")


def case(name, vol, n, lmax=0, **kw):
    hr = synth.load_hr_dirs()
    dwi = vol.dwi[:n].copy()
    sh = O.OracleShared(vol.grad, synth.RESPONSE, hr, lmax=lmax, **kw)
    r = sh.solve(dwi, nthreads=4)
    ns = np_ref.shared(vol.grad, synth.RESPONSE, hr, lmax=lmax,
                       **{k: v for k, v in kw.items() if k in ("neg_lambda", "norm_lambda", "threshold")})
    for i in range(n):
        F, it, neg = np_ref.solve_voxel(ns, dwi[i], niter=kw.get("niter", 50))
        rel = np.abs(F - r["F"][i]).max() / max(np.abs(F).max(), 1e-300)
        assert rel < 1e-10, (name, i, rel)
        assert it == r["iters"][i], (name, i, it, r["iters"][i])
        m = np.zeros(300, bool)
        m[neg] = True
        got = np.unpackbits(r["negmask"][i].view(np.uint8), bitorder="little")[:300].astype(bool)
        assert np.array_equal(m, got), (name, i)
    return {f"{name}_grad": vol.grad, f"{name}_dwi": dwi, f"{name}_F": r["F"], f"{name}_iters": r["iters"],
            f"{name}_negmask": r["negmask"], f"{name}_lmax": np.int32(sh.lmax)}


def main():
    d = {}
    d.update(case("c1", synth.config1(seed=101, voxel_limit=64), 64))
    d.update(case("c2", synth.make_volume((8, 8, 4), 6, 60, (15.0, 40.0), 8, None, seed=102), 64))
    d.update(case("l10", synth.make_volume((8, 8, 2), 8, 90, (15.0, 40.0), 10, None, seed=103), 48, lmax=10))
    d.update(case("l6thr", synth.make_volume((8, 4, 2), 6, 45, 30.0, 6, None, seed=104), 32, lmax=6,
                  threshold=0.1))
    np.savez_compressed(OUT, **d)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
