"""Generates fmls_golden.npz: FOD segmentation fixtures from the oracle's
restatement of Segmenter::operator() (oracle/fmls_ref.py).

Cases (seeded): 48 synthetic FODs at lmax 8 (sums of 1-3 truncated delta
functions, DC in [0.1, 0.5], N(0, 0.02) on every coefficient), segmented
with fod2fixel's defaults, with -fmls_no_thresholds, and with merge ratio
0.5.  Stored per case: the float32 coefficient rows, the lobe counts and the
first 24 lobes of each voxel as [mean dir (3), peak dir (3), integral, max
peak] (float32, zeros past the count).

    python tests/golden/make_fmls_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

CASES = {"default": dict(integral_threshold=0.0, peak_value_threshold=0.1, merge_ratio=1.0),
         "no_thresholds": dict(integral_threshold=0.0, peak_value_threshold=0.0, merge_ratio=1.0),
         "merge_0.5": dict(integral_threshold=0.0, peak_value_threshold=0.1, merge_ratio=0.5)}
WIDTH = 24


def main():
    from oracle import fmls_ref
    from test_fmls_host import synthetic_fods
    rows = synthetic_fods(48, 8, seed=2024, noise=0.02).astype(np.float32)
    out = {"rows": rows}
    for name, kw in CASES.items():
        seg = fmls_ref.Segmenter(8, **kw)
        counts = np.zeros(len(rows), np.int32)
        fx = np.zeros((len(rows), WIDTH, 8), np.float32)
        for v, r in enumerate(rows.astype(np.float64)):
            lobes = seg(r)
            counts[v] = len(lobes)
            for q, lb in enumerate(lobes[:WIDTH]):
                fx[v, q] = np.concatenate([lb["mean_dir"], lb["peak_dir"], [lb["integral"], lb["max_peak"]]])
        out[name + "_counts"] = counts
        out[name + "_fixels"] = fx
    np.savez_compressed(os.path.join(HERE, "fmls_golden.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
