"""Autotuner for the CSD launch shapes.

Times candidate values of the launch knobs of csd_set_launch_config (warps
per block of the persistent kernel and of the phased solve kernel, the
projection kernel -- mma.sync or tcgen05 -- and its blocks per SM) on a
probe volume, keeps the fastest, and caches
the choice per (GPU name, nSH, constraint directions, DW directions) in a
JSON file (default ~/.cache/mrtrix3_b200/launch.json, or $CSD_TUNE_CACHE).
Outputs do not depend on the knobs, so tuning never changes results.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import csd

(KNOB_PERSISTENT, KNOB_SOLVE, KNOB_PROJ, KNOB_TC_PROJECTION, KNOB_SOLVE_KIND, KNOB_SET_KIND, KNOB_INFER,
 KNOB_CYCLE_JUMP, KNOB_HOST_SLABS, KNOB_AMP2SH_KIND, KNOB_REUSE, KNOB_HOST_ASYNC, KNOB_ASSEMBLY,
 KNOB_HOST_CONC) = range(14)
# the projection kernel is chosen before its blocks per SM (which only the
# mma.sync kernel uses).  The solve kernel's warps per block apply to the
# kernel the default tcgen05 assembly feeds (up to 32 warps at lmax 8; the
# mma.sync-assembly kernel caps them at what its tables leave room for).
# The grouped solve kernels assemble with mma.sync, whose FP32 sums differ
# from the tcgen05 assembly's, so they are not tuning candidates: tuning
# never changes results.
CANDIDATES = {KNOB_PERSISTENT: [8, 12, 16], KNOB_SOLVE: [16, 24, 32], KNOB_TC_PROJECTION: [1, 2],
              KNOB_PROJ: [1, 2]}


def cache_path() -> str:
    return os.environ.get("CSD_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "mrtrix3_b200",
                                                          "launch.json"))


def _key(shared) -> str:
    import torch
    return f"{torch.cuda.get_device_name()}|nsh={shared.nSH()}|nhr={shared.n_hr}|ndw={shared.n_dw}"


def set_knob(which: int, value: int):
    csd.lib().csd_set_launch_config.argtypes = [__import__("ctypes").c_int, __import__("ctypes").c_int]
    csd.check(csd.lib().csd_set_launch_config(which, value))


def apply(config: dict):
    for k, v in config.items():
        set_knob(int(k), int(v))


def _time(fn, reps=3):
    import torch
    fn()
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    return best


def tune(shared, dwi, mask=None, use_cache: bool = True, verbose: bool = False) -> dict:
    """Pick and apply the fastest launch shapes for this scheme on this GPU."""
    path = cache_path()
    key = _key(shared)
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except Exception:
            cache = {}
        if key in cache:
            apply(cache[key]["config"])
            return cache[key]
    st = csd.State(shared, dwi.shape[0])
    best = {}
    timings = {}
    for knob, values in CANDIDATES.items():
        res = {}
        for v in values:
            set_knob(knob, v)
            if knob == KNOB_PERSISTENT:
                res[v] = _time(lambda: csd.dwi2fod_csd(shared, dwi, mask=mask))
            else:
                res[v] = _time(lambda: st.run(dwi, mask=mask))
        v_best = min(res, key=res.get)
        set_knob(knob, v_best)
        best[str(knob)] = v_best
        timings[str(knob)] = {str(k): round(t * 1e3, 3) for k, t in res.items()}
        if verbose:
            print("knob", knob, timings[str(knob)], "->", v_best, flush=True)
    entry = {"config": best, "ms": timings, "probe_voxels": int(dwi.shape[0])}
    cache[key] = entry
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        json.dump(cache, open(path, "w"), indent=1)
    except OSError:
        pass
    st.close()
    return entry
