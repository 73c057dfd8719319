"""Benchmark: single-shell CSD voxels/s on B200 (one JSON line on rank 0).

Workload (default): 140x140x96 synthetic volume, ellipsoid mask ~45%,
6 b=0 + 60 b=3000 directions, lmax 8, 300 constraint directions, SNR U[15,40]
(seed-driven synthetic data; no public dataset is named for this path).
A step is one full deconvolution of the masked volume.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--method warm|plain|persistent]

N>1 (torchrun, one process per GPU): each rank deconvolves its own volume
(different seed, same size) -- weak scaling with no data-path collective;
the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CSD voxels/s lmax8: warm-start batched vs plain GPU, p99 rel err≤1e-4 vs FP64"
UNIT = "voxels/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(seed: int):
    from mrtrix3_b200 import synth
    return synth.config5(seed=seed)


def flops_per_voxel(iters, negcount, status, n, ndw, nr, nhr=300):
    """Algorithmic FLOPs of the plain trajectory: 2*ndw*(nr+n) + T*2*nhr*n
    + S*(k*n(n+1) + n^3/3 + 2n^2), S solves (T-1 if converged), k the final
    negative-set size standing in for each solve's."""
    T = iters.astype(np.float64)
    conv = (status & 0x0F) == 1
    S = np.where(conv, T - 1, T)
    k = negcount.astype(np.float64)
    f = 2.0 * ndw * (nr + n) + T * 2.0 * nhr * n + S * (k * n * (n + 1) + n ** 3 / 3.0 + 2.0 * n * n)
    solved = (status & 0x0F) >= 1
    solved &= (status & 0x0F) <= 2
    return float(f[solved].sum())


def cpu_baseline(vol, sample_target_s: float = 12.0):
    """The FP64 oracle (a restatement of the reference's CPU path; the
    reference itself needs Eigen, absent here) on all host cores over a
    bounded sample of the masked voxels."""
    from mrtrix3_b200 import synth
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    sh = O.OracleShared(vol.grad, synth.RESPONSE, synth.load_hr_dirs())
    idx = np.nonzero(vol.mask)[0]
    rng = np.random.default_rng(0)
    probe = rng.choice(idx, min(len(idx), 400 * cores), replace=False)
    t0 = time.perf_counter()
    sh.solve(vol.dwi[probe], nthreads=cores)
    dt = time.perf_counter() - t0
    rate = len(probe) / dt
    n = int(min(len(idx), max(len(probe), rate * sample_target_s)))
    samp = rng.choice(idx, n, replace=False)
    t0 = time.perf_counter()
    sh.solve(vol.dwi[samp], nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} random masked voxels of the workload, FP64 oracle restatement, {cores} threads, "
                      f"{dt:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    vol = make_workload(seed=5)
    cb = []
    for _ in range(args.warmup):
        pass
    vals = []
    for _ in range(max(1, args.steps)):
        cb.append(cpu_baseline(vol, sample_target_s=max(3.0, 60.0 / max(1, args.steps))))
        vals.append(cb[-1]["value"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "config": workload_config(vol, "cpu-oracle"),
            "cpu_baseline": {**cb[-1], "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "vs_baseline": None}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(vol, method):
    return {"workload": "140x140x96 synthetic DWI, mask ~45%, 6 b=0 + 60 b=3000 dirs, lmax 8, 300 HR dirs, "
                        "SNR U[15,40]",
            "dims": list(vol.dims), "n_voxels": vol.n_voxels, "n_masked": vol.n_masked, "nsh": 45,
            "method": method, "l2": "inputs larger than L2 (dwi 497 MB, fod 339 MB per step)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="persistent", choices=["persistent", "plain", "warm"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    from mrtrix3_b200 import csd, synth

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    vol = make_workload(seed=5 + rank)
    sh = csd.make_shared(vol.grad, synth.RESPONSE)
    dwi = torch.from_numpy(vol.dwi).to(dev)
    mask = torch.from_numpy(vol.mask).to(dev)
    stream = torch.cuda.current_stream()

    def step():
        return csd.dwi2fod_csd(sh, dwi, mask=mask, want_negmask=True, stream=stream)

    for _ in range(max(3, args.warmup)):
        out = step()
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            out = step()
        e1.record(stream)
        barrier()
    ms_total = e0.elapsed_time(e1)
    ms = torch.tensor([ms_total], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_total = float(ms.item())
    ms_step = ms_total / args.steps
    n_masked = vol.n_masked
    value = n_masked * world / (ms_step / 1e3)

    # algorithmic work of this step
    iters = out["iterations"].cpu().numpy()
    status = out["status"].cpu().numpy()
    negc = np.unpackbits(out["negmask"].cpu().numpy().view(np.uint8), axis=1).sum(axis=1)
    flops = flops_per_voxel(iters, negc, status, sh.nSH(), sh.n_dw, sh.n_init)
    peaks, peak_kind = load_peaks()
    achieved_tflops = flops / (ms_step / 1e3) / 1e12
    roofline = {"bound": "tensor", "achieved": achieved_tflops, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                "frac": achieved_tflops / peaks["bf16_tflops"], "traffic": None,
                "peak_source": f"bf16 dense burst, {peak_kind}",
                "kernel": "csd_persistent_kernel<45>", "flops_per_launch": flops,
                "hbm_gbs": (vol.n_voxels * (66 * 4 + 45 * 4 + 3)) / (ms_step / 1e3) / 1e9}

    # end to end through the host-buffer C ABI entry point (pinned inputs)
    pinned = torch.from_numpy(vol.dwi).pin_memory()
    pmask = torch.from_numpy(vol.mask).pin_memory()
    csd.dwi2fod_csd_host(sh, pinned, pmask.numpy())
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = csd.dwi2fod_csd_host(sh, pinned, pmask.numpy())
    barrier()
    e2e_s = (time.perf_counter() - t0) / args.steps
    t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_s = float(t.item())
    e2e = {"value": n_masked * world / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(vol.dwi.nbytes + vol.mask.nbytes),
           "d2h_bytes_per_step": int(vol.n_voxels * (45 * 4 + 2)),
           "api": "csd_dwi2fod_host (pinned host buffers, copies inside the timed region)"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 (fp64 refinement residual)", "data": "synthetic",
            "config": workload_config(vol, args.method), "roofline": roofline, "e2e": e2e,
            "gpu_launches": args.steps, "clocks": clk.summary(),
            "mean_iterations": float(iters[(status & 0x0F) == 1].mean()),
            "status_counts": {"converged": int(((status & 0x0F) == 1).sum()), "niter": int(((status & 0x0F) == 2).sum()),
                              "fp64": int(((status & 0x10) != 0).sum()), "cholfail": int(((status & 0x20) != 0).sum())}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(vol)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
