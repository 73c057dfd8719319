"""Benchmark: single-shell CSD voxels/s on B200 (one JSON line on rank 0).

Workload: a 140x140x96 synthetic DWI volume (1,881,600 voxels, centred
ellipsoid mask ~45% = 846,816 voxels), 6 b=0 + 60 b=3000 Fibonacci-hemisphere
directions, lmax 8 (45 coefficients), 300 constraint directions, SNR
U[15,40], 1-3 fibres per voxel (seeded synthetic data: no public dataset is
named for this path).  A step is one full deconvolution of the masked volume.

Headline `value`: the warm-started method -- the warm-start network's
predicted first negative sets, then the phased iteration (dense tensor-core
projection of all active voxels + warp-per-voxel assembly/factorisation of
the voxels whose set changed) run to its own stopping rule -- with inputs
resident in HBM.  `methods` also reports the plain GPU method (same passes
from the plain start), the persistent work-queue kernel with and without the
warm start, and the warm-vs-plain ratio.  `e2e` is the warm-started method
through the host-buffer C ABI entry point (csd_dwi2fod_host_phased) with
pinned host buffers and every copy inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N>1 (torchrun, one process per GPU): each rank deconvolves its own volume
(own seed, same size): weak scaling, no data-path collective; step times are
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
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
WORKLOAD = ("140x140x96 synthetic DWI (mask ~45%: 846,816 voxels), 6 b=0 + 60 b=3000 directions, lmax 8, "
            "300 constraint directions, SNR U[15,40]")
WEIGHTS = os.path.join(ROOT, "mrtrix3_b200", "data", "warmstart_c5.npz")
# DRAM bytes (read + write) per solve of the dominant solve kernels, each
# from one ncu capture on a 64^3 warm-started volume (profiles/): the
# per-launch traffic reported below scales it by the solves of a launch.
# None where no capture of the current kernel exists.
# csd_solve_kernel<45> on assembled systems: the first solves of a warm-started
# 64^3 volume (262,144 solves: 1293.9 MB read + 1307.2 MB written, the factor
# store included), profiles/csd_solve_kernel_45.md
SOLVE_DRAM_BYTES_PER_VOXEL = (1293.855e6 + 1307.167e6) / 262144
# csd_assemble_tc_kernel<45>: the same pass's 262,144 systems (15.5 MB read +
# 1104.4 MB written), profiles/csd_assemble_tc_kernel_45.md
ASM_DRAM_BYTES_PER_SYSTEM = (15.497e6 + 1104.364e6) / 262144
# csd_solve_reuse_kernel<45>: its pass-2 launch on the same volume (247,196
# reuse solves: 1304.8 MB read + 24.6 MB written), profiles/csd_solve_reuse_kernel_45.md
REUSE_DRAM_BYTES_PER_VOXEL = (1304.825e6 + 24.625e6) / 247196


FP32_SIMT_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12

# The numerics of the timed path (csd_params defaults, include/csd_b200.h).
PRECISION = {
    "projection": "tcgen05, fp16 hi+lo splits of HR_trans and F (3 products, fp32 accumulate: 22 bits)",
    "assembly": ("tcgen05 (csd_assemble_tc_kernel): 0/1 set mask x HR_trans products split fp16 hi+lo, "
                 "fp32 accumulate in tensor memory, 128 voxels a tile"),
    "factorisation": "fp32 Cholesky; fp64 re-factorisation when a pivot fails or (max L_ii/min L_ii)^2 > 1e6",
    "refine": "policy 3: one fp64-residual refinement after every solve of a voxel whose set cycles in fp32",
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

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


def cpu_baseline(vol, sample_target_s: float = 12.0):
    """The FP64 oracle (a restatement of the reference's CPU path; the
    reference itself needs Eigen, absent here) on all host cores over a
    bounded random sample of the masked voxels."""
    from mrtrix3_b200 import synth
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    sh = O.OracleShared(vol.grad, synth.RESPONSE, synth.load_hr_dirs())
    idx = np.nonzero(vol.mask)[0]
    rng = np.random.default_rng(0)
    probe = rng.choice(idx, min(len(idx), 400 * cores), replace=False)
    t0 = time.perf_counter()
    sh.solve(vol.dwi[probe], nthreads=cores)
    rate = len(probe) / (time.perf_counter() - t0)
    n = int(min(len(idx), max(len(probe), rate * sample_target_s)))
    samp = rng.choice(idx, n, replace=False)
    t0 = time.perf_counter()
    sh.solve(vol.dwi[samp], nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} random masked voxels of the workload through the FP64 oracle restatement "
                      f"(oracle/csd_oracle.c), {cores} threads, {dt:.1f} s"}


def workload_config(vol):
    return {"workload": WORKLOAD, "dims": list(vol.dims), "n_voxels": vol.n_voxels, "n_masked": vol.n_masked,
            "nsh": 45, "n_hr": 300,
            "l2": "inputs larger than L2 (dwi 497 MB + per-voxel state ~1 GB per step); no flush needed"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    vol = make_workload(seed=5)
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_baseline(vol, sample_target_s=2.0)
    vals, last = [], None
    for _ in range(max(1, args.steps)):
        last = cpu_baseline(vol, sample_target_s=max(3.0, 60.0 / max(1, args.steps)))
        vals.append(last["value"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": workload_config(vol), "method": "FP64 CPU restatement of dwi2fod csd, all host cores",
            "cpu_baseline": {**last, "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "vs_baseline": None}
    print(json.dumps(line), flush=True)
    return 0


def rel_errors(fod, F64):
    den = np.abs(F64).max(axis=1)
    return np.abs(fod.astype(np.float64) - F64).max(axis=1) / np.where(den > 0, den, 1.0)


def next_rows(dwi_dev, sample_idx):
    """Measurements of the paths beyond the headline, on this GPU (rank 0,
    N = 1): multi-tissue CSD (ICLS solver) with its C FP64 baseline on the
    host cores, and amp2sh on the benchmark volume's amplitudes."""
    import torch

    from mrtrix3_b200 import msmt, sh, synth
    from oracle import icls_ref, msmt_ref
    out = {}
    # ---- msmt_csd: 64x64x32 voxels, 4 shells, 3 tissues
    resp = [synth.MSMT_RESPONSES[k] for k in ("wm", "gm", "csf")]
    s = msmt.MSMTShared(synth.msmt_scheme())
    s.set_responses(resp)
    s.init()
    rng = np.random.default_rng(5)
    n = 64 * 64 * 32
    dwi = synth.rician(rng, synth.msmt_truth(rng, n) @ s.C.T, rng.uniform(1000.0 / 40, 1000.0 / 15, n))
    dwi = dwi.astype(np.float32)
    d = torch.from_numpy(dwi).cuda()
    x, it = s.solve(d)
    for _ in range(2):
        s.solve(d, out=x, niter=it)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    reps = 3
    for _ in range(reps):
        s.solve(d, out=x, niter=it)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # end to end through the host-buffer C ABI call (csd_icls_solve_host):
    # copies of the measurements in and the solutions out inside the timed region
    s.solve_host(dwi)
    t0 = time.perf_counter()
    for _ in range(2):
        s.solve_host(dwi)
    e2e_s = (time.perf_counter() - t0) / 2
    P = msmt_ref.problem(s.grad, s.shells, resp, [8, 0, 0], s.HR_dirs)
    idx = np.random.default_rng(1).choice(n, 500, replace=False)
    cores = os.cpu_count() or 1
    xr, itr = icls_ref.solve_batch_c(P, dwi[idx].astype(np.float64), nthreads=cores)
    xg = x.cpu().numpy()[idx].astype(np.float64)
    rel = np.abs(xg - xr).max(1) / np.abs(xr).max(1)
    # CPU baseline: the C restatement on all host cores, a bounded sample
    m = min(n, 400 * cores)
    t0 = time.perf_counter()
    icls_ref.solve_batch_c(P, dwi[:m].astype(np.float64), nthreads=cores)
    cpu_s = time.perf_counter() - t0
    out["msmt_csd"] = {
        "workload": "64x64x32 synthetic voxels (no mask: 131,072), 6 b=0 + 30/45/60 directions at b=1000/2000/3000, "
                    "3 tissues (WM lmax 8, GM, CSF: 47 parameters, 302 constraints), Rician SNR U[15,40]",
        "value": n / (ms / 1e3), "unit": "voxels/s", "ms": ms, "dtype": "f64",
        "solver_rounds_mean": float(it.float().mean().item()),
        "e2e": {"value": n / e2e_s, "unit": "voxels/s", "h2d_bytes_per_step": int(dwi.nbytes),
                "d2h_bytes_per_step": int(n * (47 + 1) * 4),
                "api": "csd_icls_solve_host (host buffers, pageable; copies made inside the timed region)"},
        "parity": {"vs": "oracle/icls_oracle.c (FP64)", "sample_voxels": len(idx),
                   "p99_rel_err": float(np.percentile(rel, 99)), "max_rel_err": float(rel.max()),
                   "rounds_equal": float(np.mean(it.cpu().numpy()[idx] == itr))},
        "cpu_baseline": {"value": m / cpu_s, "unit": "voxels/s", "cores": cores, "kind": "port",
                         "sample": f"the first {m} voxels through oracle/icls_oracle.c (FP64, refactoring per "
                                   f"solve as the reference), {cores} threads, {cpu_s:.1f} s"}}
    # ---- amp2sh: the benchmark volume's 66 amplitudes a voxel, 60-direction fit at lmax 8
    grad = synth.config5_scheme()
    from mrtrix3_b200 import csd as C
    sch = C.Shared(grad)
    sch.set_response(np.array([1.0, -0.5]))
    sch.init()
    dwis = np.asarray(sch.dwis)
    bz = np.nonzero(grad[:, 3] <= 10.0)[0]
    fit = sh.pinv(sh.init_transform(sh.cartesian_to_azel(grad[dwis, :3]), 8))
    plan = C.Amp2SHCommon(fit, dwis, bz, normalise=True)
    y = plan(dwi_dev)
    for _ in range(3):
        plan(dwi_dev, y)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(10):
        plan(dwi_dev, y)
    e1.record()
    torch.cuda.synchronize()
    ms_a = e0.elapsed_time(e1) / 10
    na = dwi_dev.shape[0]
    sel = torch.from_numpy(np.asarray(sample_idx, np.int64)).to(dwi_dev.device)
    a = dwi_dev[sel].cpu().numpy().astype(np.float64)
    ref = (a[:, dwis] * (len(bz) / (1.0 + a[:, bz].sum(1)))[:, None]) @ fit.T
    got = y[sel].cpu().numpy().astype(np.float64)
    err = np.abs(got - ref).max(1) / np.abs(ref).max(1)
    out["amp2sh"] = {
        "workload": f"{na} voxels x 66 volumes (the benchmark volume), 60 directions, lmax 8, -normalise",
        "value": na / (ms_a / 1e3), "unit": "voxels/s", "ms": ms_a, "dtype": "f64",
        "achieved_tflops_fp64": na * 2 * 45 * 60 / (ms_a / 1e3) / 1e12,
        "achieved_gbs": na * (66 + 45) * 4 / (ms_a / 1e3) / 1e9,
        "parity": {"vs": "numpy FP64 fit", "sample_voxels": len(sample_idx), "max_rel_err": float(err.max())}}
    try:
        out["fod2fixel"] = fod2fixel_row()
    except Exception as ex:  # the headline line is printed whatever happens here
        out["fod2fixel"] = {"error": f"{type(ex).__name__}: {ex}"}
    return out


def config_rows(net):
    """The benchmark's other workloads on this GPU (rank 0, N = 1), each with
    its FP64 oracle parity and CPU baseline: (1) 32x32x20, 64 directions,
    plain; (2) 96x96x60, 60 directions, plain and warm-started (the
    network's scheme); (3) 140x140x96, 90 directions, lmax 10, plain, with the
    per-voxel iteration counts; (4) 16 uneven volumes with independent random
    direction sets in one persistent work-queue launch replayed from a
    captured CUDA graph, the launch shape picked by the project's autotuner,
    beside the phased method run volume by volume."""
    import torch

    from mrtrix3_b200 import autotune, csd, synth
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    hr = synth.load_hr_dirs()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_ms(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def parity(fod, negmask, ref):
        r = rel_errors(fod, ref["F"])
        return {"p99_rel_err": float(f"{np.percentile(r, 99):.3g}"), "max_rel_err": float(f"{r.max():.3g}"),
                "negset_match": float(np.mean(np.all(negmask.view(np.uint32) == ref["negmask"], axis=1))),
                "sample_voxels": int(len(r))}

    def cpu(osh, rows, target_s=3.0):
        probe = rows[:min(len(rows), 100 * cores)]
        t0 = time.perf_counter()
        osh.solve(probe, nthreads=cores)
        rate = len(probe) / (time.perf_counter() - t0)
        m = int(min(len(rows), max(len(probe), rate * target_s)))
        t0 = time.perf_counter()
        osh.solve(rows[:m], nthreads=cores)
        dt = time.perf_counter() - t0
        return {"value": float(f"{m / dt:.4g}"), "unit": UNIT, "cores": cores, "kind": "port",
                "sample": f"{m} masked voxels, FP64 oracle restatement, {cores} threads, {dt:.1f} s"}

    def solve_tflops(stt, n):
        fl = stt["sum_neg"] * n * (n + 1) + (stt["solved"] - stt["reuse_solved"]) * (n ** 3 / 3.0 + 2 * n * n)
        ms = stt["ms_solve"] - stt["ms_reuse"]
        return float(f"{fl / max(1e-9, ms / 1e3) / 1e12:.4g}")

    def phased(v, s, lmax, warm_net=None, n_sample=3000, seed=0, reps=3):
        d = torch.from_numpy(v.dwi).cuda()
        m = torch.from_numpy(v.mask).cuda() if v.mask is not None else None
        n = v.n_masked
        st = csd.State(s, v.n_voxels)
        row = {}
        runs = [("plain", None)] + ([("warm", warm_net)] if warm_net is not None else [])
        outs = {}
        for name, nt in runs:
            ms = timed_ms(lambda: st.run(d, mask=m, warm=nt.predict(d, mask=m) if nt is not None else None), reps)
            stt = st.stats()
            outs[name] = st.fod()
            row[name] = {"voxels_per_s": float(f"{n / ms * 1e3:.4g}"), "ms": float(f"{ms:.4g}"),
                         "solves_per_voxel": float(f"{stt['solved'] / n:.3g}"),
                         "solve_kernel_tflops": solve_tflops(stt, s.nSH())}
        if warm_net is not None:
            row["warm_vs_plain"] = float(f"{row['plain']['ms'] / row['warm']['ms']:.4g}")
        st.close()
        inside = np.nonzero(v.mask)[0] if v.mask is not None else np.arange(v.n_voxels)
        idx = np.sort(np.random.default_rng(seed).choice(inside, min(n_sample, len(inside)), replace=False))
        osh = O.OracleShared(v.grad, synth.RESPONSE, hr, lmax=lmax)
        ref = osh.solve(v.dwi[idx], nthreads=cores)
        row["parity"] = {k: parity(o["fod"][idx], o["negmask"][idx], ref) for k, o in outs.items()}
        row["cpu_baseline"] = cpu(osh, v.dwi[inside])
        return row, outs

    def cpu4(rows):
        # the oracle over the first masked voxels of every volume (each its own scheme)
        t = 0.0
        m = 0
        for v, r in zip(vols, rows):
            osh = O.OracleShared(v.grad, synth.RESPONSE, hr)
            t0 = time.perf_counter()
            osh.solve(r, nthreads=cores)
            t += time.perf_counter() - t0
            m += len(r)
        return {"value": float(f"{m / t:.4g}"), "unit": UNIT, "cores": cores, "kind": "port",
                "sample": f"{m} masked voxels (1500 of each volume), FP64 oracle restatement, {cores} threads, "
                          f"{t:.1f} s"}

    out = {}
    v = synth.config1()
    out["1"], _ = phased(v, csd.make_shared(v.grad, synth.RESPONSE), 8, n_sample=v.n_voxels)
    out["1"]["workload"] = "32x32x20 (20,480 voxels), 6 b=0 + 64 DW, SNR 30, lmax 8"
    v = synth.config2()
    out["2"], _ = phased(v, csd.make_shared(v.grad, synth.RESPONSE), 8, warm_net=net, n_sample=4000)
    out["2"]["workload"] = "96x96x60, ellipsoid mask 50% (276,344 voxels), 6 b=0 + 60 DW, SNR U[15,40], lmax 8"
    v = synth.config3()
    out["3"], o3 = phased(v, csd.make_shared(v.grad, synth.RESPONSE, lmax=10), 10, n_sample=3000, reps=2)
    it = o3["plain"]["iterations"][v.mask.astype(bool)]
    out["3"]["iterations_per_voxel"] = {"mean": float(f"{it.mean():.3g}"), "p99": int(np.percentile(it, 99)),
                                        "max": int(it.max()),
                                        "histogram": {int(k): int(c) for k, c in enumerate(np.bincount(it)) if c}}
    out["3"]["workload"] = "140x140x96, mask 45% (846,816 voxels), 8 b=0 + 90 DW, SNR U[15,40], lmax 10"
    del v, o3
    # config 4: 16 uneven volumes in one persistent launch, captured and replayed
    vols = synth.config4(workers=min(16, cores))
    shs = [csd.make_shared(v.grad, synth.RESPONSE) for v in vols]
    ds = [torch.from_numpy(v.dwi).cuda() for v in vols]
    ms_ = [torch.from_numpy(v.mask).cuda() for v in vols]
    n4 = int(sum(v.n_masked for v in vols))
    big = max(range(len(vols)), key=lambda i: vols[i].n_voxels)
    tuned = autotune.tune(shs[big], ds[big][:262144], use_cache=False)
    s4 = torch.cuda.Stream()
    with torch.cuda.stream(s4):
        csd.solve_volumes(shs, ds, masks=ms_, want_negmask=True, stream=s4)  # workspace before capture
    s4.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s4):
        outs4 = csd.solve_volumes(shs, ds, masks=ms_, want_negmask=True, stream=s4)
    ms_graph = timed_ms(g.replay, 3)
    del g
    # the phased method, every volume's passes on its own stream, all in one
    # captured graph (csd_state_run_async: no host synchronisation)
    sts = [csd.State(sh_i, v.n_voxels) for sh_i, v in zip(shs, vols)]
    for st, d_i, m_i in zip(sts, ds, ms_):
        st.run_async(d_i, mask=m_i)
    torch.cuda.synchronize()
    main, side = torch.cuda.Stream(), [torch.cuda.Stream() for _ in vols]
    gp = torch.cuda.CUDAGraph()
    outs_p = []
    with torch.cuda.graph(gp, stream=main):
        for st, d_i, m_i, sd in zip(sts, ds, ms_, side):
            sd.wait_stream(main)
            with torch.cuda.stream(sd):
                st.run_async(d_i, mask=m_i, stream=sd)
                outs_p.append(st.fod(stream=sd, as_numpy=False))
            main.wait_stream(sd)
    ms_phased_graph = timed_ms(gp.replay, 3)
    left = [st.async_result()[0] for st in sts]
    ms_phased = 0.0
    for st, d_i, m_i in zip(sts, ds, ms_):
        ms_phased += timed_ms(lambda: st.run(d_i, mask=m_i), 1)
    refs, gots = [], []
    for i, (v, o) in enumerate(zip(vols, outs4)):
        inside = np.nonzero(v.mask)[0]
        idx = np.sort(np.random.default_rng(i).choice(inside, 200, replace=False))
        osh = O.OracleShared(v.grad, synth.RESPONSE, hr)
        r = osh.solve(v.dwi[idx], nthreads=cores)
        refs.append(r)
        gots.append((o["fod"].cpu().numpy()[idx], o["negmask"].cpu().numpy()[idx]))
    ref4 = {"F": np.concatenate([r["F"] for r in refs]), "negmask": np.concatenate([r["negmask"] for r in refs])}
    rows4 = [v.dwi[np.nonzero(v.mask)[0][:1500]] for v in vols]
    out["4"] = {"workload": f"16 volumes, dims U[64^3 .. 128x128x80] ({sum(v.n_voxels for v in vols):,} voxels, "
                            f"{n4:,} masked), 6 b=0 + 60 random DW each, SNR U[15,40], lmax 8",
                "persistent_graph": {"voxels_per_s": float(f"{n4 / ms_graph * 1e3:.4g}"), "ms": float(f"{ms_graph:.4g}"),
                                     "launches": 1, "tuned_shape": tuned["config"]},
                "phased_graph": {"voxels_per_s": float(f"{n4 / ms_phased_graph * 1e3:.4g}"),
                                 "ms": float(f"{ms_phased_graph:.4g}"), "graph_launches": 1,
                                 "streams": len(vols), "voxels_left_active": int(sum(left))},
                "phased_per_volume": {"voxels_per_s": float(f"{n4 / ms_phased * 1e3:.4g}"),
                                      "ms": float(f"{ms_phased:.4g}")},
                "parity": parity(np.concatenate([a for a, _ in gots]), np.concatenate([b for _, b in gots]), ref4),
                "cpu_baseline": cpu4(rows4)}
    autotune.apply({str(k): 0 for k in autotune.CANDIDATES})
    del gp
    for st in sts:
        st.close()
    return out


def fod2fixel_row():
    """fod2fixel's FMLS segmentation (csd_fmls_segment) of 65,536 synthetic
    FODs at lmax 8, default thresholds; parity and the CPU baseline from the
    C restatement (oracle/fmls_oracle.c) on samples."""
    import torch

    from mrtrix3_b200 import fmls, sh
    from oracle import fmls_ref
    rng = np.random.default_rng(17)
    n, lmax = 65536, 8
    k = rng.integers(1, 4, n)
    c = np.zeros((n, sh.n_for_l(lmax)))
    for j in range(3):
        azel = np.stack([rng.uniform(-np.pi, np.pi, n), np.arccos(rng.uniform(-1, 1, n))], 1)
        c += ((j < k) * rng.uniform(0.3, 1.0, n))[:, None] * sh.init_transform(azel, lmax)
    c = c / c[:, :1] * rng.uniform(0.1, 0.5, (n, 1)) + rng.normal(0.0, 0.01, c.shape)
    c[:, 0] = np.abs(c[:, 0])
    rows = c.astype(np.float32)
    seg = fmls.Segmenter(lmax)
    d = torch.from_numpy(rows).cuda()
    counts, fx = seg.segment(d, max_fixels=16)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    reps = 2
    for _ in range(reps):
        seg.segment(d, max_fixels=16)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    counts, fx = counts.cpu().numpy(), fx.cpu().numpy()
    ref = fmls_ref.Segmenter(lmax)
    cores = os.cpu_count() or 1
    # parity: the C restatement on the first 4096 voxels
    sample = 4096
    rc, rf = fmls_ref.segment_batch_c(ref, rows[:sample].astype(np.float64), max_out=16, nthreads=cores)
    same = np.minimum(rc, 16) == counts[:sample]
    maxd = float(np.abs(fx[:sample][same] - rf[same]).max()) if same.any() else None
    # CPU baseline: the same restatement on all host cores, a bounded sample
    m = min(n, 1500 * cores)
    t0 = time.perf_counter()
    fmls_ref.segment_batch_c(ref, rows[:m].astype(np.float64), max_out=16, nthreads=cores)
    cpu_s = time.perf_counter() - t0
    return {"workload": f"{n} synthetic FODs (lmax 8, 1-3 fibres + N(0, 0.01) on each coefficient), 1281 "
                        "directions, default thresholds, at most 16 fixels a voxel",
            "value": n / (ms / 1e3), "unit": "voxels/s", "ms": ms, "dtype": "f64",
            "fixels_per_voxel": float(np.minimum(counts, 16).mean()),
            "parity": {"vs": "oracle/fmls_oracle.c (FP64)", "sample_voxels": sample,
                       "counts_equal": float(same.mean()), "max_abs_diff": maxd},
            "cpu_baseline": {"value": m / cpu_s, "unit": "voxels/s", "cores": cores, "kind": "port",
                             "sample": f"the first {m} voxels through oracle/fmls_oracle.c (FP64, the reference's "
                                       f"vector of lobes), {cores} threads, {cpu_s:.1f} s"}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-next-rows", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the other workloads (configs 1-4)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    from mrtrix3_b200 import autotune, csd, synth
    from mrtrix3_b200.warmstart import WarmStartNet, train_warm_start
    from oracle import oracle as O

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    vol = make_workload(seed=5 + rank)
    sh = csd.make_shared(vol.grad, synth.RESPONSE)
    d = torch.from_numpy(vol.dwi).to(dev)
    m = torch.from_numpy(vol.mask).to(dev)
    stream = torch.cuda.current_stream()
    if os.path.exists(WEIGHTS):
        net = WarmStartNet.load(WEIGHTS)
        net_src = "mrtrix3_b200/data/warmstart_c5.npz (trained by python -m mrtrix3_b200.train_warmstart)"
    else:
        net, _ = train_warm_start(vol.grad, n_train=2_000_000, epochs=60, lr=4e-3, seed=11)
        net_src = "trained in this run (2M voxels, 60 epochs)"
    st = csd.State(sh, vol.n_voxels)

    def warm_step():
        st.run(d, mask=m, warm=net.predict(d, mask=m, stream=stream), stream=stream)
        return st

    def plain_step():
        st.run(d, mask=m, stream=stream)
        return st

    def persistent_step(warm):
        w = net.predict(d, mask=m, stream=stream) if warm else None
        return csd.dwi2fod_csd(sh, d, mask=m, warm=w, stream=stream)

    def timed(fn, steps):
        for _ in range(max(3, args.warmup)):
            fn()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps)

    # ---- headline: warm-started method, inputs resident in HBM -----------
    for _ in range(max(3, args.warmup)):
        warm_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            warm_step()
        e1.record(stream)
        barrier()
    ms_warm = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    wstats = st.stats()
    # the inference alone (the rest of the step is in the state's counters)
    barrier()
    e0.record(stream)
    for _ in range(3):
        net.predict(d, mask=m, stream=stream)
    e1.record(stream)
    barrier()
    ms_infer = e0.elapsed_time(e1) / 3
    # the FP64 final residual check of the last step's voxels (csd_state_check), timed on its own
    barrier()
    e0.record(stream)
    checked, resolved = st.check(1e-6, stream=stream)
    e1.record(stream)
    barrier()
    fp64_check = {"ms": float(f"{e0.elapsed_time(e1):.4g}"), "checked": checked, "resolved": resolved,
                  "tol": "max|b - W_S F| <= 1e-6 max|b| in FP64, else FP64 re-solve"}
    warm_out = st.fod()
    value = vol.n_masked * world / (ms_warm / 1e3)

    # ---- the other methods (same timing rules) -----------------------------
    ms_plain = timed(plain_step, args.steps)
    pstats = st.stats()
    plain_out = st.fod()
    # ablation: the network's first sets without the factor reuse of the later solves
    autotune.set_knob(autotune.KNOB_REUSE, 2)
    try:
        ms_warm_noreuse = timed(warm_step, args.steps)
        nstats = st.stats()
    finally:
        autotune.set_knob(autotune.KNOB_REUSE, 0)
    # ablation: both methods with the rank-k assembly inside the solve kernel
    # (mma.sync) instead of on tcgen05 ahead of it
    autotune.set_knob(autotune.KNOB_ASSEMBLY, 1)
    try:
        ms_warm_mma = timed(warm_step, args.steps)
        ms_plain_mma = timed(plain_step, args.steps)
    finally:
        autotune.set_knob(autotune.KNOB_ASSEMBLY, 0)
    ms_pers_plain = timed(lambda: persistent_step(False), max(2, args.steps // 2))
    ms_pers_warm = timed(lambda: persistent_step(True), max(2, args.steps // 2))

    def rate(ms):
        return vol.n_masked * world / (ms / 1e3)

    def r4(x):
        return float(f"{x:.4g}")

    methods = {
        "warm_vs_plain": r4(ms_plain / ms_warm),
        "warm_phase_ms": {"set": r4(wstats["ms_set"]), "infer": r4(ms_infer), "project": r4(wstats["ms_project"]),
                          "solve_full": r4(wstats["ms_solve"] - wstats["ms_reuse"]), "solve_reuse": r4(wstats["ms_reuse"])},
        "plain_phase_ms": {"set": r4(pstats["ms_set"]), "project": r4(pstats["ms_project"]),
                           "solve_full": r4(pstats["ms_solve"])},
        "warm_phased": {"voxels_per_s": r4(value), "ms": r4(ms_warm), "passes": wstats["passes"],
                        "solves_per_voxel": r4(wstats["solved"] / vol.n_masked),
                        "reuse_solves_per_voxel": r4(wstats["reuse_solved"] / vol.n_masked),
                        "mean_changed_dirs": r4(wstats["reuse_sum_changes"] / max(1.0, wstats["reuse_solved"]))},
        "warm_phased_no_reuse": {"voxels_per_s": r4(rate(ms_warm_noreuse)), "ms": r4(ms_warm_noreuse),
                                 "solves_per_voxel": r4(nstats["solved"] / vol.n_masked)},
        "plain_phased": {"voxels_per_s": r4(rate(ms_plain)), "ms": r4(ms_plain), "passes": pstats["passes"],
                         "solves_per_voxel": r4(pstats["solved"] / vol.n_masked)},
        "mma_sync_assembly": {"warm_ms": r4(ms_warm_mma), "plain_ms": r4(ms_plain_mma),
                              "warm_vs_plain": r4(ms_plain_mma / ms_warm_mma)},
        "fp64_check": fp64_check,
        "persistent_plain_ms": r4(ms_pers_plain),
        "persistent_warm_ms": r4(ms_pers_warm),
    }

    # ---- parity of the warm and plain outputs on a sample ------------------
    inside = np.nonzero(vol.mask)[0]
    idx = np.random.default_rng(1).choice(inside, 4000, replace=False)
    ref = O.OracleShared(vol.grad, synth.RESPONSE, synth.load_hr_dirs()).solve(vol.dwi[idx])
    parity = {"vs": "FP64 oracle (oracle/csd_oracle.c)", "sample_voxels": len(idx)}
    for name, out in (("warm", warm_out), ("plain", plain_out)):
        r = rel_errors(out["fod"][idx], ref["F"])
        parity[name] = {"p99_rel_err": float(f"{np.percentile(r, 99):.3g}"), "max_rel_err": float(f"{r.max():.3g}"),
                        "negset_match": float(np.mean(np.all(out["negmask"][idx].view(np.uint32) == ref["negmask"],
                                                             axis=1)))}

    # ---- roofline of the solve kernels --------------------------------------
    # Per kernel, algorithmic flops and DRAM bytes per unit of work (n = 45,
    # k = |negative set|, r = changed directions, WSZ = 1104 packed floats):
    #   csd_assemble_tc_kernel<45>  (rank-k assembly on tcgen05) per system:
    #     k n(n+1) flops; the set words in (40 B) and W out (4 WSZ = 4416 B).
    #     It issues 2 x 2 x 320 x 1120 dense FP16 flops (0/1 mask x hi and lo
    #     product tables, padded), reported beside.
    #   csd_solve_kernel<45>  (factorisation + substitutions of assembled W)
    #     per solve: n^3/3 + 2n^2 flops; W in (4416 B), b in (360 B), F out
    #     (180 B), sets (80 B); a warm-started voxel's first solve also stores
    #     its factor (4800 B).
    #   csd_solve_reuse_kernel<45>  (stored factor + Woodbury correction) per
    #     solve: r n(n-1) + r(r+1) n + 4 r n + n^2 + r^3 flops; the factor in
    #     (4800 B), sets in (80 B), F out (180 B), sets out (80 B).
    # Each against its own device time (CUDA events of the state's passes); the
    # binding roof of a kernel is the one it comes closer to: measured HBM
    # bandwidth for the bytes, the measured dense bf16 tensor peak for flops.
    n, wsz = 45, 1104
    peaks, peak_kind = load_peaks()
    full_solves = wstats["solved"] - wstats["reuse_solved"]
    full_ms = wstats["ms_solve"] - wstats["ms_reuse"]
    asm_ms = wstats["ms_asm"]
    rr = wstats["reuse_sum_changes"] / max(1.0, wstats["reuse_solved"])
    kernels = {
        "csd_solve_kernel<45>": {
            "ms_per_step": full_ms - asm_ms, "solves": full_solves,
            "flops": full_solves * (n ** 3 / 3.0 + 2 * n * n) + (0 if asm_ms > 0 else wstats["sum_neg"] * n * (n + 1)),
            "bytes": full_solves * ((4 * wsz if asm_ms > 0 else 0) + 360 + 180 + 80) + vol.n_masked * 4800},
        "csd_solve_reuse_kernel<45>": {
            "ms_per_step": wstats["ms_reuse"], "solves": wstats["reuse_solved"],
            "flops": wstats["reuse_solved"] * (rr * n * (n - 1) + rr * (rr + 1) * n + 4 * rr * n + n * n + rr ** 3),
            "bytes": wstats["reuse_solved"] * (4800 + 80 + 180 + 80)},
    }
    if asm_ms > 0:
        kernels["csd_assemble_tc_kernel<45>"] = {
            "ms_per_step": asm_ms, "solves": full_solves, "flops": wstats["sum_neg"] * n * (n + 1),
            "bytes": full_solves * (40 + 4 * wsz), "issued_tensor_flops": full_solves * 2 * 2 * 320 * 1120}
    for v in kernels.values():
        sec = max(1e-12, v["ms_per_step"] / 1e3)
        v["tflops"] = v["flops"] / sec / 1e12
        v["gbs"] = v["bytes"] / sec / 1e9
        v["frac_tensor"] = v["tflops"] / peaks["bf16_tflops"]
        v["frac_hbm"] = v["gbs"] / peaks["hbm_gbs"]
        v["bound"] = "hbm" if v["frac_hbm"] >= v["frac_tensor"] else "tensor"
    solve_launches = max(1.0, wstats["passes"])
    dom = max(kernels, key=lambda k: kernels[k]["ms_per_step"])
    kd = kernels[dom]
    per_solve = {"csd_solve_kernel<45>": SOLVE_DRAM_BYTES_PER_VOXEL,
                 "csd_solve_reuse_kernel<45>": REUSE_DRAM_BYTES_PER_VOXEL,
                 "csd_assemble_tc_kernel<45>": ASM_DRAM_BYTES_PER_SYSTEM}.get(dom)
    traffic = per_solve * kd["solves"] / solve_launches if per_solve is not None else None
    if kd["bound"] == "hbm":
        achieved, peak, unit = kd["gbs"], peaks["hbm_gbs"], "GB/s"
        alg = {"algorithmic_bytes_per_launch": kd["bytes"] / solve_launches}
        peak_source = f"HBM copy bandwidth ({peak_kind})"
    else:
        achieved, peak, unit = kd["tflops"], peaks["bf16_tflops"], "TFLOP/s"
        alg = {"algorithmic_flops_per_launch": kd["flops"] / solve_launches}
        peak_source = f"dense bf16 tensor peak, burst ({peak_kind})"
    roofline = {"bound": kd["bound"], "achieved": achieved, "peak": peak, "unit": unit, "frac": achieved / peak,
                "traffic": traffic, "kernel": dom, "peak_source": peak_source, **alg,
                "avg_launch_ms": kd["ms_per_step"] / solve_launches,
                "kernel_share_of_step": kd["ms_per_step"] / ms_warm,
                # context: the factorisations and substitutions run on the FP32 SIMT pipes
                # (148 SMs x 128 FMA lanes x 2 flops x 1.965 GHz, nominal, not measured)
                "fp32_simt_nominal_tflops": FP32_SIMT_NOMINAL_TFLOPS,
                "kernels": {k: {"ms_per_step": r4(v["ms_per_step"]), "solves": int(v["solves"]),
                                "bound": v["bound"], "tflops": r4(v["tflops"]), "gbs": r4(v["gbs"]),
                                "frac_hbm": r4(v["frac_hbm"]), "frac_tensor": r4(v["frac_tensor"]),
                                "frac_of_fp32_simt_nominal": r4(v["tflops"] / FP32_SIMT_NOMINAL_TFLOPS),
                                **({"issued_tensor_tflops": r4(v["issued_tensor_flops"]
                                                               / max(1e-9, v["ms_per_step"] / 1e3) / 1e12),
                                    "issued_frac_of_tensor_peak": r4(v["issued_tensor_flops"]
                                                                     / max(1e-9, v["ms_per_step"] / 1e3) / 1e12
                                                                     / peaks["bf16_tflops"])}
                                   if "issued_tensor_flops" in v else {})}
                            for k, v in kernels.items()}}

    # ---- end to end through the host-buffer C ABI (pinned buffers) ---------
    pinned = torch.from_numpy(vol.dwi).pin_memory()
    pmask = torch.from_numpy(vol.mask).pin_memory()
    pfod = torch.empty((vol.n_voxels, 45), dtype=torch.float32).pin_memory()
    csd.dwi2fod_csd_host_phased(sh, pinned, pmask, net=net, fod=pfod)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        csd.dwi2fod_csd_host_phased(sh, pinned, pmask, net=net, fod=pfod)
    barrier()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    e2e = {"value": vol.n_masked * world / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(vol.dwi.nbytes + vol.mask.nbytes),
           "d2h_bytes_per_step": int(vol.n_voxels * (45 * 4 + 2)),
           "api": "csd_dwi2fod_host_phased (warm start, pinned host buffers, copies inside the timed region)"}

    mlp_launches = 2  # masked-voxel compaction + the fused inference kernel (weights already packed)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_warm, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp32 (tensor-core projection/assembly on fp16 hi+lo splits, fp64 fallback/refinement)",
            "data": "synthetic",
            "config": workload_config(vol),
            "method": "warm-started phased CSD (network first sets + plain iteration)",
            "roofline": roofline, "e2e": e2e,
            "gpu_launches": int(wstats["launches"] + mlp_launches) * args.steps,
            "clocks": clk.summary(), "warm_start_net": net_src}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(vol)
    if rank == 0 and world == 1 and not args.no_next_rows:
        line["next_rows"] = next_rows(d, np.nonzero(vol.mask)[0][:2000])
    if rank == 0 and world == 1 and not args.no_configs:
        try:
            line["configs"] = config_rows(net)
        except Exception as ex:  # the headline line is printed whatever happens here
            line["configs"] = {"error": f"{type(ex).__name__}: {ex}"}
    # the metric's own figures last: a reader of the line's tail sees them
    line["precision"] = PRECISION
    line["methods"] = methods
    line["parity"] = parity
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
