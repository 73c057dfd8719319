"""Run one CSD method on a synthetic case, for profilers (ncu) and timing.

    python -m mrtrix3_b200.profile_case [--dims 64 64 64] [--lmax 8]
        [--method warm|plain|persistent|persistent_warm|predict|peaks|fod2fixel|amp2sh|msmt|tensor|amp2response]
        [--reps 2]
        [--projection mma|tcgen05] [--solve warp|group16|group8] [--amp2sh-kernel auto|row|tile|mma]
        [--passes N]

Every voxel is inside the volume (no mask); the scheme is 6 b=0 + 60 DW
(lmax 8) or 8 b=0 + 90 DW (lmax 10).  Prints the state's work / time
counters of the last repetition.
"""
import argparse
import os
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs=3, default=[64, 64, 64])
    ap.add_argument("--lmax", type=int, default=8)
    ap.add_argument("--method", default="warm", choices=["warm", "plain", "persistent", "persistent_warm", "predict", "peaks",
                                                          "fod2fixel", "amp2sh", "msmt", "tensor", "amp2response"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--projection", default="tcgen05", choices=["mma", "tcgen05"])
    ap.add_argument("--solve", default="warp", choices=["warp", "group16", "group8"])
    ap.add_argument("--amp2sh-kernel", default="auto", choices=["auto", "row", "tile", "mma"])
    ap.add_argument("--passes", type=int, default=0,
                    help="warm / plain: stop the phased run after this many passes (0: run to the end), so "
                         "that the state's counters describe exactly the launches a profiler captured")
    a = ap.parse_args()
    import torch

    from . import autotune, csd, synth
    autotune.set_knob(autotune.KNOB_TC_PROJECTION, 2 if a.projection == "tcgen05" else 1)
    autotune.set_knob(autotune.KNOB_SOLVE_KIND, {"warp": 1, "group16": 2, "group8": 3}[a.solve])
    autotune.set_knob(autotune.KNOB_AMP2SH_KIND, ["auto", "row", "tile", "mma"].index(a.amp2sh_kernel))
    if a.method in ("tensor", "amp2response"):
        # the tensor fit (FA, principal vector) of a 4-shell volume, then the
        # amp2response accumulation over every voxel of its largest shell
        from . import amp2response as AR
        from . import msmt
        from .tensor import dwi2tensor
        grad = synth.msmt_scheme()
        n = int(np.prod(a.dims))
        rng = np.random.default_rng(3)
        clean = 1000.0 * np.exp(-grad[:, 3] * 0.8e-3)[None, :].repeat(n, axis=0)
        dwi = torch.from_numpy(synth.rician(rng, clean, 20.0)).float().cuda()  # isotropic, SNR 50 at b=0
        g = msmt.normalise_scheme(grad)
        vols = msmt.cluster_shells(g[:, 3])[-1]
        da = msmt.direction_matrix(g, vols)
        cart = np.stack([np.cos(da[:, 0]) * np.sin(da[:, 1]), np.sin(da[:, 0]) * np.sin(da[:, 1]), np.cos(da[:, 1])], 1)
        _, _, _, vec = dwi2tensor(dwi, grad)
        vec = vec + torch.tensor([0.0, 0.0, 1.0], device=vec.device)  # a direction everywhere
        run = (lambda: dwi2tensor(dwi, grad)) if a.method == "tensor" else \
            (lambda: AR.accumulate(dwi, vec, cart, vols, 10))
        run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.reps):
            run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
        print(f"{a.method}: {n} voxels x {grad.shape[0]} volumes in {ms:.3f} ms per call "
              f"({n / ms / 1e3:.1f}M voxels/s)")
        return
    if a.method == "msmt":  # 3-tissue MSMT-CSD on a 4-shell scheme (6 b=0 + 30/45/60 DW)
        from . import msmt
        s = msmt.MSMTShared(synth.msmt_scheme())
        s.set_responses([synth.MSMT_RESPONSES[k] for k in ("wm", "gm", "csf")])
        s.init()
        rng = np.random.default_rng(5)
        n = int(np.prod(a.dims))
        clean = synth.msmt_truth(rng, n) @ s.C.T
        dwi = synth.rician(rng, clean, rng.uniform(1000.0 / 40, 1000.0 / 15, n)).astype(np.float32)
        d = torch.from_numpy(dwi).cuda()
        x, it = s.solve(d)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.reps):
            s.solve(d, out=x, niter=it)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
        itn = it.cpu().numpy()
        print(f"msmt: {n} voxels in {ms:.3f} ms per call ({n / ms / 1e3:.2f}M voxels/s), solver rounds mean "
              f"{itn.mean():.2f} max {itn.max()}")
        return
    from .warmstart import WarmStartNet
    ndw, nb0 = (60, 6) if a.lmax <= 8 else (90, 8)
    v = synth.make_volume(tuple(a.dims), nb0, ndw, (15.0, 40.0), a.lmax, None, 5)
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=a.lmax)
    d = torch.from_numpy(v.dwi).cuda()
    net = None
    if a.method in ("warm", "persistent_warm", "predict"):
        net = WarmStartNet.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_c5.npz"))
    st = csd.State(s, d.shape[0]) if a.method in ("warm", "plain", "peaks", "fod2fixel") else None
    fod = None
    if a.method == "amp2sh":  # the SH fit of this volume's DW amplitudes (normalised by its b=0 volumes)
        from . import sh
        dwis = np.asarray(s.dwis)
        bzeros = np.nonzero(v.grad[:, 3] <= 10.0)[0]
        fit = sh.pinv(sh.init_transform(sh.cartesian_to_azel(v.grad[dwis, :3]), a.lmax))
        plan = csd.Amp2SHCommon(fit, dwis, bzeros, normalise=True)
        out = plan(d)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.reps):
            plan(d, out)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
        nbytes = d.shape[0] * (len(dwis) + len(bzeros) + fit.shape[0]) * 4
        print(f"amp2sh: {d.shape[0]} voxels in {ms:.3f} ms per call, {nbytes / ms / 1e6:.0f} GB/s "
              f"({d.shape[0] / ms / 1e3:.1f}M voxels/s)")
        return
    if a.method in ("peaks", "fod2fixel"):  # sh2peaks / FMLS segmentation of this volume's FODs
        st.run(d)
        fod = st.fod(as_numpy=False)["fod"]
    if a.method == "fod2fixel":
        from . import fmls
        seg = fmls.Segmenter(a.lmax)
        counts, _ = seg.segment(fod, max_fixels=16)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.reps):
            seg.segment(fod, max_fixels=16)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
        print(f"fod2fixel: {fod.shape[0]} voxels in {ms:.3f} ms per call ({fod.shape[0] / ms / 1e3:.3f}M voxels/s), "
              f"{counts.float().mean().item():.2f} fixels a voxel")
        return
    t0 = time.perf_counter()
    for _ in range(a.reps):
        if a.method == "predict":
            net.predict(d)
        elif a.method == "peaks":
            csd.sh2peaks(fod)
        elif st is not None and a.passes > 0:
            w = net.predict(d) if net is not None else None
            st.set(d)
            if w is not None:
                st.warm(w)
            st.iterate_all(max_passes=a.passes)
        elif st is not None:
            st.run(d, warm=net.predict(d) if net is not None else None)
        else:
            csd.dwi2fod_csd(s, d, warm=net.predict(d) if net is not None else None)
    torch.cuda.synchronize()
    print(f"{a.method}: {d.shape[0]} voxels x {a.reps} reps in {time.perf_counter() - t0:.3f} s")
    if st is not None:
        print(st.stats())


if __name__ == "__main__":
    main()
