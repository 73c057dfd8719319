"""``dwi2fod csd`` / ``dwi2fod msmt_csd`` on MRtrix image files, computed by
the B200 library.

    python -m mrtrix3_b200.dwi2fod csd <dwi> <response.txt> <fod_out> [options]
    python -m mrtrix3_b200.dwi2fod msmt_csd <dwi> <resp1.txt> <out1> [<resp2.txt> <out2> ...] [options]

Mirrors cmd/dwi2fod.cpp:236-276 for the csd algorithm: the DW image (4-D,
any MRtrix datatype, .mif / .mif.gz / .mih) with its embedded ``dw_scheme``
(or ``-grad``), the single-shell response (one row or column of even
zonal SH coefficients), an optional 3-D mask; the output is a float32 FOD
image whose SH axis is contiguous on file, the spatial axes keeping the
input's order, with the gradient table moved to ``prior_dw_scheme`` and
the phase-encoding keys removed (dwi2fod.cpp:240-243, 270-271).

Options (csd.cpp:318-346, dwi2fod.cpp:38-59, gradient.cpp:36-60):
  -mask image        only voxels inside the mask are processed
  -lmax N            maximum harmonic order of the output
  -directions file   constraint directions, [az el] pairs in radians
  -filter file       initial linear filter, one value per even order
  -neg_lambda v      weight of the non-negativity constraint (1)
  -norm_lambda v     weight of the norm regulariser (1)
  -threshold v       amplitude below which a direction is constrained (0)
  -niter N           maximum iterate() calls per voxel (50)
  -shells b         the non-b=0 shell to deconvolve (one b-value; default the
                     largest shell; shells.cpp:100-239)
  -grad file         gradient table [x y z b] rows, instead of dw_scheme
  -fslgrad bvecs bvals   FSL gradient files (image-axis directions)
  -warm_start file   a warm-start network (.npz) trained for this scheme
                     (no counterpart in MRtrix3; off by default)
  -force             overwrite the output
  -nthreads N, -quiet, -info   accepted and ignored

msmt_csd (dwi2fod.cpp:283-326, msmt_csd.cpp:24-48): one response file per
tissue ([shells][even zonal coefficients]) and one output per tissue, every
b-value shell used (or those -shells b1,b2,.. selects); -lmax takes one
value per tissue; -norm_lambda /
-neg_lambda default 1e-10; -predicted_signal image writes the modelled DW
signal (float32, the input's layout); -mask, -directions, -grad as above.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import mif

_VALUED = {"-mask", "-lmax", "-directions", "-filter", "-neg_lambda", "-norm_lambda", "-threshold", "-niter",
           "-grad", "-warm_start", "-nthreads", "-predicted_signal", "-shells"}
_FLAGS = {"-force", "-quiet", "-info"}


def _parse(argv):
    pos, opt = [], {}
    i = 0
    while i < len(argv):
        a = argv[i]
        if a.startswith("-") and len(a) > 1 and not _is_number(a):
            key = "-" + a.lstrip("-")
            if key == "-fslgrad":
                if i + 2 >= len(argv):
                    raise SystemExit("dwi2fod: option \"-fslgrad\" expects two values (bvecs bvals)")
                opt[key] = (argv[i + 1], argv[i + 2])
                i += 3
                continue
            if key in _VALUED:
                if i + 1 >= len(argv):
                    raise SystemExit(f"dwi2fod: option \"{a}\" expects a value")
                opt[key] = argv[i + 1]
                i += 2
                continue
            if key in _FLAGS:
                opt[key] = True
                i += 1
                continue
            raise SystemExit(f"dwi2fod: unknown option \"{a}\"")
        pos.append(a)
        i += 1
    return pos, opt


def _is_number(s):
    try:
        float(s)
        return True
    except ValueError:
        return False


def output_layout(in_layout, ndim_in: int):
    """Stride::contiguous_along_axis(3, header_in): axis 3 fastest, the
    spatial axes after it in the input's order and directions."""
    lay = list(in_layout) if in_layout else list(range(1, ndim_in + 1))
    spatial = sorted(range(3), key=lambda a: abs(lay[a]))
    out = [0, 0, 0, 1]
    for rank, a in enumerate(spatial):
        out[a] = (rank + 2) * (1 if lay[a] > 0 else -1)
    return out


def run(argv) -> int:
    pos, opt = _parse(argv)
    if len(pos) < 1 or pos[0] not in ("csd", "msmt_csd"):
        raise SystemExit("usage: python -m mrtrix3_b200.dwi2fod csd <dwi> <response> <fod_out> [options]")
    if pos[0] == "msmt_csd":
        return run_msmt(pos, opt)
    if len(pos) != 4:
        raise SystemExit("CSD algorithm expects a single input response function and single output FOD image")
    _, dwi_path, resp_path, out_path = pos
    if os.path.exists(out_path) and not opt.get("-force"):
        raise SystemExit(f"dwi2fod: output image \"{out_path}\" already exists (use -force to replace it)")

    from . import csd
    img = mif.read(dwi_path)
    if img.data.ndim != 4:
        raise SystemExit(f"dwi2fod: input image \"{dwi_path}\" is not 4-D")
    try:
        grad = mif.dw_scheme(img, opt)
    except ValueError as e:
        raise SystemExit(f"dwi2fod: {e} (\"{dwi_path}\")")
    nx, ny, nz, nvol = img.data.shape
    if grad.shape != (nvol, 4):
        raise SystemExit(f"dwi2fod: number of volumes in the gradient table ({grad.shape[0]}) does not match the "
                         f"image ({nvol})")
    mask = None
    if "-mask" in opt:
        m = mif.read(opt["-mask"])
        if m.data.shape[:3] != (nx, ny, nz):
            raise SystemExit("dwi2fod: the mask's dimensions do not match the DW image")
        mask = np.ascontiguousarray((m.data.reshape(nx, ny, nz) != 0).reshape(-1).astype(np.uint8))

    shared = csd.Shared(grad)
    kw = {}
    if "-lmax" in opt:
        kw["lmax"] = [int(v) for v in opt["-lmax"].split(",")]
    if "-directions" in opt:
        kw["directions"] = mif.load_matrix(opt["-directions"])
    if "-filter" in opt:
        kw["filter"] = mif.load_vector(opt["-filter"])
    for name in ("neg_lambda", "norm_lambda", "threshold"):
        if "-" + name in opt:
            kw[name] = float(opt["-" + name])
    if "-niter" in opt:
        kw["niter"] = int(opt["-niter"])
    if "-shells" in opt:
        kw["shells"] = [float(v) for v in opt["-shells"].split(",")]
    shared.parse_cmdline_options(**kw)
    shared.set_response(mif.load_vector(resp_path))
    try:
        shared.init()
    except csd.CSDError as e:
        raise SystemExit(f"dwi2fod: {e}")

    net = None
    if "-warm_start" in opt:
        from .warmstart import WarmStartNet
        net = WarmStartNet.load(opt["-warm_start"])
        if net.n_in != nvol:
            raise SystemExit("dwi2fod: the warm-start network was trained for a different number of volumes")

    dwi = np.ascontiguousarray(img.data.reshape(-1, nvol), np.float32)  # voxel-interleaved
    out = csd.dwi2fod_csd_host_phased(shared, dwi, mask, net=net)
    nsh = shared.nSH()
    fod = out["fod"].reshape(nx, ny, nz, nsh)

    kv = {k: v for k, v in img.keyval.items()
          if k not in ("dw_scheme", "prior_dw_scheme", "pe_scheme", "PhaseEncodingDirection", "TotalReadoutTime")}
    kv["prior_dw_scheme"] = mif.scheme_to_text(grad)
    vox = list(img.vox) + [float("nan")] * (4 - len(img.vox))
    out_img = mif.Image(data=fod, vox=vox[:4], transform=img.transform, keyval=kv)
    mif.write(out_path, out_img, layout=output_layout(img.layout, 4),
              datatype="Float32LE" if np.little_endian else "Float32BE")
    st = out["status"]
    n_niter = int(np.sum((st & 0x0F) == csd.STATUS_NITER))
    if n_niter and not opt.get("-quiet"):
        print(f"dwi2fod: {n_niter} voxels did not reach full convergence", file=sys.stderr)
    return 0


def _load_dwi(dwi_path, opt):
    img = mif.read(dwi_path)
    if img.data.ndim != 4:
        raise SystemExit(f"dwi2fod: input image \"{dwi_path}\" is not 4-D")
    try:
        grad = mif.dw_scheme(img, opt)
    except ValueError as e:
        raise SystemExit(f"dwi2fod: {e} (\"{dwi_path}\")")
    nvol = img.data.shape[3]
    if grad.shape != (nvol, 4):
        raise SystemExit(f"dwi2fod: number of volumes in the gradient table ({grad.shape[0]}) does not match the "
                         f"image ({nvol})")
    mask = None
    if "-mask" in opt:
        m = mif.read(opt["-mask"])
        if m.data.shape[:3] != img.data.shape[:3]:
            raise SystemExit("dwi2fod: the mask's dimensions do not match the DW image")
        mask = np.ascontiguousarray((m.data.reshape(img.data.shape[:3]) != 0).reshape(-1).astype(np.uint8))
    return img, grad, mask


def run_msmt(pos, opt) -> int:
    """dwi2fod.cpp:283-326 (the msmt_csd branch) with MSMT_Processor (:178-218)."""
    if len(pos) % 2:
        raise SystemExit("MSMT_CSD algorithm expects pairs of (input response function & output FOD image) to be "
                         "provided")
    pairs = [(pos[i], pos[i + 1]) for i in range(2, len(pos), 2)]
    outs = [o for _, o in pairs] + ([opt["-predicted_signal"]] if "-predicted_signal" in opt else [])
    for o in outs:
        if os.path.exists(o) and not opt.get("-force"):
            raise SystemExit(f"dwi2fod: output image \"{o}\" already exists (use -force to replace it)")
    from . import msmt
    img, grad, mask = _load_dwi(pos[1], opt)
    try:
        shared = msmt.MSMTShared(grad, shells=[float(v) for v in opt["-shells"].split(",")] if "-shells" in opt
                                 else None)
    except ValueError as e:
        raise SystemExit(f"dwi2fod: {e}")
    kw = {}
    if "-lmax" in opt:
        kw["lmax"] = [int(v) for v in opt["-lmax"].split(",")]
    if "-directions" in opt:
        kw["directions"] = mif.load_matrix(opt["-directions"])
    for name in ("norm_lambda", "neg_lambda"):
        if "-" + name in opt:
            kw[name] = float(opt["-" + name])
    shared.parse_cmdline_options(**kw)
    try:
        shared.set_responses([r for r, _ in pairs])
    except Exception as e:
        raise SystemExit(f"MSMT_CSD algorithm expects the first file in each argument pair to be an input response "
                         f"function file ({e})")
    try:
        shared.init()
    except ValueError as e:
        raise SystemExit(f"dwi2fod: {e}")

    import torch
    nx, ny, nz, nvol = img.data.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    dwi = torch.from_numpy(np.ascontiguousarray(img.data.reshape(-1, nvol), np.float32)).to(dev)
    m = torch.from_numpy(mask).to(dev) if mask is not None else None
    pred = torch.empty((dwi.shape[0], nvol), dtype=torch.float32, device=dev) if "-predicted_signal" in opt else None
    x, it = shared.solve(dwi, mask=m, predicted=pred)
    x = x.cpu().numpy()
    it = it.cpu().numpy()

    kv = {k: v for k, v in img.keyval.items() if k not in ("dw_scheme", "prior_dw_scheme")}
    kv["prior_dw_scheme"] = mif.scheme_to_text(shared.grad)
    vox = list(img.vox) + [float("nan")] * (4 - len(img.vox))
    dt = "Float32LE" if np.little_endian else "Float32BE"
    for (_, path), part in zip(pairs, shared.split(x)):
        out_img = mif.Image(data=part.reshape(nx, ny, nz, -1), vox=vox[:4], transform=img.transform, keyval=kv)
        mif.write(path, out_img, layout=output_layout(img.layout, 4), datatype=dt)
    if pred is not None:
        p_img = mif.Image(data=pred.cpu().numpy().reshape(nx, ny, nz, nvol), vox=img.vox, transform=img.transform,
                          keyval=dict(img.keyval))
        mif.write(opt["-predicted_signal"], p_img, layout=img.layout, datatype=dt)
    n_niter = int(np.sum(it >= shared.max_niter()))
    if n_niter and not opt.get("-quiet"):
        print(f"dwi2fod: {n_niter} voxels did not reach full convergence", file=sys.stderr)
    return 0


def main():
    sys.exit(run(sys.argv[1:]))


if __name__ == "__main__":
    main()
