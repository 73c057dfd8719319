"""``dwi2response fa | manual | tournier | tax`` on the GPU: a single-fibre
response function from a DW image (lib/mrtrix3/dwi2response/fa.py,
manual.py, tournier.py, tax.py), from the library's tensor fit
(csd_dwi2tensor), CSD (csd_solve), FMLS segmentation (csd_fmls_segment) and
amp2response (csd_amp2response_accumulate + the ICLS solver).

    python -m mrtrix3_b200.dwi2response fa <dwi> <response.txt> -mask <mask> [options]
    python -m mrtrix3_b200.dwi2response manual <dwi> <in_voxels> <response.txt> [options]
    python -m mrtrix3_b200.dwi2response tournier|tax <dwi> <response.txt> -mask <mask> [options]

fa (fa.py): the tensor fit inside the mask; its FA and FA-modulated principal
eigenvector; the voxels of the ``-number`` (300) highest FA values (all
voxels with FA >= the threshold value mrthreshold -top gives) or FA >=
``-threshold``; the response of the largest non-b=0 shell (dwiextract
-singleshell -no_bzero) at lmax ``-lmax`` (default 10).
manual (manual.py): the given voxels; fibre directions from ``-dirs`` or
from the tensor fit over those voxels; the response of every shell, one row
each (``-lmax`` one per shell; default 0 for b=0, else 10).
tournier (tournier.py:53-150) and tax (tax.py:53-160): on the largest
non-b=0 shell (or the one ``-shells`` names), iterate CSD, FMLS segmentation
without thresholds and the response fit over single-fibre voxels chosen by
the first two lobes' peak amplitudes; options -number, -iter_voxels,
-dilate, -max_iters (tournier), -peak_ratio, -max_iters, -convergence (tax).
Options: -mask (required by fa, tournier and tax: the brain mask the script
would otherwise make with dwi2mask, which is not provided here), -number,
-threshold, -lmax, -dirs, -voxels image, -grad file, -fslgrad bvecs bvals,
-shells, -force.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import amp2response as AR
from . import mif, msmt
from .tensor import dwi2tensor

_VALUED = {"-mask", "-number", "-threshold", "-lmax", "-dirs", "-voxels", "-grad", "-nthreads", "-erode",
           "-iter_voxels", "-dilate", "-max_iters", "-peak_ratio", "-convergence", "-shells"}
_FLAGS = {"-force", "-quiet", "-info"}


def _parse(argv):
    pos, opt = [], {}
    i = 0
    while i < len(argv):
        a = argv[i]
        key = "-" + a.lstrip("-") if a.startswith("-") and len(a) > 1 else None
        if key == "-fslgrad":
            if i + 2 >= len(argv):
                raise SystemExit("dwi2response: option \"-fslgrad\" expects two values (bvecs bvals)")
            opt[key] = (argv[i + 1], argv[i + 2])
            i += 3
            continue
        if key in _VALUED:
            if i + 1 >= len(argv):
                raise SystemExit(f"dwi2response: option \"{a}\" expects a value")
            opt[key] = argv[i + 1]
            i += 2
        elif key in _FLAGS:
            opt[key] = True
            i += 1
        elif key is not None:
            raise SystemExit(f"dwi2response: unknown option \"{a}\"")
        else:
            pos.append(a)
            i += 1
    return pos, opt


def top_threshold(values: np.ndarray, number: int) -> float:
    """mrthreshold -top N (cmd/mrthreshold.cpp:227-245): the value at index
    size - N of the sorted finite values; voxels >= it are selected."""
    data = np.sort(values[np.isfinite(values)])
    idx = len(data) - number
    if idx < 0 or idx >= len(data):
        raise SystemExit(f"Number of valid input image values ({len(data)}) less than number of voxels requested "
                         f"via -top option ({number})")
    return float(data[idx])


def dilate(mask3: np.ndarray, npass: int) -> np.ndarray:
    """maskfilter dilate (core/filter/dilate.h:84-109): npass passes, a voxel
    set when it or one of its 6 face neighbours is set."""
    m = np.asarray(mask3, bool)
    for _ in range(npass):
        o = m.copy()
        for ax in range(3):
            sl_lo = [slice(None)] * 3
            sl_hi = [slice(None)] * 3
            sl_lo[ax] = slice(0, -1)
            sl_hi[ax] = slice(1, None)
            o[tuple(sl_lo)] |= m[tuple(sl_hi)]
            o[tuple(sl_hi)] |= m[tuple(sl_lo)]
        m = o
    return m


def _str6(x: float) -> float:
    """A statistic as mrstats prints it and the scripts read it back
    (MRtrix str(): 6 significant digits)."""
    return float(f"{x:.6g}")


def masked_mean_std(values: np.ndarray, mask: np.ndarray):
    """image.statistics (dwi, mask, allvolumes) (core/stats.h:55-75): mean
    and standard deviation (count - 1) of the finite values of every volume
    inside the mask, as printed."""
    v = np.asarray(values, np.float64)[np.asarray(mask, bool)].reshape(-1)
    v = v[np.isfinite(v)]
    return _str6(float(v.mean())), _str6(float(v.std(ddof=1)))


def tournier_loop(step, fit, mask, dims, number=300, iter_voxels=0, dilate_passes=1, max_iters=10, lmax=None):
    """tournier.py:53-150.  step(rf, voxels) -> (first peak amplitude, second
    peak amplitude, first direction) per voxel row, for CSD with response rf
    and FMLS segmentation without thresholds inside ``voxels``; fit(sf,
    first_dir, lmax) -> response row.  Rows are z-major ([z][y][x] of
    ``dims`` = (nx, ny, nz)).  Returns (response, single-fibre rows, iterations)."""
    if max_iters < 2:
        raise SystemExit("Number of iterations must be at least 2")
    if iter_voxels == 0:
        iter_voxels = 10 * number
    elif iter_voxels < number:
        raise SystemExit("Number of selected voxels (-iter_voxels) must be greater than number of voxels desired "
                         "(-number)")
    nx, ny, nz = dims
    rf = np.array([1.0, -1.0, 1.0])
    mask_in = np.asarray(mask, bool)
    prev_sf = None
    for it in range(max_iters):
        p1, p2, first_dir = step(rf, mask_in)
        p1 = np.asarray(p1, np.float32)
        p2 = np.asarray(p2, np.float32)
        with np.errstate(divide="ignore", invalid="ignore"):
            cf = (np.sqrt(p1.astype(np.float64)) * (1.0 - p2.astype(np.float64) / p1) ** 2).astype(np.float32)
        count = int(np.isfinite(cf).sum())
        sf = cf >= top_threshold(cf, min(number, count))
        rf = fit(sf, first_dir, 4 if it == 0 else lmax)
        if it > 0 and not (sf.astype(np.int8) - prev_sf.astype(np.int8)).max():
            return rf, sf, it + 1
        prev_sf = sf
        top = cf >= top_threshold(cf, min(iter_voxels, count))
        grown = dilate(top.reshape(nz, ny, nx), dilate_passes).reshape(-1)
        mask_in = np.asarray(mask, bool) & grown
    return rf, prev_sf, max_iters


def tax_loop(step, fit, mask, init_rf, peak_ratio=0.1, max_iters=20, convergence=0.5, lmax=None):
    """tax.py:53-160 (step and fit as for tournier_loop; init_rf from the
    masked mean / std of the data).  Returns (response, single-fibre rows,
    iterations)."""
    change = 0.01 * convergence
    rf = np.asarray(init_rf, np.float64)
    mask_in = np.asarray(mask, bool)
    sf = None
    for it in range(max_iters):
        p1, p2, first_dir = step(rf, mask_in)
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = (np.asarray(p2, np.float32) / np.asarray(p1, np.float32)).astype(np.float32)
        sf = (ratio < peak_ratio) & mask_in
        if not sf.any():
            raise SystemExit("Aborting: All voxels have been excluded from single-fibre selection")
        new_rf = fit(sf, first_dir, lmax)
        if it > 0:
            reiterate = False
            for old, new in zip(rf, new_rf):
                old, new = float(old), float(new)  # as the script's floats: a zero mean raises
                mean = 0.5 * (old + new)
                diff = abs(0.5 * (old - new))
                if diff / mean > change:
                    reiterate = True
            if not reiterate:
                return new_rf, sf, it + 1
        rf = new_rf
        mask_in = sf
    return rf, sf, max_iters


def iterative(algo, opt, g, shells, dwi, mask, dims):
    """dwi2response tournier / tax on device rows ``dwi`` [n][volumes] with
    the normalised scheme g: the single shell (dwiextract -singleshell
    -no_bzero, or the one -shells names), then the loop on the GPU steps."""
    import torch

    from . import csd, fmls, sh
    dw = [v for v in shells if float(np.mean(g[v, 3])) > 10.0]
    if not dw:
        raise SystemExit("dwi2response: no non-b=0 shell in the data")
    if "-shells" in opt:
        try:
            keep = msmt.select_shells(g[:, 3], shells, [float(opt["-shells"])])
        except ValueError as e:
            raise SystemExit(f"dwi2response: {e}")
        vols = shells[keep[0]]
        if float(np.mean(g[vols, 3])) <= 10.0:
            raise SystemExit("dwi2response: the shell given by -shells is b=0")
    else:
        vols = dw[-1]
    vols = np.asarray(vols)
    grad = g[vols]
    dw_dev = dwi[:, torch.from_numpy(vols).to(dwi.device)].contiguous()
    dirs = msmt.direction_matrix(grad, np.arange(len(vols)))
    lmax = int(opt["-lmax"]) if "-lmax" in opt else None
    dev = dwi.device

    segmenters = {}  # one per FOD lmax (4 in tournier's first round, then the CSD's lmax)

    def step(rf, voxels):
        s = csd.make_shared(grad, np.asarray(rf, np.float64))
        m = torch.from_numpy(np.asarray(voxels, np.uint8)).to(dev)
        fod = csd.dwi2fod_csd(s, dw_dev, m)["fod"]
        L = sh.l_for_n(s.nSH())
        if L not in segmenters:
            segmenters[L] = fmls.Segmenter(L, 0.0, 0.0, fmls.MERGE_RATIO_DEFAULT)  # -fmls_no_thresholds
        seg = segmenters[L]
        counts, fx = seg.segment(fod, m, max_fixels=2)
        c = counts.cpu().numpy()
        f = fx.cpu().numpy()
        p1 = np.where(c >= 1, f[:, 0, 7], 0.0).astype(np.float32)   # fixel2voxel none, -number 2
        p2 = np.where(c >= 2, f[:, 1, 7], 0.0).astype(np.float32)
        d1 = np.where((c >= 1)[:, None], f[:, 0, 0:3], np.nan).astype(np.float32)  # fixel2peaks -number 1
        return p1, p2, d1

    def fit(sf, first_dir, L):
        L = L if L is not None else 10   # amp2response's default for a shell without b=0
        r = AR.responses(dw_dev, torch.from_numpy(np.nan_to_num(first_dir)).to(dev),
                         torch.from_numpy(np.asarray(sf, np.uint8)).to(dev), [dirs], [np.arange(len(vols))], [L])[0]
        return np.array([float(f"{v:.10g}") for v in r])   # as written to and read back from RF.txt

    if algo == "tournier":
        return tournier_loop(step, fit, mask, dims, number=int(opt.get("-number", 300)),
                             iter_voxels=int(opt.get("-iter_voxels", 0)), dilate_passes=int(opt.get("-dilate", 1)),
                             max_iters=int(opt.get("-max_iters", 10)), lmax=lmax)
    mean, std = masked_mean_std(dw_dev.cpu().numpy(), mask)
    mean, std = mean * np.sqrt(4.0 * np.pi), std * np.sqrt(4.0 * np.pi)
    init_rf = [mean, -0.5 * std, 0.25 * std * std / mean]
    return tax_loop(step, fit, mask, init_rf, peak_ratio=float(opt.get("-peak_ratio", 0.1)),
                    max_iters=int(opt.get("-max_iters", 20)), convergence=float(opt.get("-convergence", 0.5)),
                    lmax=lmax)


def _load(path, opt):
    img = mif.read(path)
    if img.data.ndim != 4:
        raise SystemExit("dwi2response: the DW image must be 4-D")
    try:
        grad = mif.dw_scheme(img, opt)
    except ValueError as e:
        raise SystemExit(f"dwi2response: {e}")
    return img, grad


def run(argv) -> int:
    pos, opt = _parse(argv)
    if not pos or pos[0] not in ("fa", "manual", "tournier", "tax"):
        raise SystemExit("usage: python -m mrtrix3_b200.dwi2response fa|manual|tournier|tax ... (other algorithms "
                         "are not provided)")
    algo = pos[0]
    if algo in ("fa", "tournier", "tax") and len(pos) != 3 or algo == "manual" and len(pos) != 4:
        raise SystemExit(f"dwi2response {algo}: wrong number of arguments")
    if "-shells" in opt and algo in ("fa", "manual"):
        raise SystemExit(f"dwi2response {algo}: -shells is provided for tournier and tax only")
    if algo in ("tournier", "tax"):
        if "-lmax" in opt and len(opt["-lmax"].split(",")) != 1:
            raise SystemExit("Can only specify a single lmax value for single-shell algorithms")
        if "-shells" in opt and len(opt["-shells"].split(",")) != 1:
            raise SystemExit("Can only specify a single b-value shell for single-shell algorithms")
    out_path = pos[-1]
    if os.path.exists(out_path) and not opt.get("-force"):
        raise SystemExit(f"dwi2response: output file \"{out_path}\" already exists (use -force to replace it)")
    if algo in ("fa", "tournier", "tax") and "-mask" not in opt:
        raise SystemExit(f"dwi2response {algo}: -mask is required (no automatic brain mask is provided)")
    img, grad = _load(pos[1], opt)
    nx, ny, nz, nvol = img.data.shape
    dims = (nx, ny, nz)
    g = msmt.normalise_scheme(grad)
    shells = msmt.cluster_shells(g[:, 3])
    first_b0 = float(np.mean(g[shells[0], 3])) <= 10.0

    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    # voxel rows in the image's x-fastest order (mif.Image data is [x][y][z][..])
    dwi = torch.from_numpy(np.ascontiguousarray(
        img.data.transpose(2, 1, 0, 3).reshape(-1, nvol), np.float32)).to(dev)

    def rows(a):  # [x y z (c)] -> [z y x] rows
        a = np.asarray(a)
        return np.ascontiguousarray(a.transpose((2, 1, 0) + tuple(range(3, a.ndim))).reshape(nx * ny * nz, -1)
                                    if a.ndim > 3 else a.transpose(2, 1, 0).reshape(-1))

    if algo in ("tournier", "tax"):
        mask = rows(mif.read(opt["-mask"]).data.reshape(dims) != 0)
        if not mask.any():
            raise SystemExit("Provided mask image does not contain any voxels")
        try:
            resp, voxels, _ = iterative(algo, opt, g, shells, dwi, mask, dims)
        except ZeroDivisionError:
            raise SystemExit(f"dwi2response {algo}: a response coefficient's mean over two rounds is zero "
                             "(the script stops with a division by zero there)")
        np.savetxt(out_path, resp.reshape(1, -1), fmt="%.10g")
        if "-voxels" in opt:
            vox = voxels.reshape(nz, ny, nx).transpose(2, 1, 0).astype(np.float64)
            mif.write(opt["-voxels"], mif.Image(data=vox, vox=list(img.vox)[:3], transform=img.transform),
                      datatype="UInt8")
        return 0

    if algo == "fa":
        mask = rows(mif.read(opt["-mask"]).data.reshape(dims) != 0)
        _, _, fa, vec = dwi2tensor(dwi, grad, torch.from_numpy(mask.astype(np.uint8)).to(dev))
        fa_h = fa.cpu().numpy()
        if "-threshold" in opt:
            voxels = fa_h >= float(opt["-threshold"])
        else:
            voxels = fa_h >= top_threshold(fa_h, int(opt.get("-number", 300)))
        # the largest non-b=0 shell only (dwiextract -singleshell -no_bzero)
        dw_shells = [v for v in shells if float(np.mean(g[v, 3])) > 10.0]
        vols = dw_shells[-1]
        lmax = [int(opt["-lmax"])] if "-lmax" in opt else [10]
        resp = AR.responses(dwi, vec, torch.from_numpy(voxels.astype(np.uint8)).to(dev),
                            [msmt.direction_matrix(g, vols)], [vols], lmax)
    else:
        voxels = rows(mif.read(pos[2]).data.reshape(dims) != 0)
        vm = torch.from_numpy(voxels.astype(np.uint8)).to(dev)
        if "-dirs" in opt:
            d = mif.read(opt["-dirs"]).data
            if d.ndim != 4 or d.shape[3] < 3 or d.shape[:3] != dims:
                raise SystemExit("dwi2response manual: the -dirs image must be [x y z 3]")
            vec = torch.from_numpy(rows(d[..., :3]).astype(np.float32)).to(dev)
        else:
            _, _, _, vec = dwi2tensor(dwi, grad, vm)
        if "-lmax" in opt:
            lmax = [int(v) for v in opt["-lmax"].split(",")]
            if len(lmax) != len(shells):
                raise SystemExit(f"Number of manually-defined lmax's ({len(lmax)}) does not match number of b-value "
                                 f"shells ({len(shells)})")
            if any(l % 2 or l < 0 for l in lmax):
                raise SystemExit("Values for lmax must be even and non-negative")
        else:
            lmax = AR.default_lmax(len(shells), first_b0)
        resp = AR.responses(dwi, vec, vm, [msmt.direction_matrix(g, v) for v in shells], shells, lmax)
    np.savetxt(out_path, resp, fmt="%.10g")
    if "-voxels" in opt:
        vox = voxels.reshape(nz, ny, nx).transpose(2, 1, 0).astype(np.float64)
        mif.write(opt["-voxels"], mif.Image(data=vox, vox=list(img.vox)[:3], transform=img.transform),
                  datatype="UInt8")
    return 0


def main():
    sys.exit(run(sys.argv[1:]))


if __name__ == "__main__":
    main()
