"""``fod2fixel`` on MRtrix image files, the FMLS segmentation on the GPU.

    python -m mrtrix3_b200.fod2fixel <fod> <fixel_directory> [options]

Mirrors cmd/fod2fixel.cpp:288-330: the FOD image (4-D, SH coefficients) is
segmented voxel by voxel (fmls.cu); the fixel directory receives
``index.mif`` (UInt32 [x y z 2]: fixels in the voxel, offset of its first;
``nfixels`` key), ``directions.mif`` (Float32 [nfixels 3 1]) and the
optional metric images (Float32 [nfixels 1 1]).  Fixels are stored in voxel
order, x fastest (the reference's order is that of its worker threads;
per voxel the fixels and their order are the same).

Options: -afd image, -peak_amp image, -disp image, -mask image, -maxnum N,
-dirpeak, -nii (not provided: .mif only), -fmls_integral v,
-fmls_peak_value v, -fmls_no_thresholds, -fmls_lobe_merge_ratio v.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import fmls, mif, sh

_VALUED = {"-afd", "-peak_amp", "-disp", "-mask", "-maxnum", "-fmls_integral", "-fmls_peak_value",
           "-fmls_lobe_merge_ratio", "-nthreads"}
_FLAGS = {"-dirpeak", "-fmls_no_thresholds", "-force", "-quiet", "-info", "-nii"}


def _parse(argv):
    pos, opt = [], {}
    i = 0
    while i < len(argv):
        a = argv[i]
        key = "-" + a.lstrip("-") if a.startswith("-") and len(a) > 1 and not _number(a) else None
        if key is not None and key not in _VALUED and key not in _FLAGS:
            # an unambiguous prefix names its option (as -peak for -peak_amp)
            cand = [o for o in sorted(_VALUED | _FLAGS) if o.startswith(key)]
            if len(cand) == 1:
                key = cand[0]
        if key in _VALUED:
            if i + 1 >= len(argv):
                raise SystemExit(f"fod2fixel: option \"{a}\" expects a value")
            opt[key] = argv[i + 1]
            i += 2
        elif key in _FLAGS:
            opt[key] = True
            i += 1
        elif key is not None:
            raise SystemExit(f"fod2fixel: unknown option \"{a}\"")
        else:
            pos.append(a)
            i += 1
    return pos, opt


def _number(s):
    try:
        float(s)
        return True
    except ValueError:
        return False


def thresholds(opt):
    """load_fmls_thresholds (fmls.cpp:56-84)."""
    integral, peak = fmls.INTEGRAL_THRESHOLD_DEFAULT, fmls.PEAK_VALUE_THRESHOLD_DEFAULT
    if opt.get("-fmls_no_thresholds"):
        integral = peak = 0.0
    else:
        if "-fmls_integral" in opt:
            integral = float(opt["-fmls_integral"])
        if "-fmls_peak_value" in opt:
            peak = float(opt["-fmls_peak_value"])
    merge = float(opt.get("-fmls_lobe_merge_ratio", fmls.MERGE_RATIO_DEFAULT))
    if integral < 0.0 or peak < 0.0:
        raise SystemExit("fod2fixel: FMLS thresholds must be non-negative")
    if not 0.0 <= merge <= 1.0:
        raise SystemExit("fod2fixel: -fmls_lobe_merge_ratio must be within [0, 1]")
    return integral, peak, merge


def run(argv) -> int:
    pos, opt = _parse(argv)
    if len(pos) != 2:
        raise SystemExit("usage: python -m mrtrix3_b200.fod2fixel <fod> <fixel_directory> [options]")
    if opt.get("-nii"):
        raise SystemExit("fod2fixel: -nii is not provided (fixel images are written as .mif)")
    in_path, out_dir = pos
    img = mif.read(in_path)
    if img.data.ndim != 4:
        raise SystemExit("fod2fixel: the FOD image must be 4-D")
    nx, ny, nz, nc = img.data.shape
    lmax = sh.l_for_n(nc)
    if sh.n_for_l(lmax) != nc:
        raise SystemExit("fod2fixel: the number of volumes does not match a valid SH series")
    maxnum = int(opt.get("-maxnum", 0))
    if "-maxnum" in opt and maxnum < 1:
        raise SystemExit("fod2fixel: -maxnum must be at least 1")
    integral, peak, merge = thresholds(opt)
    mask = None
    if "-mask" in opt:
        m = mif.read(opt["-mask"])
        if m.data.shape[:3] != (nx, ny, nz):
            raise SystemExit(f"Cannot use image \"{opt['-mask']}\" as mask image; dimensions do not match FOD image")
        mask = m.data.reshape(nx, ny, nz, -1)[..., 0] != 0
    if os.path.exists(out_dir):
        if not os.path.isdir(out_dir):
            raise SystemExit(f"{out_dir} is not a directory")
        if os.listdir(out_dir):
            raise SystemExit(f"Output fixel directory \"{out_dir}\" is not empty")

    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    # voxel rows x fastest (the reference's loop order over axes 0..2)
    rows = np.ascontiguousarray(img.data.transpose(2, 1, 0, 3).reshape(-1, nc), np.float32)
    mrows = None if mask is None else np.ascontiguousarray(mask.transpose(2, 1, 0).reshape(-1))
    seg = fmls.Segmenter(lmax, integral, peak, merge)
    counts, fixels = seg.segment(torch.from_numpy(rows).to(dev),
                                 None if mrows is None else torch.from_numpy(mrows.astype(np.uint8)).to(dev),
                                 max_fixels=maxnum)
    counts, offsets, dirs, afd, pk, disp = fmls.pack(counts.cpu().numpy(), fixels.cpu().numpy(),
                                                     dirpeak=bool(opt.get("-dirpeak")))
    nfix = int(counts.sum())
    os.makedirs(out_dir, exist_ok=True)
    if nfix == 0:
        return 0  # the reference writes nothing when there are no fixels (fod2fixel.cpp:202-203)
    offsets = np.where(counts > 0, offsets, 0)
    vox3 = list(img.vox)[:3]
    keyval = dict(img.keyval)
    index = np.stack([counts, offsets], axis=1).reshape(nz, ny, nx, 2).transpose(2, 1, 0, 3)
    mif.write(os.path.join(out_dir, "index.mif"),
              mif.Image(data=index, vox=vox3 + [1.0], transform=img.transform, keyval={**keyval, "nfixels": str(nfix)}),
              datatype=mif._spec(np.dtype("=u4")))

    def data_image(name, arr):
        mif.write(os.path.join(out_dir, name), mif.Image(data=arr, vox=vox3, transform=img.transform, keyval=keyval))

    data_image("directions.mif", dirs.reshape(nfix, 3, 1))
    for key, arr in (("-afd", afd), ("-peak_amp", pk), ("-disp", disp)):
        if key in opt:
            data_image(opt[key], arr.reshape(nfix, 1, 1))
    return 0


def main():
    sys.exit(run(sys.argv[1:]))


if __name__ == "__main__":
    main()
