"""``sh2peaks`` on MRtrix image files, computed by the B200 library.

    python -m mrtrix3_b200.sh2peaks <SH> <output> [options]

Mirrors cmd/sh2peaks.cpp:304-375: the input is a 4-D image of SH
coefficients (e.g. dwi2fod's FODs); the output holds, per voxel, the x, y, z
components of each peak direction scaled by its amplitude (3 volumes per
peak, float32, NaN where there is no peak).

Options:
  -num N                number of peaks (3)
  -direction phi theta  a peak direction to estimate, in degrees (repeatable;
                        sets the number of peaks)
  -peaks image          find the peaks closest to those in this image
  -threshold v          only peaks with amplitude above v
  -seeds file           [az el] seed directions in radians (the built-in 60)
  -mask image           only voxels inside the mask
  -fast                 accepted; the exact Legendre functions are always used
  -force                overwrite the output
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

from . import mif


def run(argv) -> int:
    pos, opt, dirs = [], {}, []
    i = 0
    while i < len(argv):
        a = argv[i]
        key = "-" + a.lstrip("-") if a.startswith("-") and len(a) > 1 else None
        if key in ("-num", "-peaks", "-threshold", "-seeds", "-mask", "-nthreads"):
            if i + 1 >= len(argv):
                raise SystemExit(f"sh2peaks: option \"{a}\" expects a value")
            opt[key] = argv[i + 1]
            i += 2
        elif key == "-direction":
            if i + 2 >= len(argv):
                raise SystemExit("sh2peaks: option \"-direction\" expects phi and theta")
            dirs.append((float(argv[i + 1]), float(argv[i + 2])))
            i += 3
        elif key in ("-fast", "-force", "-quiet", "-info"):
            opt[key] = True
            i += 1
        elif key is not None and not _number(a):
            raise SystemExit(f"sh2peaks: unknown option \"{a}\"")
        else:
            pos.append(a)
            i += 1
    if len(pos) != 2:
        raise SystemExit("usage: python -m mrtrix3_b200.sh2peaks <SH> <output> [options]")
    in_path, out_path = pos
    if os.path.exists(out_path) and not opt.get("-force"):
        raise SystemExit(f"sh2peaks: output image \"{out_path}\" already exists (use -force to replace it)")
    if dirs and "-peaks" in opt:
        raise SystemExit("you can't specify both a peaks file and orientations to be estimated at the same time")

    import torch

    from . import csd
    img = mif.read(in_path)
    if img.data.ndim != 4:
        raise SystemExit("sh2peaks: the SH image must be 4-D")
    nx, ny, nz, nsh = img.data.shape
    lmax = int(round((math.sqrt(8 * nsh + 1) - 3) / 2))
    if (lmax + 1) * (lmax + 2) // 2 != nsh:
        raise SystemExit("sh2peaks: the number of volumes is not a valid number of SH coefficients")
    npeaks = int(opt.get("-num", 3))
    seeds = mif.load_matrix(opt["-seeds"]) if "-seeds" in opt else None
    if seeds is not None and seeds.shape[1] != 2:
        raise SystemExit("expecting 2 columns for search directions matrix")
    directions = None
    if dirs:
        # Direction(pi phi / 180, pi theta / 180) (sh2peaks.cpp:329-331)
        ph = np.array([math.pi * d[0] / 180.0 for d in dirs])
        th = np.array([math.pi * d[1] / 180.0 for d in dirs])
        directions = np.stack([np.cos(ph) * np.sin(th), np.sin(ph) * np.sin(th), np.cos(th)], axis=1)
        npeaks = len(dirs)
    dev = torch.device("cuda", torch.cuda.current_device())
    sh = torch.from_numpy(np.ascontiguousarray(img.data.reshape(-1, nsh), np.float32)).to(dev)
    mask = None
    if "-mask" in opt:
        m = mif.read(opt["-mask"])
        if m.data.shape[:3] != (nx, ny, nz):
            raise SystemExit("sh2peaks: the mask's dimensions do not match the SH image")
        mask = torch.from_numpy((m.data.reshape(nx, ny, nz) != 0).reshape(-1).astype(np.uint8)).to(dev)
    peaks_in = None
    if "-peaks" in opt:
        p = mif.read(opt["-peaks"])
        if p.data.shape[:3] != (nx, ny, nz):
            raise SystemExit("sh2peaks: the peaks image's dimensions do not match the SH image")
        npeaks = p.data.shape[3] // 3
        peaks_in = torch.from_numpy(np.ascontiguousarray(p.data.reshape(-1, p.data.shape[3])[:, :3 * npeaks],
                                                         np.float32)).to(dev)
    threshold = float(opt.get("-threshold", -np.inf))
    out = csd.sh2peaks(sh, lmax=lmax, mask=mask, seeds=seeds, npeaks=npeaks, threshold=threshold,
                       directions=directions, peaks=peaks_in).cpu().numpy()
    from .dwi2fod import output_layout
    res = mif.Image(data=out.reshape(nx, ny, nz, 3 * npeaks), vox=img.vox, transform=img.transform,
                    keyval=dict(img.keyval))
    mif.write(out_path, res, layout=output_layout(img.layout, 4),
              datatype="Float32LE" if np.little_endian else "Float32BE")
    return 0


def _number(s):
    try:
        float(s)
        return True
    except ValueError:
        return False


def main():
    sys.exit(run(sys.argv[1:]))


if __name__ == "__main__":
    main()
