"""``dwi2response fa`` and ``dwi2response manual`` on the GPU: a single-fibre
response function from a DW image (lib/mrtrix3/dwi2response/fa.py,
manual.py), from the library's tensor fit (csd_dwi2tensor) and amp2response
(csd_amp2response_accumulate + the ICLS solver).

    python -m mrtrix3_b200.dwi2response fa <dwi> <response.txt> -mask <mask> [options]
    python -m mrtrix3_b200.dwi2response manual <dwi> <in_voxels> <response.txt> [options]

fa (fa.py): the tensor fit inside the mask; its FA and FA-modulated principal
eigenvector; the voxels of the ``-number`` (300) highest FA values (all
voxels with FA >= the threshold value mrthreshold -top gives) or FA >=
``-threshold``; the response of the largest non-b=0 shell (dwiextract
-singleshell -no_bzero) at lmax ``-lmax`` (default 10).
manual (manual.py): the given voxels; fibre directions from ``-dirs`` or
from the tensor fit over those voxels; the response of every shell, one row
each (``-lmax`` one per shell; default 0 for b=0, else 10).
Options: -mask (required by fa: the brain mask the script would otherwise
make with dwi2mask, which is not provided here, and which it would then
erode), -number, -threshold, -lmax, -dirs, -voxels image, -grad file,
-fslgrad bvecs bvals, -force.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import amp2response as AR
from . import mif, msmt
from .tensor import dwi2tensor

_VALUED = {"-mask", "-number", "-threshold", "-lmax", "-dirs", "-voxels", "-grad", "-nthreads", "-erode"}
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
    if not pos or pos[0] not in ("fa", "manual"):
        raise SystemExit("usage: python -m mrtrix3_b200.dwi2response fa|manual ... (other algorithms are not "
                         "provided)")
    algo = pos[0]
    if algo == "fa" and len(pos) != 3 or algo == "manual" and len(pos) != 4:
        raise SystemExit(f"dwi2response {algo}: wrong number of arguments")
    out_path = pos[-1]
    if os.path.exists(out_path) and not opt.get("-force"):
        raise SystemExit(f"dwi2response: output file \"{out_path}\" already exists (use -force to replace it)")
    if algo == "fa" and "-mask" not in opt:
        raise SystemExit("dwi2response fa: -mask is required (no automatic brain mask is provided)")
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
