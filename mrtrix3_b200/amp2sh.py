"""``amp2sh`` on MRtrix image files, computed by the B200 library.

    python -m mrtrix3_b200.amp2sh <amp> <SH> [options]

Mirrors cmd/amp2sh.cpp:205-265: the directions of the amplitudes come from
``-directions`` ([az el] or [x y z] rows), else the header's ``directions``
key (moved to ``basis_directions`` in the output), else the DW gradient
table (``dw_scheme`` or ``-grad``): the largest shell's volumes are fit, the
b=0 volumes serve ``-normalise``, and the table moves to
``prior_dw_scheme``.  The fit is pinv of the SH-to-amplitude mapping that
DWI::compute_SH2amp_mapping chooses (lmax from the direction count, at most
8 unless ``-lmax`` asks, lowered while poorly conditioned); the output is
float32 with the input's layout.

Options: -lmax N, -normalise, -directions file, -grad file, -rician noise
(a 3-D noise-level image: the fit reweighted for the Rician bias,
amp2sh.cpp:129-150), -force.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import mif, sh


def run(argv) -> int:
    pos, opt = [], {}
    i = 0
    while i < len(argv):
        a = argv[i]
        key = "-" + a.lstrip("-") if a.startswith("-") and len(a) > 1 else None
        if key in ("-lmax", "-directions", "-grad", "-rician", "-nthreads"):
            if i + 1 >= len(argv):
                raise SystemExit(f"amp2sh: option \"{a}\" expects a value")
            opt[key] = argv[i + 1]
            i += 2
        elif key in ("-normalise", "-force", "-quiet", "-info"):
            opt[key] = True
            i += 1
        elif key is not None:
            raise SystemExit(f"amp2sh: unknown option \"{a}\"")
        else:
            pos.append(a)
            i += 1
    if len(pos) != 2:
        raise SystemExit("usage: python -m mrtrix3_b200.amp2sh <amp> <SH> [options]")
    in_path, out_path = pos
    if os.path.exists(out_path) and not opt.get("-force"):
        raise SystemExit(f"amp2sh: output image \"{out_path}\" already exists (use -force to replace it)")
    img = mif.read(in_path)
    if img.data.ndim != 4:
        raise SystemExit("amp2sh: the amplitude image must be 4-D")
    nx, ny, nz, nvol = img.data.shape
    kv = dict(img.keyval)
    dwis, bzeros = np.arange(nvol), np.zeros(0, int)
    if "-directions" in opt:
        dirs = mif.load_matrix(opt["-directions"])
        if dirs.shape[1] == 3:
            dirs = sh.cartesian_to_azel(dirs)
    elif "directions" in kv:
        vals = [float(v) for line in kv["directions"].split("\n") for v in line.replace(",", " ").split()]
        dirs = np.array(vals, np.float64).reshape(-1, 2)
        kv["basis_directions"] = kv.pop("directions")
    else:
        if "-grad" in opt:
            grad = mif.load_matrix(opt["-grad"])
        elif "dw_scheme" in kv:
            grad = mif.parse_scheme(kv["dw_scheme"])
        else:
            raise SystemExit("amp2sh: no directions or diffusion encoding found")
        from . import csd
        # the largest shell's volumes, by the library's shell clustering (the
        # scheme object needs an anisotropic response; any serves here)
        shared = csd.Shared(grad)
        shared.set_response(np.array([1.0, -0.5]))
        shared.init()
        dwis = np.asarray(shared.dwis)
        bzeros = np.nonzero(grad[:, 3] <= shared.bzero_threshold)[0]
        dirs = sh.cartesian_to_azel(grad[dwis, :3])
        kv.pop("dw_scheme", None)
        kv["prior_dw_scheme"] = mif.scheme_to_text(grad)
    for k in ("pe_scheme", "PhaseEncodingDirection", "TotalReadoutTime"):
        kv.pop(k, None)
    if len(dirs) != len(dwis):
        raise SystemExit("amp2sh: the number of directions does not match the number of volumes")
    if opt.get("-normalise") and not len(bzeros):
        raise SystemExit("the normalise option is only available if the input data contains b=0 images.")
    mapping, lmax = sh.sh2amp_mapping(dirs, int(opt["-lmax"]) if "-lmax" in opt else None)
    fit = sh.pinv(mapping)

    import torch

    from . import csd
    dev = torch.device("cuda", torch.cuda.current_device())
    amp = torch.from_numpy(np.ascontiguousarray(img.data.reshape(-1, nvol), np.float32)).to(dev)
    noise = None
    if "-rician" in opt:
        nimg = mif.read(opt["-rician"])
        if nimg.data.shape[:3] != (nx, ny, nz) or int(np.prod(nimg.data.shape[3:])) != 1:
            raise SystemExit("amp2sh: the noise image must be 3-D, with the amplitude image's dimensions")
        noise = torch.from_numpy(np.ascontiguousarray(nimg.data.reshape(-1), np.float32)).to(dev)
    plan = csd.Amp2SHCommon(fit, dwis, bzeros, normalise=bool(opt.get("-normalise")), device=dev,
                            sh2amp=mapping if noise is not None else None)
    out = plan(amp, noise=noise).cpu().numpy()
    res = mif.Image(data=out.reshape(nx, ny, nz, -1), vox=img.vox, transform=img.transform, keyval=kv)
    mif.write(out_path, res, layout=img.layout, datatype="Float32LE" if np.little_endian else "Float32BE")
    return 0


def main():
    sys.exit(run(sys.argv[1:]))


if __name__ == "__main__":
    main()
