"""``amp2response`` on the GPU: a response function from the amplitudes of
single-fibre voxels (MRtrix3 cmd/amp2response.cpp:199-380).

    python -m mrtrix3_b200.amp2response <amps> <mask> <directions> <response.txt> [options]

Per b-value shell (every shell of the gradient table, or one set of
``-directions`` / header ``directions``): the normal equations of the zonal
fit are accumulated on the GPU over the mask's voxels, each voxel's volumes
placed by their elevation from the voxel's fibre direction
(csd_amp2response_accumulate); then the fit is solved on the GPU, by the
ICLS solver in standard form with the response's amplitude and its
derivative in elevation kept non-negative at 0, 1, .., 90 degrees
(amp2response.cpp:337-349), or unconstrained (``-noconstraint``, and for
lmax 0: M^-1 b).  The output holds one row per shell of even zonal
coefficients, padded to the largest lmax.

Options: -lmax l1,l2,.. (one per shell; default 0 for a b=0 shell, else
10), -isotropic (lmax 0 everywhere), -noconstraint, -directions file,
-shells b1,b2,.. (Shells::select_shells), -grad file, -force.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

from . import mif, sh


def zonal_amp_transform(els, lmax: int) -> np.ndarray:
    """ZSH::init_amp_transform (core/math/ZSH.h:66-77): [n][lmax/2 + 1]
    normalised Legendre P_l0(cos el), even l."""
    els = np.asarray(els, np.float64)
    P = sh.plm_sph(lmax, 0, np.cos(els))
    return np.stack([P[l] for l in range(0, lmax + 1, 2)], axis=1)


def zonal_deriv_transform(els, lmax: int) -> np.ndarray:
    """ZSH::init_deriv_transform (ZSH.h:87-99): d/d(el) of the zonal basis,
    sqrt(l (l + 1)) P_l1(cos el) for l >= 2, 0 for l = 0."""
    els = np.asarray(els, np.float64)
    P = sh.plm_sph(lmax, 1, np.cos(els)) if lmax >= 1 else None
    cols = [np.zeros(len(els))]
    for l in range(2, lmax + 1, 2):
        cols.append(P[l] * math.sqrt(l * (l + 1)))
    return np.stack(cols, axis=1)


def constraint_matrix(lmax: int) -> np.ndarray:
    """Amplitude and elevation-derivative rows at 0, 1, .., 90 degrees
    (amp2response.cpp:337-344)."""
    els = np.arange(91) * math.pi / 180.0
    return np.vstack([zonal_amp_transform(els, lmax), zonal_deriv_transform(els, lmax)])


def accumulate(amp, fibre_dir, shell_dirs, volumes, lmax: int, mask=None, stream=None):
    """(M [nz][nz] lower, b [nz]) device float64 for one shell: amp device
    float32 [n][volumes]; fibre_dir device float32 [n][3]; shell_dirs host
    [nd][3] unit vectors (NaN rows for b=0 volumes); volumes their indices."""
    import ctypes

    import torch

    from . import csd
    dev = amp.device
    nz = lmax // 2 + 1
    M = torch.zeros((nz, nz), dtype=torch.float64, device=dev)
    b = torch.zeros(nz, dtype=torch.float64, device=dev)
    d = torch.from_numpy(np.ascontiguousarray(shell_dirs, np.float64)).to(dev)
    vol = np.asarray(volumes, np.int64)
    if len(vol) and (vol.min() < 0 or vol.max() >= amp.shape[1]):
        raise ValueError("amp2response: volume index out of range")
    v = torch.from_numpy(np.ascontiguousarray(vol, np.int32)).to(dev)
    if fibre_dir.dim() != 2 or fibre_dir.shape[1] < 3 or fibre_dir.shape[0] != amp.shape[0]:
        raise ValueError("amp2response: fibre directions must be [n][>= 3]")
    m = None if mask is None else mask.to(torch.uint8)
    csd.check(csd.lib().csd_amp2response_accumulate(
        ctypes.c_void_p(amp.data_ptr()), amp.shape[0], amp.stride(0), amp.stride(1),
        ctypes.c_void_p(fibre_dir.data_ptr()), fibre_dir.stride(0), fibre_dir.stride(1),
        ctypes.c_void_p(m.data_ptr()) if m is not None else None, ctypes.c_void_p(d.data_ptr()), len(vol),
        ctypes.c_void_p(v.data_ptr()), int(lmax), ctypes.c_void_p(M.data_ptr()), ctypes.c_void_p(b.data_ptr()),
        ctypes.c_void_p(csd._stream_ptr(stream))))
    return M, b


def fit(M, b, lmax: int, constrained: bool = True) -> np.ndarray:
    """The shell's response coefficients from the accumulated normal
    equations, on the GPU (amp2response.cpp:330-351)."""
    import torch

    from .msmt import ICLSProblem
    Mh = M.cpu().numpy()
    Mh = np.tril(Mh) + np.tril(Mh, -1).T
    nz = lmax // 2 + 1
    if lmax == 0 or not constrained:
        # M^-1 b: the solver's unconstrained step (one constraint that can never bind)
        P = ICLSProblem(Mh, np.eye(1, nz), np.array([-1.0e300]), standard_form=True)
    else:
        P = ICLSProblem(Mh, constraint_matrix(lmax), None, 0, 1e-10, 1e-10, 0, 0.0, standard_form=True)
    x, _ = P.solve_f64(b.reshape(1, -1).to(torch.float64).contiguous())
    return x.cpu().numpy()[0]


def responses(amp, fibre_dir, mask, dirs_azel, volumes, lmax, constrained: bool = True) -> np.ndarray:
    """The response rows for the shells given by their [az el] directions and
    volume indices (device amp [n][volumes], fibre_dir [n][3], mask [n]):
    [shells][lmax_max/2 + 1], each row padded with zeros."""
    max_lmax = max(lmax)
    rows = []
    for s, (da, vols, L) in enumerate(zip(dirs_azel, volumes, lmax)):
        if L and not np.isfinite(zonal_amp_transform(da[:, 1], L)).all():
            raise ValueError(f"Unable to construct A2SH transformation for shell {s}; lmax ({L}) may be too large "
                             "for this shell")
        cart = np.stack([np.cos(da[:, 0]) * np.sin(da[:, 1]), np.sin(da[:, 0]) * np.sin(da[:, 1]), np.cos(da[:, 1])],
                        axis=1)
        M, b = accumulate(amp, fibre_dir, cart, vols, L, mask)
        rf = fit(M, b, L, constrained=constrained)
        row = np.zeros(max_lmax // 2 + 1)
        row[:len(rf)] = rf
        rows.append(row)
    return np.array(rows)


def default_lmax(n_shells: int, first_is_bzero: bool):
    """amp2response.cpp:287-294: 0 for a b=0 first shell, else 10."""
    return [0 if (i == 0 and first_is_bzero) else 10 for i in range(n_shells)]


def _parse(argv):
    pos, opt = [], {}
    i = 0
    while i < len(argv):
        a = argv[i]
        key = "-" + a.lstrip("-") if a.startswith("-") and len(a) > 1 else None
        if key in ("-lmax", "-directions", "-grad", "-nthreads", "-shells"):
            if i + 1 >= len(argv):
                raise SystemExit(f"amp2response: option \"{a}\" expects a value")
            opt[key] = argv[i + 1]
            i += 2
        elif key in ("-isotropic", "-noconstraint", "-force", "-quiet", "-info"):
            opt[key] = True
            i += 1
        elif key is not None:
            raise SystemExit(f"amp2response: unknown option \"{a}\"")
        else:
            pos.append(a)
            i += 1
    return pos, opt


def run(argv) -> int:
    pos, opt = _parse(argv)
    if len(pos) != 4:
        raise SystemExit("usage: python -m mrtrix3_b200.amp2response <amps> <mask> <directions> <response> [options]")
    amp_path, mask_path, dir_path, out_path = pos
    if os.path.exists(out_path) and not opt.get("-force"):
        raise SystemExit(f"amp2response: output file \"{out_path}\" already exists (use -force to replace it)")
    img = mif.read(amp_path)
    if img.data.ndim != 4:
        raise SystemExit("amp2response: the amplitude image must be 4-D")
    nx, ny, nz_, nvol = img.data.shape
    from . import msmt
    shells_b0 = False
    if "-directions" in opt or "directions" in img.keyval:
        if "-directions" in opt:
            d = mif.load_matrix(opt["-directions"])
        else:
            vals = [float(v) for line in img.keyval["directions"].split("\n") for v in line.replace(",", " ").split()]
            d = np.array(vals, np.float64).reshape(-1, 2)
        if d.shape[1] == 3:
            d = sh.cartesian_to_azel(d)
        dirs_azel, volumes = [d], [np.arange(len(d))]
    else:
        grad = mif.load_matrix(opt["-grad"]) if "-grad" in opt else (
            mif.parse_scheme(img.keyval["dw_scheme"]) if "dw_scheme" in img.keyval else None)
        if grad is None:
            raise SystemExit("amp2response: no directions or diffusion encoding found")
        grad = msmt.normalise_scheme(grad)
        shells = msmt.cluster_shells(grad[:, 3])
        if "-shells" in opt:
            try:
                keep = msmt.select_shells(grad[:, 3], shells, [float(v) for v in opt["-shells"].split(",")])
            except ValueError as e:
                raise SystemExit(f"amp2response: {e}")
            shells = [shells[i] for i in keep]
        shells_b0 = float(np.mean(grad[shells[0], 3])) <= 10.0
        volumes = shells
        dirs_azel = [msmt.direction_matrix(grad, v) for v in shells]
    if opt.get("-isotropic"):
        lmax = [0] * len(dirs_azel)
    elif "-lmax" in opt:
        lmax = [int(v) for v in opt["-lmax"].split(",")]
        if len(lmax) != len(dirs_azel):
            raise SystemExit(f"Number of lmax's specified ({len(lmax)}) does not match number of b-value shells "
                             f"({len(dirs_azel)})")
        if any(l % 2 for l in lmax):
            raise SystemExit("Values specified for lmax must be even")
    else:
        lmax = default_lmax(len(dirs_azel), shells_b0)
    m = mif.read(mask_path)
    if m.data.shape[:3] != (nx, ny, nz_) or int(np.prod(m.data.shape[3:])) != 1:
        raise SystemExit("amp2response: the mask must be a 3-D image of the amplitude image's dimensions")
    dimg = mif.read(dir_path)
    if dimg.data.ndim < 4 or dimg.data.shape[3] < 3 or dimg.data.shape[:3] != (nx, ny, nz_):
        raise SystemExit(f"amp2response: input direction image \"{dir_path}\" does not have expected dimensions")
    mask = (m.data.reshape(-1) != 0)
    if not mask.any():
        raise SystemExit("input mask does not contain any voxels")

    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    amp = torch.from_numpy(np.ascontiguousarray(img.data.reshape(-1, nvol), np.float32)).to(dev)
    fdir = torch.from_numpy(np.ascontiguousarray(dimg.data.reshape(-1, dimg.data.shape[3])[:, :3], np.float32)).to(dev)
    mk = torch.from_numpy(mask.astype(np.uint8)).to(dev)
    try:
        rows = responses(amp, fdir, mk, dirs_azel, volumes, lmax, constrained=not opt.get("-noconstraint"))
    except ValueError as e:
        raise SystemExit(str(e))
    np.savetxt(out_path, rows, fmt="%.10g")
    return 0


def main():
    sys.exit(run(sys.argv[1:]))


if __name__ == "__main__":
    main()
