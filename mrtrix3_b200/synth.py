"""Seeded synthetic single-shell DWI volumes for parity tests and benchmarks.

No public dataset is named for this path, so every workload is generated:

* gradient table rows ``[x y z b]``: b=0 rows are ``[0 0 0 0]``; DW rows are
  unit vectors at b=3000, either a Fibonacci hemisphere or (``random_dirs``)
  an independent uniform random set;
* each voxel holds 1-3 fibres (count uniform), orientations uniform on the
  sphere with >= 30 degrees pairwise separation (axial, so |u.v| <= cos 30),
  volume fractions Dirichlet(1);
* the DW signal of fibre u at gradient g is ``sum_l r_l sqrt((2l+1)/4pi)
  P_l(g.u)`` with zonal response ``r = [1700,-700,240,-60,10]`` -- exactly
  CSD's forward model M . delta_u; b=0 volumes hold S0 (default 1500);
* Rician noise with sigma = S0 / SNR (SNR defined on b=0);
* storage float32, voxel-interleaved ``[z][y][x][volume]`` (the layout
  dwi2fod reads with ``with_direct_io(3)``, cmd/dwi2fod.cpp:279).

Masks are centred ellipsoids scaled to the requested volume fraction.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

RESPONSE = np.array([1700.0, -700.0, 240.0, -60.0, 10.0])
S0_DEFAULT = 1500.0


def fibonacci_hemisphere(n: int) -> np.ndarray:
    i = np.arange(n) + 0.5
    z = 1.0 - i / n
    phi = math.pi * (1.0 + math.sqrt(5.0)) * i
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)


def random_directions(n: int, rng: np.random.Generator) -> np.ndarray:
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    u[u[:, 2] < 0] *= -1.0
    return u


def grad_table(n_b0: int, dirs: np.ndarray, bval: float = 3000.0) -> np.ndarray:
    """Gradient table [n_b0 + ndw][4] with the b=0 rows spread through it."""
    ndw = len(dirs)
    nvol = n_b0 + ndw
    b0pos = set(int(round(k * nvol / max(n_b0, 1))) for k in range(n_b0))
    g = np.zeros((nvol, 4))
    j = 0
    for v in range(nvol):
        if v in b0pos:
            continue
        g[v, :3] = dirs[j]
        g[v, 3] = bval
        j += 1
    assert j == ndw
    return g


def _zonal_sum(x: np.ndarray, coef: np.ndarray) -> np.ndarray:
    """sum_k coef[k] P_{2k}(x) via Bonnet's recursion."""
    lmax = 2 * (len(coef) - 1)
    acc = np.full_like(x, coef[0])
    p0 = np.ones_like(x)
    p1 = x.copy()
    for l in range(1, lmax):
        p2 = (2 * l + 1) / (l + 1) * x * p1
        p2 -= l / (l + 1) * p0
        p0, p1 = p1, p2
        if (l + 1) % 2 == 0:
            acc += coef[(l + 1) // 2] * p2
    return acc


def _sample_fibres(rng: np.random.Generator, nv: int):
    k = rng.integers(1, 4, size=nv)
    u = rng.normal(size=(nv, 3, 3))
    u /= np.linalg.norm(u, axis=2, keepdims=True)
    c30 = math.cos(math.radians(30.0))

    def bad(u, k):
        d01 = np.abs(np.einsum("ij,ij->i", u[:, 0], u[:, 1])) > c30
        d02 = np.abs(np.einsum("ij,ij->i", u[:, 0], u[:, 2])) > c30
        d12 = np.abs(np.einsum("ij,ij->i", u[:, 1], u[:, 2])) > c30
        return ((k >= 2) & d01) | ((k >= 3) & (d02 | d12))

    b = bad(u, k)
    while b.any():
        idx = np.nonzero(b)[0]
        r = rng.normal(size=(len(idx), 3, 3))
        r /= np.linalg.norm(r, axis=2, keepdims=True)
        u[idx] = r
        b[idx] = bad(u[idx], k[idx])
    f = rng.dirichlet(np.ones(3), size=nv)
    # Dirichlet(1) over the first k fibres: renormalise the unused tail away
    for kk in (1, 2):
        sel = k == kk
        if sel.any():
            g = rng.dirichlet(np.ones(kk), size=int(sel.sum()))
            f[sel] = 0.0
            f[np.ix_(np.nonzero(sel)[0], np.arange(kk))] = g
    return k, u, f


def voxel_signals(rng: np.random.Generator, grad: np.ndarray, nv: int, snr, s0: float = S0_DEFAULT,
                  response: np.ndarray = RESPONSE, chunk: int = 4096) -> np.ndarray:
    """[nv][nvol] float32 noisy signals.  ``snr`` is a number or (lo, hi)."""
    nvol = grad.shape[0]
    dw = grad[:, 3] > 10.0
    gd = grad[dw, :3]
    lmax = 2 * (len(response) - 1)
    coef = np.array([response[l // 2] * math.sqrt((2 * l + 1) / (4 * math.pi)) for l in range(0, lmax + 1, 2)])
    out = np.empty((nv, nvol), np.float32)
    for s in range(0, nv, chunk):
        m = min(chunk, nv - s)
        k, u, f = _sample_fibres(rng, m)
        sig = np.zeros((m, gd.shape[0]))
        for fi in range(3):
            sig += f[:, fi:fi + 1] * _zonal_sum(u[:, fi] @ gd.T, coef)
        full = np.empty((m, nvol))
        full[:, dw] = sig
        full[:, ~dw] = s0
        if isinstance(snr, tuple):
            snr_v = rng.uniform(snr[0], snr[1], size=(m, 1))
        else:
            snr_v = np.full((m, 1), float(snr))
        sigma = s0 / snr_v
        n1 = rng.normal(size=full.shape)
        n2 = rng.normal(size=full.shape)
        out[s:s + m] = np.sqrt((full + sigma * n1) ** 2 + (sigma * n2) ** 2).astype(np.float32)
    return out


def _signals_block(args):
    grad, n, snr, seed, index = args
    return voxel_signals(np.random.default_rng([seed, index]), grad, n, snr)


def voxel_signals_parallel(grad: np.ndarray, nv: int, snr, seed: int, workers: int = 0,
                           block: int = 1 << 20) -> np.ndarray:
    """voxel_signals over blocks of ``block`` voxels, block i drawn from the
    generator seeded [seed, i]: the result depends on (seed, nv, block) only,
    not on the number of worker processes (``workers`` <= 1: this process).
    Workers are spawned, so this is safe to call after CUDA is initialised."""
    jobs = [(grad, min(block, nv - a), snr, seed, i) for i, a in enumerate(range(0, nv, block))]
    if workers <= 1 or len(jobs) == 1:
        parts = [_signals_block(j) for j in jobs]
    else:
        import concurrent.futures
        import multiprocessing
        with concurrent.futures.ProcessPoolExecutor(max_workers=workers,
                                                    mp_context=multiprocessing.get_context("spawn")) as ex:
            parts = list(ex.map(_signals_block, jobs))
    return np.concatenate(parts) if parts else np.empty((0, grad.shape[0]), np.float32)


def ellipsoid_mask(dims, fraction: float) -> np.ndarray:
    """uint8 [z][y][x] centred ellipsoid covering about ``fraction`` of the box."""
    nx, ny, nz = dims
    s = (fraction / (math.pi / 6.0)) ** (1.0 / 3.0)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r = (((x - (nx - 1) / 2) / (s * nx / 2)) ** 2 + ((y - (ny - 1) / 2) / (s * ny / 2)) ** 2
         + ((z - (nz - 1) / 2) / (s * nz / 2)) ** 2)
    return (r <= 1.0).astype(np.uint8).reshape(-1)


@dataclasses.dataclass
class Volume:
    dims: tuple
    grad: np.ndarray          # [nvol][4]
    dwi: np.ndarray           # [nvox][nvol] float32
    mask: np.ndarray | None   # [nvox] uint8
    lmax: int
    s0: float

    @property
    def n_voxels(self) -> int:
        return self.dwi.shape[0]

    @property
    def n_masked(self) -> int:
        return int(self.mask.sum()) if self.mask is not None else self.n_voxels


def make_volume(dims, n_b0: int, ndw: int, snr, lmax: int, mask_fraction: float | None, seed: int,
                random_dirs: bool = False, s0: float = S0_DEFAULT, voxel_limit: int | None = None) -> Volume:
    """A synthetic DWI volume.  Voxels outside the mask hold noise only."""
    rng = np.random.default_rng(seed)
    dirs = random_directions(ndw, rng) if random_dirs else fibonacci_hemisphere(ndw)
    grad = grad_table(n_b0, dirs)
    nvox = int(np.prod(dims))
    mask = ellipsoid_mask(dims, mask_fraction) if mask_fraction else None
    if voxel_limit is not None and voxel_limit < nvox:
        nvox = voxel_limit
        if mask is not None:
            mask = mask[:nvox]
    nvol = grad.shape[0]
    if mask is None:
        dwi = voxel_signals(rng, grad, nvox, snr, s0)
    else:
        dwi = np.empty((nvox, nvol), np.float32)
        inside = np.nonzero(mask)[0]
        dwi[inside] = voxel_signals(rng, grad, len(inside), snr, s0)
        outside = np.nonzero(mask == 0)[0]
        sigma = s0 / (snr[0] if isinstance(snr, tuple) else snr)
        for a in range(0, len(outside), 16384):
            o = outside[a:a + 16384]
            n1 = rng.standard_normal(size=(len(o), nvol), dtype=np.float32)
            n2 = rng.standard_normal(size=(len(o), nvol), dtype=np.float32)
            dwi[o] = sigma * np.sqrt(n1 * n1 + n2 * n2)
    return Volume(tuple(dims), grad, dwi, mask, lmax, s0)


# The five workloads (sizes, schemes and noise as the benchmark defines them).
def config1(seed=1, voxel_limit=None):
    """32x32x20, 6 b=0 + 64 DW, SNR 30, no mask, lmax 8."""
    return make_volume((32, 32, 20), 6, 64, 30.0, 8, None, seed, voxel_limit=voxel_limit)


def config2(seed=2, voxel_limit=None):
    """96x96x60, ellipsoid mask ~50%, 6 + 60, SNR U[15,40], lmax 8."""
    return make_volume((96, 96, 60), 6, 60, (15.0, 40.0), 8, 0.5, seed, voxel_limit=voxel_limit)


def config3(seed=3, voxel_limit=None):
    """140x140x96, mask ~45%, 8 + 90, SNR U[15,40], lmax 10."""
    return make_volume((140, 140, 96), 8, 90, (15.0, 40.0), 10, 0.45, seed, voxel_limit=voxel_limit)


def _config4_specs(seed, n_volumes, scale):
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_volumes):
        dims = (int(rng.integers(64, 129) * scale), int(rng.integers(64, 129) * scale),
                int(rng.integers(64, 81) * scale))
        specs.append((tuple(max(4, d) for d in dims), seed * 1000 + i))
    return specs


def _config4_volume(spec):
    dims, vseed = spec
    return make_volume(dims, 6, 60, (15.0, 40.0), 8, 0.5, vseed, random_dirs=True)


def config4(seed=4, n_volumes=16, scale=1.0, workers: int = 0):
    """16 volumes, dims uniform in [64^3, 128x128x80], 6 b=0 + 60 DW each with an
    independent random direction set, SNR U[15,40], lmax 8, mask ~50%.  With
    workers > 1 the volumes are generated by that many spawned processes (the
    same volumes: each has its own seed)."""
    specs = _config4_specs(seed, n_volumes, scale)
    if workers <= 1:
        return [_config4_volume(sp) for sp in specs]
    import concurrent.futures
    import multiprocessing
    with concurrent.futures.ProcessPoolExecutor(max_workers=workers,
                                                mp_context=multiprocessing.get_context("spawn")) as ex:
        return list(ex.map(_config4_volume, specs))


def config5(seed=5, voxel_limit=None):
    """140x140x96, mask ~45%, 6 + 60, SNR U[15,40], lmax 8 (warm-start evaluation)."""
    return make_volume((140, 140, 96), 6, 60, (15.0, 40.0), 8, 0.45, seed, voxel_limit=voxel_limit)


def config5_scheme():
    """The gradient table of config 5 (Fibonacci hemisphere, 6 b=0 + 60 DW)."""
    return grad_table(6, fibonacci_hemisphere(60))


def training_signals(n: int, seed: int = 11, chunk: int = 4096) -> np.ndarray:
    """[n][66] noisy signals on the config-5 scheme for training the warm-start network."""
    rng = np.random.default_rng(seed)
    return voxel_signals(rng, config5_scheme(), n, (15.0, 40.0), chunk=chunk)


def load_hr_dirs() -> np.ndarray:
    """The 300 [az, el] constraint directions (float64)."""
    import os
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "electrostatic_repulsion_300.txt")
    return np.loadtxt(p, dtype=np.float64)


# ---- multi-shell, multi-tissue synthetic data (dwi2fod msmt_csd) ----------

# Per-tissue responses on the shells b = 0, 1000, 2000, 3000 (rows), even
# zonal coefficients l = 0, 2, .. (columns): white matter (anisotropic),
# grey matter and CSF (isotropic).  Invented, of the usual shape.
MSMT_BVALUES = (0.0, 1000.0, 2000.0, 3000.0)
MSMT_RESPONSES = {
    "wm": np.array([[3000.0, 0.0, 0.0, 0.0, 0.0],
                    [1900.0, -650.0, 170.0, -30.0, 4.0],
                    [1300.0, -700.0, 290.0, -85.0, 18.0],
                    [950.0, -640.0, 340.0, -130.0, 35.0]]),
    "gm": np.array([[2600.0], [1150.0], [620.0], [380.0]]),
    "csf": np.array([[4200.0], [1550.0], [580.0], [230.0]]),
}


def msmt_scheme(n_b0: int = 6, ndir=(30, 45, 60)) -> np.ndarray:
    """b = 0 volumes then one shell per entry of ``ndir`` at b = 1000, 2000,
    3000 (Fibonacci hemispheres, each shell rotated about z)."""
    rows = [np.zeros((n_b0, 4))]
    for s, nd in enumerate(ndir):
        d = fibonacci_hemisphere(nd)
        a = 0.37 * (s + 1)
        rot = np.array([[math.cos(a), -math.sin(a), 0.0], [math.sin(a), math.cos(a), 0.0], [0.0, 0.0, 1.0]])
        rows.append(np.hstack([d @ rot.T, np.full((nd, 1), MSMT_BVALUES[s + 1])]))
    return np.vstack(rows)


def msmt_truth(rng: np.random.Generator, nv: int, lmax: int = 8) -> np.ndarray:
    """[nv][nSH(lmax) + 2] true parameters: a white-matter ODF (fraction x the
    SH of 1-3 fibre deltas, truncated at lmax), grey matter, CSF; fractions
    Dirichlet(1, 1, 1), every tenth voxel pure CSF or pure grey matter."""
    from . import sh
    frac = rng.dirichlet([1.0, 1.0, 1.0], nv)
    frac[::10] = [0.0, 0.0, 1.0]
    frac[5::10] = [0.0, 1.0, 0.0]
    k, u, w = _sample_fibres(rng, nv)
    y00 = 1.0 / math.sqrt(4.0 * math.pi)
    out = np.zeros((nv, sh.n_for_l(lmax) + 2))
    for f in range(3):
        d = u[:, f]
        azel = np.stack([np.arctan2(d[:, 1], d[:, 0]), np.arccos(np.clip(d[:, 2], -1, 1))], axis=1)
        Y = sh.init_transform(azel, lmax)
        out[:, :-2] += (w[:, f] * (f < k))[:, None] * Y
    out[:, :-2] *= frac[:, :1]
    out[:, -2] = frac[:, 1] * y00
    out[:, -1] = frac[:, 2] * y00
    return out


def rician(rng: np.random.Generator, clean: np.ndarray, sigma) -> np.ndarray:
    sigma = np.asarray(sigma, np.float64)
    if sigma.ndim == 1:
        sigma = sigma[:, None]
    re = clean + rng.normal(size=clean.shape) * sigma
    im = rng.normal(size=clean.shape) * sigma
    return np.sqrt(re * re + im * im)
