"""The tensor fit (csd_dwi2tensor) and ``dwi2response fa`` / ``manual``
(mrtrix3_b200/dwi2response.py) against the FP64 restatements
(oracle/tensor_ref.py, oracle/amp2response_ref.py): tensors to 1e-5 of
their largest element, FA to 1e-5, principal directions to 1e-6 in
|cos|; the selected voxels identical and the responses to 1e-6."""
import numpy as np
import pytest

from mrtrix3_b200 import mif, msmt, synth
from mrtrix3_b200.tensor import bmatrix, dwi2tensor
from oracle import amp2response_ref as AREF
from oracle import tensor_ref as TREF

pytestmark = pytest.mark.gpu


def _tensors(rng, n, frac_aniso=0.5):
    f = rng.normal(size=(n, 3))
    f /= np.linalg.norm(f, axis=1, keepdims=True)
    lam = np.where(rng.uniform(size=(n, 1)) < frac_aniso, [[1.7e-3, 0.3e-3, 0.3e-3]], [[0.8e-3, 0.75e-3, 0.7e-3]])
    D = []
    for i in range(n):
        a = f[i]
        h = np.array([0.3, -0.7, 0.64])
        e2 = np.cross(a, h)
        e2 /= np.linalg.norm(e2)
        e3 = np.cross(a, e2)
        R = np.stack([a, e2, e3], axis=1)
        D.append(R @ np.diag(lam[i]) @ R.T)
    return np.array(D), f


def _signals(rng, grad, D, s0=1000.0, sigma=10.0):
    g = grad[:, :3]
    q = np.einsum("vi,nij,vj->nv", g, D, g)
    clean = s0 * np.exp(-grad[:, 3][None, :] * q)
    return synth.rician(rng, clean, sigma).astype(np.float32)


def test_tensor_fit_matches_oracle(cuda):
    import torch
    rng = np.random.default_rng(2)
    grad = synth.msmt_scheme()
    D, f = _tensors(rng, 400)
    dwi = _signals(rng, grad, D)
    mask = (np.arange(400) % 7 != 0).astype(np.uint8)
    dt, b0, fa, vec = dwi2tensor(torch.from_numpy(dwi).to(cuda), grad, torch.from_numpy(mask).to(cuda))
    dt, b0, fa, vec = (t.cpu().numpy().astype(np.float64) for t in (dt, b0, fa, vec))
    B = bmatrix(msmt.normalise_scheme(grad))
    assert not dt[mask == 0].any() and not fa[mask == 0].any()
    for i in np.nonzero(mask)[0][::3]:
        p = TREF.fit(dwi[i].astype(np.float64), B)
        assert np.abs(dt[i] - p[:6]).max() <= 1e-5 * np.abs(p[:6]).max()
        assert abs(b0[i] - np.exp(p[6])) <= 1e-5 * np.exp(p[6])
        fr = TREF.fa(p[:6])
        assert abs(fa[i] - fr) <= 1e-5
        if fr > 0.2:
            v = vec[i] / np.linalg.norm(vec[i])
            assert abs(v @ TREF.principal(p[:6])) >= 1 - 1e-6
            assert abs(np.linalg.norm(vec[i]) - fr) <= 1e-5


def _volume(tmp_path, seed, dims=(9, 8, 7)):
    rng = np.random.default_rng(seed)
    grad = synth.msmt_scheme()
    n = int(np.prod(dims))
    D, f = _tensors(rng, n, 0.4)
    dwi = _signals(rng, grad, D)
    mask = np.ones(n, np.uint8)
    mask[:n // 10] = 0
    nx, ny, nz = dims

    def img(rows_):  # x-fastest rows -> [x y z ...]
        a = np.asarray(rows_)
        return a.reshape((nz, ny, nx) + a.shape[1:]).transpose((2, 1, 0) + tuple(range(3, a.ndim + 2))[:a.ndim - 1])
    p = {k: str(tmp_path / f"{k}.mif") for k in ("dwi", "mask", "dirs", "vox")}
    mif.write(p["dwi"], mif.Image(data=img(dwi), vox=[2.0] * 4, keyval={"dw_scheme": mif.scheme_to_text(grad)}))
    mif.write(p["mask"], mif.Image(data=img(mask).astype(np.float64), vox=[2.0] * 3), datatype="UInt8")
    mif.write(p["dirs"], mif.Image(data=img(f), vox=[2.0] * 4))
    return grad, dwi, mask, f, p


def test_dwi2response_fa(cuda, tmp_path):
    from mrtrix3_b200.dwi2response import run, top_threshold
    grad, dwi, mask, f, p = _volume(tmp_path, 3)
    out = str(tmp_path / "resp.txt")
    assert run(["fa", p["dwi"], out, "-mask", p["mask"], "-number", "40", "-voxels", p["vox"]]) == 0
    got = np.atleast_2d(np.loadtxt(out))
    g = msmt.normalise_scheme(grad)
    B = bmatrix(g)
    fa = np.zeros(len(dwi))
    vec = np.zeros((len(dwi), 3))
    for i in np.nonzero(mask)[0]:
        pr = TREF.fit(dwi[i].astype(np.float64), B)
        fa[i] = TREF.fa(pr[:6])
        vec[i] = TREF.principal(pr[:6]) * fa[i]
    sel = fa >= top_threshold(fa, 40)
    vox = mif.read(p["vox"]).data.transpose(2, 1, 0).reshape(-1) != 0
    np.testing.assert_array_equal(vox, sel)
    shells = msmt.cluster_shells(g[:, 3])
    vols = shells[-1]
    da = msmt.direction_matrix(g, vols)
    cart = np.stack([np.cos(da[:, 0]) * np.sin(da[:, 1]), np.sin(da[:, 0]) * np.sin(da[:, 1]), np.cos(da[:, 1])], 1)
    M, b = AREF.accumulate(dwi, vec, sel, cart, vols, 10)
    want = AREF.fit(M, b, 10)
    assert got.shape == (1, 6)
    assert np.abs(got[0] - want).max() <= 1e-6 * np.abs(want).max()


def test_dwi2response_manual(cuda, tmp_path):
    from mrtrix3_b200.dwi2response import run
    grad, dwi, mask, f, p = _volume(tmp_path, 4)
    g = msmt.normalise_scheme(grad)
    shells = msmt.cluster_shells(g[:, 3])
    for with_dirs in (True, False):
        out = str(tmp_path / f"resp{int(with_dirs)}.txt")
        args = ["manual", p["dwi"], p["mask"], out, "-lmax", "0,2,4,6"] + (["-dirs", p["dirs"]] if with_dirs else [])
        assert run(args) == 0
        got = np.loadtxt(out)
        assert got.shape == (4, 4)
        if with_dirs:
            fd = f
        else:
            B = bmatrix(g)
            fd = np.zeros((len(dwi), 3))
            for i in np.nonzero(mask)[0]:
                pr = TREF.fit(dwi[i].astype(np.float64), B)
                fd[i] = TREF.principal(pr[:6]) * TREF.fa(pr[:6])
        for s, (vols, L) in enumerate(zip(shells, (0, 2, 4, 6))):
            da = msmt.direction_matrix(g, vols)
            cart = np.stack([np.cos(da[:, 0]) * np.sin(da[:, 1]), np.sin(da[:, 0]) * np.sin(da[:, 1]),
                             np.cos(da[:, 1])], 1)
            M, b = AREF.accumulate(dwi, fd, mask, cart, vols, L)
            want = AREF.fit(M, b, L)
            assert np.abs(got[s, :len(want)] - want).max() <= 1e-6 * np.abs(want).max(), s


def _phantom(tmp_path, dims=(12, 10, 6), seed=5):
    """Single-shell data (6 b=0 + 60 directions at b=3000) of 1-3 fibres with
    the zonal response synth.RESPONSE (lmax 8), SNR 50, all voxels in the mask."""
    rng = np.random.default_rng(seed)
    grad = synth.grad_table(6, synth.fibonacci_hemisphere(60))
    n = int(np.prod(dims))
    dwi = synth.voxel_signals(rng, grad, n, 50.0)
    nx, ny, nz = dims
    p = {"dwi": str(tmp_path / "dwi.mif"), "mask": str(tmp_path / "mask.mif"), "vox": str(tmp_path / "vox.mif")}
    data = dwi.reshape(nz, ny, nx, -1).transpose(2, 1, 0, 3)
    mif.write(p["dwi"], mif.Image(data=data, vox=[2.0, 2.0, 2.0, 1.0],
                                  keyval={"dw_scheme": mif.scheme_to_text(grad)}))
    mif.write(p["mask"], mif.Image(data=np.ones(dims, np.float32), vox=[2.0, 2.0, 2.0]), datatype="UInt8")
    return grad, dwi, p


@pytest.mark.parametrize("algo,extra", [("tournier", ["-number", "60", "-iter_voxels", "240"]),
                                        ("tax", ["-max_iters", "8"])])
def test_dwi2response_iterative(cuda, tmp_path, algo, extra):
    from mrtrix3_b200.dwi2response import run
    grad, dwi, p = _phantom(tmp_path)
    out = str(tmp_path / "resp.txt")
    assert run([algo, p["dwi"], out, "-mask", p["mask"], "-voxels", p["vox"], "-lmax", "8"] + extra) == 0
    got = np.atleast_2d(np.loadtxt(out))
    assert got.shape == (1, 5)
    # the single-fibre response the data were made with, to a tenth of its l = 0 term
    assert np.abs(got[0] - synth.RESPONSE).max() <= 0.1 * synth.RESPONSE[0], got
    vox = mif.read(p["vox"]).data != 0
    assert vox.sum() >= (60 if algo == "tournier" else 20)


@pytest.mark.parametrize("algo", ["tournier", "tax"])
def test_dwi2response_iterative_matches_oracle(cuda, algo):
    """The whole loop on the GPU steps against the same loop on the FP64 CPU
    restatements of CSD, FMLS and amp2response (oracle/dwi2response_ref.py):
    the same iterations, the same single-fibre voxels, responses to 1e-4 of
    the l = 0 term."""
    import torch

    from mrtrix3_b200 import dwi2response as D
    from oracle import dwi2response_ref as R
    rng = np.random.default_rng(5)
    grad = synth.grad_table(6, synth.fibonacci_hemisphere(60))
    dims, n = (5, 4, 3), 60
    dwi = synth.voxel_signals(rng, grad, n, 50.0)
    g = msmt.normalise_scheme(grad)
    shells = msmt.cluster_shells(g[:, 3])
    mask = np.ones(n, bool)
    if algo == "tournier":
        opt, kw = {"-lmax": "8", "-number": "10", "-iter_voxels": "30"}, dict(number=10, iter_voxels=30)
    else:
        opt, kw = {"-lmax": "8", "-max_iters": "4"}, dict(max_iters=4)
    rf, sf, it = D.iterative(algo, opt, g, shells, torch.from_numpy(dwi).cuda(), mask, dims)
    vols = shells[-1]
    rr, sr, ir = R.iterative_ref(algo, g[vols], dwi[:, vols], mask, dims, synth.load_hr_dirs(), lmax=8, **kw)
    assert it == ir
    np.testing.assert_array_equal(sf, sr)
    assert np.abs(rf - rr).max() <= 1e-4 * abs(rr[0]), (rf, rr)
