"""amp2response on the GPU (csd_amp2response_accumulate + the ICLS solver in
standard form, mrtrix3_b200/amp2response.py) against the FP64 restatement
(oracle/amp2response_ref.py): the accumulated normal equations to 1e-10,
the fitted response to 1e-7 of its largest coefficient; single-fibre voxels
made from a known response give it back; the command line on .mif files."""
import numpy as np
import pytest

from mrtrix3_b200 import amp2response as AR
from mrtrix3_b200 import mif, msmt, synth
from oracle import amp2response_ref as REF

pytestmark = pytest.mark.gpu

RESP = np.array([1700.0, -700.0, 240.0, -60.0, 10.0])


def _voxels(n, grad, seed, noise=0.0):
    rng = np.random.default_rng(seed)
    f = rng.normal(size=(n, 3))
    f /= np.linalg.norm(f, axis=1, keepdims=True)
    g = grad[:, :3]
    cos = np.abs(f @ g.T)
    els = np.arccos(np.clip(cos, -1, 1))
    T = np.stack([REF._zonal(e, 8) for e in els])  # [n][vol][5]
    amp = T @ RESP
    dw = grad[:, 3] > 10.0
    amp[:, ~dw] = RESP[0] * 0.282094791773878
    amp = amp + noise * rng.normal(size=amp.shape)
    return amp.astype(np.float32), (f * rng.uniform(0.5, 2.0, (n, 1))).astype(np.float32)


@pytest.mark.parametrize("lmax,constrained", [(8, True), (10, True), (10, False), (0, True)])
def test_amp2response_matches_oracle(cuda, lmax, constrained):
    import torch
    grad = synth.config5_scheme()
    dwi_vols = np.nonzero(grad[:, 3] > 10.0)[0]
    amp, f = _voxels(500, grad, 3, noise=20.0)
    mask = (np.arange(500) % 4 != 0).astype(np.uint8)
    d = grad[dwi_vols, :3] / np.linalg.norm(grad[dwi_vols, :3], axis=1, keepdims=True)
    M, b = AR.accumulate(torch.from_numpy(amp).to(cuda), torch.from_numpy(f).to(cuda), d, dwi_vols, lmax,
                         torch.from_numpy(mask).to(cuda))
    Mr, br = REF.accumulate(amp, f, mask, d, dwi_vols, lmax)
    Mg = M.cpu().numpy()
    assert np.abs(np.tril(Mg) - np.tril(Mr)).max() <= 1e-10 * np.abs(Mr).max()
    assert np.abs(b.cpu().numpy() - br).max() <= 1e-10 * np.abs(br).max()
    rf = AR.fit(M, b, lmax, constrained)
    rr = REF.fit(Mr, br, lmax, constrained)
    assert np.abs(rf - rr).max() <= 1e-7 * np.abs(rr).max()


def test_amp2response_recovers_a_known_response(cuda):
    import torch
    grad = synth.config5_scheme()
    dwi_vols = np.nonzero(grad[:, 3] > 10.0)[0]
    amp, f = _voxels(300, grad, 4)
    d = grad[dwi_vols, :3] / np.linalg.norm(grad[dwi_vols, :3], axis=1, keepdims=True)
    M, b = AR.accumulate(torch.from_numpy(amp).to(cuda), torch.from_numpy(f).to(cuda), d, dwi_vols, 8)
    rf = AR.fit(M, b, 8, constrained=True)
    np.testing.assert_allclose(rf, RESP, atol=1e-3)


def test_amp2response_command_line(cuda, tmp_path):
    grad = synth.config5_scheme()
    dims = (6, 5, 4)
    n = int(np.prod(dims))
    amp, f = _voxels(n, grad, 5, noise=10.0)
    mask = np.ones(n, np.uint8)
    mask[::3] = 0

    def vol(x):
        return x.reshape(dims[2], dims[1], dims[0], -1).transpose(2, 1, 0, 3)
    pa, pm, pd, out = (str(tmp_path / k) for k in ("amp.mif", "mask.mif", "dir.mif", "resp.txt"))
    mif.write(pa, mif.Image(data=vol(amp), vox=[2.0] * 4, keyval={"dw_scheme": mif.scheme_to_text(grad)}))
    mif.write(pm, mif.Image(data=vol(mask)[..., 0].astype(np.float64), vox=[2.0] * 3), datatype="UInt8")
    mif.write(pd, mif.Image(data=vol(f), vox=[2.0] * 4))
    assert AR.run([pa, pm, pd, out, "-lmax", "0,8"]) == 0
    got = np.loadtxt(out)
    assert got.shape == (2, 5)
    g = msmt.normalise_scheme(grad)
    shells = msmt.cluster_shells(g[:, 3])
    rows = []
    for vols, L in zip(shells, (0, 8)):
        da = msmt.direction_matrix(g, vols)
        cart = np.stack([np.cos(da[:, 0]) * np.sin(da[:, 1]), np.sin(da[:, 0]) * np.sin(da[:, 1]),
                         np.cos(da[:, 1])], axis=1)
        Mr, br = REF.accumulate(amp, f, mask, cart, vols, L)
        r = REF.fit(Mr, br, L)
        rows.append(np.pad(r, (0, 5 - len(r))))
    np.testing.assert_allclose(got, np.array(rows), rtol=1e-7, atol=1e-7 * np.abs(rows[1]).max())
    with pytest.raises(SystemExit, match="does not match number of b-value shells"):
        AR.run([pa, pm, pd, out, "-lmax", "8", "-force"])
