"""amp2sh on the GPU (csd_amp2sh through mrtrix3_b200.csd.amp2sh and the
``python -m mrtrix3_b200.amp2sh`` command line) against an FP64 numpy
restatement of cmd/amp2sh.cpp:153-171: c = pinv(SH2amp) a, a = the selected
volumes' amplitudes, scaled by nb0 / (1 + sum of the b=0 amplitudes) with
-normalise.  The kernel computes in FP64 and stores float32, so the bound is
float32 rounding of the result: |got - ref| <= 1e-6 (|ref| + max |ref| of the
voxel)."""
import numpy as np
import pytest

from mrtrix3_b200 import csd, mif, sh, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _ref(amp, fit, dwis, bzeros, normalise):
    a = amp.astype(np.float64)
    norm = np.ones(len(a))
    if normalise:
        norm = len(bzeros) / (1.0 + a[:, bzeros].sum(1))
    return (a[:, dwis] * norm[:, None]) @ fit.T


def _check(got, ref):
    scale = np.abs(ref).max(1, keepdims=True)
    assert np.all(np.abs(got - ref) <= 1e-6 * (np.abs(ref) + scale) + 1e-30)


def _fit(grad, lmax=8):
    shared = csd.Shared(grad)
    shared.set_response(np.array([1.0, -0.5]))
    shared.init()
    dwis = np.asarray(shared.dwis)
    dirs = sh.cartesian_to_azel(grad[dwis, :3])
    # the fit from the oracle's transform, independently of the host set-up
    fit = np.linalg.pinv(O.init_transform(dirs, lmax))
    bzeros = np.nonzero(grad[:, 3] <= 10.0)[0]
    return fit, dwis, bzeros


@pytest.mark.parametrize("normalise", [False, True])
def test_amp2sh_matches_fp64_fit(cuda, normalise):
    import torch
    grad = synth.config5_scheme()
    fit, dwis, bzeros = _fit(grad)
    assert len(dwis) == 60 and len(bzeros) == 6
    n = 20011  # not a multiple of the 32-voxel tile
    amp = synth.voxel_signals(np.random.default_rng(7), grad, n, (15.0, 40.0)).astype(np.float32)
    got = csd.amp2sh(torch.from_numpy(amp).to(cuda), fit, dwis, bzeros, normalise=normalise)
    torch.cuda.synchronize()
    _check(got.cpu().numpy().astype(np.float64), _ref(amp, fit, dwis, bzeros, normalise))


def test_amp2sh_volume_major_input_and_round_trip(cuda):
    import torch
    grad = synth.config5_scheme()
    fit, dwis, bzeros = _fit(grad)
    m = O.init_transform(sh.cartesian_to_azel(grad[dwis, :3]), 8)
    rng = np.random.default_rng(11)
    n = 4099
    c0 = rng.normal(size=(n, 45))
    amp = np.zeros((n, grad.shape[0]), np.float32)
    amp[:, dwis] = (c0 @ m.T).astype(np.float32)
    amp[:, bzeros] = rng.uniform(0.5, 2.0, (n, len(bzeros)))
    # volume-major storage: voxel stride 1, volume stride n
    vm = torch.from_numpy(np.ascontiguousarray(amp.T)).to(cuda).t()
    assert vm.stride() == (1, n)
    got = csd.amp2sh(vm, fit, dwis, bzeros).cpu().numpy().astype(np.float64)
    _check(got, _ref(amp, fit, dwis, bzeros, False))
    # amplitudes of a known SH function give it back (to float32 input rounding)
    assert np.max(np.abs(got - c0)) <= 1e-5 * np.abs(c0).max()
    # a plan reused, writing into the first 45 columns of a wider output
    plan = csd.Amp2SHCommon(fit, dwis, bzeros, normalise=True)
    wide = torch.full((n, 64), 7.0, dtype=torch.float32, device=cuda)
    for _ in range(2):
        plan(vm, wide)
    w = wide.cpu().numpy()
    _check(w[:, :45].astype(np.float64), _ref(amp, fit, dwis, bzeros, True))
    assert (w[:, 45:] == 7.0).all()
    with pytest.raises(ValueError):
        plan(vm[:, :60])


def test_amp2sh_edge_cases(cuda):
    import torch
    grad = synth.config5_scheme()
    fit, dwis, bzeros = _fit(grad, lmax=4)
    empty = torch.zeros((0, grad.shape[0]), dtype=torch.float32, device=cuda)
    assert csd.amp2sh(empty, fit, dwis, bzeros).shape == (0, 15)
    one = torch.ones((1, grad.shape[0]), dtype=torch.float32, device=cuda)
    got = csd.amp2sh(one, fit, dwis, bzeros).cpu().numpy()
    _check(got.astype(np.float64), _ref(np.ones((1, grad.shape[0])), fit, dwis, bzeros, False))
    with pytest.raises(ValueError):
        csd.amp2sh(one, fit, np.append(dwis[:-1], grad.shape[0]), bzeros)
    with pytest.raises(ValueError):
        csd.amp2sh(one, fit[:, :-1], dwis, bzeros)
    with pytest.raises(csd.CSDError):
        csd.amp2sh(one, fit, dwis, None, normalise=True)


def test_amp2sh_command_line(cuda, tmp_path):
    from mrtrix3_b200.amp2sh import run
    grad = synth.config5_scheme()
    dims = (7, 5, 3)
    n = int(np.prod(dims))
    amp = synth.voxel_signals(np.random.default_rng(5), grad, n, (15.0, 40.0)).astype(np.float32)
    data = amp.reshape(dims[2], dims[1], dims[0], -1).transpose(2, 1, 0, 3)
    p = str(tmp_path / "dwi.mif")
    kv = {"dw_scheme": mif.scheme_to_text(grad), "pe_scheme": "0,1,0,0.05"}
    mif.write(p, mif.Image(data=data, vox=[2.0, 2.0, 2.0, 1.0], transform=np.eye(4)[:3], keyval=kv),
              layout=[-2, 3, 4, 1])
    out = str(tmp_path / "sh.mif")
    assert run([p, out, "-normalise"]) == 0
    img = mif.read(out)
    assert img.data.shape == dims + (45,) and img.datatype.startswith("Float32")
    assert img.layout == [-2, 3, 4, 1]
    assert "dw_scheme" not in img.keyval and "pe_scheme" not in img.keyval
    np.testing.assert_allclose(mif.parse_scheme(img.keyval["prior_dw_scheme"]), grad)
    fit, dwis, bzeros = _fit(grad)
    got = img.data.transpose(2, 1, 0, 3).reshape(n, -1).astype(np.float64)
    _check(got, _ref(amp, fit, dwis, bzeros, True))
    # -lmax and a header "directions" key (moved to basis_directions)
    dirs = sh.cartesian_to_azel(grad[dwis, :3])
    p2 = str(tmp_path / "amp.mif")
    kv2 = {"directions": "\n".join(f"{float(a)!r},{float(e)!r}" for a, e in dirs)}
    mif.write(p2, mif.Image(data=data[..., dwis], vox=[2.0, 2.0, 2.0, 1.0], keyval=kv2))
    out2 = str(tmp_path / "sh6.mif")
    assert run([p2, out2, "-lmax", "6"]) == 0
    img2 = mif.read(out2)
    assert img2.data.shape == dims + (28,)
    assert "directions" not in img2.keyval and "basis_directions" in img2.keyval
    fit6 = np.linalg.pinv(O.init_transform(dirs, 6))
    got2 = img2.data.transpose(2, 1, 0, 3).reshape(n, -1).astype(np.float64)
    _check(got2, _ref(amp[:, dwis], fit6, np.arange(60), [], False))


@pytest.fixture
def amp2sh_kernel():
    from mrtrix3_b200 import autotune

    def use(kind):
        autotune.set_knob(autotune.KNOB_AMP2SH_KIND, kind)
    yield use
    use(0)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
@pytest.mark.parametrize("ndir,lmax", [(30, 4), (59, 4), (60, 8), (64, 8), (90, 10), (300, 12), (300, 16), (800, 8)])
def test_amp2sh_fit_shapes(cuda, amp2sh_kernel, ndir, lmax, kind):
    """Every kernel (1 row, 2 tile, 3 FP64 tensor cores, 0 the automatic
    choice; a kernel that does not apply falls back to one that does) on odd
    direction counts (padded k-steps), one to three column groups of 32 in
    the tile kernel, the tensor-core limits (64 directions, lmax 8) and fits
    too large for shared memory (300 directions at lmax 12 / 16)."""
    import torch
    amp2sh_kernel(kind)
    rng = np.random.default_rng(ndir + lmax)
    dirs = np.stack([rng.uniform(0, 2 * np.pi, ndir), np.arccos(rng.uniform(-1, 1, ndir))], axis=1)
    fit = np.linalg.pinv(O.init_transform(dirs, lmax))
    nvol = ndir + 5
    perm = rng.permutation(nvol)
    dwis, bzeros = np.sort(perm[:ndir]), np.sort(perm[ndir:])
    n = 3001
    amp = rng.uniform(0.0, 2.0, (n, nvol)).astype(np.float32)
    d = torch.from_numpy(amp).to(cuda)
    for normalise in (False, True):
        got = csd.amp2sh(d, fit, dwis, bzeros, normalise=normalise).cpu().numpy().astype(np.float64)
        _check(got, _ref(amp, fit, dwis, bzeros, normalise))


@pytest.mark.parametrize("kind", [0, 2])
def test_amp2sh_row_layouts(cuda, amp2sh_kernel, kind):
    """Voxel rows padded beyond the volumes (voxel stride 70 for 66 volumes),
    rows that start off a 16-byte boundary (a column slice), and a voxel
    stride above what the tensor-core kernel stages whole (300): all give the
    fit of the selected volumes."""
    import torch
    amp2sh_kernel(kind)
    grad = synth.config5_scheme()
    fit, dwis, bzeros = _fit(grad)
    rng = np.random.default_rng(17)
    n = 5003
    for width, first in ((70, 0), (70, 1), (300, 3)):
        wide = rng.uniform(0.1, 2.0, (n, width)).astype(np.float32)
        d = torch.from_numpy(wide).to(cuda)[:, first:first + grad.shape[0]]
        assert d.stride() == (width, 1)
        amp = wide[:, first:first + grad.shape[0]]
        for normalise in (False, True):
            got = csd.amp2sh(d, fit, dwis, bzeros, normalise=normalise).cpu().numpy().astype(np.float64)
            _check(got, _ref(amp, fit, dwis, bzeros, normalise))


@pytest.mark.parametrize("normalise", [False, True])
def test_amp2sh_rician_matches_oracle(cuda, normalise):
    """-rician: the reweighted fit against the FP64 restatement
    (oracle/amp2sh_ref.py); a noise level of ~SNR 20 a voxel."""
    import torch
    from oracle import amp2sh_ref
    grad = synth.config5_scheme()
    fit, dwis, bzeros = _fit(grad)
    m = O.init_transform(sh.cartesian_to_azel(grad[dwis, :3]), 8)
    rng = np.random.default_rng(13)
    n = 1003
    amp = synth.voxel_signals(rng, grad, n, (15.0, 40.0)).astype(np.float32)
    noise = (amp[:, bzeros].mean(1) / rng.uniform(10.0, 30.0, n)).astype(np.float32)
    if normalise:
        noise = noise * (len(bzeros) / (1.0 + amp[:, bzeros].sum(1))).astype(np.float32)
    plan = csd.Amp2SHCommon(fit, dwis, bzeros, normalise=normalise, sh2amp=m)
    got = plan(torch.from_numpy(amp).to(cuda), noise=torch.from_numpy(noise).to(cuda)).cpu().numpy()
    plain = plan(torch.from_numpy(amp).to(cuda)).cpu().numpy()
    for i in range(0, n, 17):
        a = amp2sh_ref.amps(amp[i], dwis, bzeros, normalise)
        ref = amp2sh_ref.fit_rician(a, m, fit, float(noise[i]))
        assert np.abs(got[i] - ref).max() <= 1e-5 * np.abs(ref).max()
    # the correction changes the fit (it is not the plain one)
    assert np.abs(got - plain).max() > 1e-3 * np.abs(plain).max()


def test_amp2sh_rician_command_line(cuda, tmp_path):
    from mrtrix3_b200.amp2sh import run
    from oracle import amp2sh_ref
    grad = synth.config5_scheme()
    dims = (5, 4, 3)
    n = int(np.prod(dims))
    rng = np.random.default_rng(6)
    amp = synth.voxel_signals(rng, grad, n, (15.0, 40.0)).astype(np.float32)
    noise = np.full(n, 60.0, np.float32)
    data = amp.reshape(dims[2], dims[1], dims[0], -1).transpose(2, 1, 0, 3)
    p, pn, out = str(tmp_path / "dwi.mif"), str(tmp_path / "noise.mif"), str(tmp_path / "sh.mif")
    mif.write(p, mif.Image(data=data, vox=[2.0, 2.0, 2.0, 1.0], keyval={"dw_scheme": mif.scheme_to_text(grad)}))
    mif.write(pn, mif.Image(data=noise.reshape(dims[2], dims[1], dims[0]).transpose(2, 1, 0),
                            vox=[2.0, 2.0, 2.0]))
    assert run([p, out, "-rician", pn]) == 0
    got = mif.read(out).data.transpose(2, 1, 0, 3).reshape(n, -1).astype(np.float64)
    fit, dwis, bzeros = _fit(grad)
    m = O.init_transform(sh.cartesian_to_azel(grad[dwis, :3]), 8)
    for i in range(0, n, 7):
        ref = amp2sh_ref.fit_rician(amp2sh_ref.amps(amp[i], dwis), m, fit, 60.0)
        assert np.abs(got[i] - ref).max() <= 1e-5 * np.abs(ref).max()
