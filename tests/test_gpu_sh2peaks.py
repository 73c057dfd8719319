"""GPU sh2peaks (csd_sh2peaks, mrtrix3_b200/sh2peaks.py) against the FP64
restatement of cmd/sh2peaks.cpp + SH::get_peak (oracle/sh2peaks_ref.py):
FODs of a synthetic volume from the library's own CSD, the reference's 60
seeds, the number of peaks and their order identical on >= 99% of voxels,
directions within 2e-3 rad and amplitudes within 1e-3 relative; the edge
cases of check_input (masked, NaN, isotropic), the threshold, target
directions, per-voxel target peaks, more requested peaks than found, and
custom seeds; the command line on .mif files."""
import numpy as np
import pytest

from mrtrix3_b200 import csd, mif, synth
from oracle import sh2peaks_ref as S

pytestmark = pytest.mark.gpu


def _fods(n, seed, lmax=8):
    import torch
    v = synth.make_volume((n, 1, 1), 6, 60, (15.0, 40.0), lmax, None, seed)
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=lmax)
    return csd.dwi2fod_csd(s, torch.from_numpy(v.dwi).cuda())["fod"]


def _compare(got, ref):
    ref = np.asarray(ref).reshape(len(got), -1)
    ok_count = np.all(np.isnan(got[:, 0::3]) == np.isnan(ref[:, 0::3]), axis=1)
    both = ~np.isnan(ref[:, 0::3])
    a_g = np.linalg.norm(got.reshape(len(got), -1, 3), axis=2)
    a_r = np.linalg.norm(ref.reshape(len(ref), -1, 3), axis=2)
    with np.errstate(invalid="ignore"):
        cosang = np.abs(np.sum(got.reshape(len(got), -1, 3) * ref.reshape(len(ref), -1, 3), axis=2)) / (a_g * a_r)
        same = np.where(both, (np.arccos(np.clip(cosang, -1, 1)) < 2e-3) & (np.abs(a_g - a_r) <= 1e-3 * a_r), True)
    return ok_count & np.all(same, axis=1)


@pytest.mark.parametrize("lmax", [6, 8, 10])
def test_peaks_match_oracle(cuda, lmax):
    fod = _fods(300, 70 + lmax, lmax)
    seeds = csd.default_peak_seeds()
    got = csd.sh2peaks(fod, npeaks=3).cpu().numpy()
    f = fod.cpu().numpy().astype(np.float64)
    ref = np.stack([S.voxel_peaks(f[i], lmax, seeds, npeaks=3) for i in range(len(f))])
    assert _compare(got, ref).mean() >= 0.99
    assert np.isfinite(got[:, :3]).all()  # every voxel has at least one peak


def test_edge_cases_threshold_and_targets(cuda):
    import torch
    fod = _fods(64, 5)
    f = fod.clone()
    f[0, 3] = float("nan")           # non-finite input
    f[1, 1:] = 0.0                   # isotropic: no peaks
    mask = torch.ones(64, dtype=torch.uint8, device=f.device)
    mask[2] = 0                      # outside the mask
    seeds = csd.default_peak_seeds()
    got = csd.sh2peaks(f, mask=mask, npeaks=5, threshold=0.05).cpu().numpy()
    assert np.isnan(got[:3]).all()
    fh = f.cpu().numpy().astype(np.float64)
    ref = np.stack([S.voxel_peaks(fh[i], 8, seeds, npeaks=5, threshold=0.05) for i in range(3, 64)])
    assert _compare(got[3:], ref).mean() >= 0.98
    assert np.isnan(got[3:, 12:]).any()  # fewer than 5 peaks above the threshold somewhere
    # -direction: the peak closest to each given direction
    dirs = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0]])
    got = csd.sh2peaks(fod, directions=dirs).cpu().numpy()
    fo = fod.cpu().numpy().astype(np.float64)
    ref = np.stack([S.voxel_peaks(fo[i], 8, seeds, npeaks=2, targets=dirs) for i in range(64)])
    assert _compare(got, ref).mean() >= 0.98
    # -peaks: per-voxel targets (this run's own peaks in reverse order)
    first = csd.sh2peaks(fod, npeaks=2)
    targets = torch.cat([first[:, 3:6], first[:, 0:3]], dim=1).contiguous()
    got = csd.sh2peaks(fod, peaks=targets).cpu().numpy()
    t = targets.cpu().numpy().astype(np.float64)
    ref = np.stack([S.voxel_peaks(fo[i], 8, seeds, npeaks=2, targets=t[i].reshape(2, 3))
                    if np.isfinite(t[i, 0]) else np.full((2, 3), np.nan) for i in range(64)])
    assert _compare(got, ref.reshape(64, 6)).mean() >= 0.98
    # custom seeds
    rng = np.random.default_rng(1)
    my = np.c_[rng.uniform(-np.pi, np.pi, 20), np.arccos(rng.uniform(-1, 1, 20))].astype(np.float32)
    got = csd.sh2peaks(fod, seeds=my).cpu().numpy()
    ref = np.stack([S.voxel_peaks(fo[i], 8, my, npeaks=3) for i in range(64)])
    assert _compare(got, ref).mean() >= 0.98


def test_sh2peaks_command_line(cuda, tmp_path):
    from mrtrix3_b200.sh2peaks import run
    fod = _fods(60, 9).cpu().numpy()
    data = fod.reshape(5, 4, 3, 45)
    p_in, p_out = str(tmp_path / "fod.mif"), str(tmp_path / "peaks.mif")
    mif.write(p_in, mif.Image(data=data, vox=[2.0, 2.0, 2.0, float("nan")]), layout=[2, 3, 4, 1])
    assert run([p_in, p_out, "-num", "2", "-force"]) == 0
    out = mif.read(p_out)
    assert out.data.shape == (5, 4, 3, 6)
    import torch
    direct = csd.sh2peaks(torch.from_numpy(np.ascontiguousarray(data.reshape(-1, 45))).cuda(), npeaks=2)
    np.testing.assert_array_equal(out.data.reshape(-1, 6), direct.cpu().numpy())
    assert run([p_in, p_out, "-direction", "0", "0", "-force"]) == 0
    assert mif.read(p_out).data.shape == (5, 4, 3, 3)
