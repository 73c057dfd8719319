"""``dwi2fod csd`` on MRtrix image files (mrtrix3_b200/dwi2fod.py) on the
GPU: a synthetic DW image stored with reversed / permuted axes and int16 +
scaling, a mask, a response file; the FOD image equals the library's
host-buffer result voxel for voxel, sits on the FP64 oracle, and carries
the reference's output header (float32, SH axis contiguous, gradient table
moved to prior_dw_scheme, phase-encoding keys dropped)."""
import numpy as np
import pytest

from mrtrix3_b200 import csd, mif, synth
from mrtrix3_b200.dwi2fod import run
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_dwi2fod_csd_on_mif_files(cuda, hr_dirs, tmp_path):
    dims = (14, 11, 9)
    v = synth.make_volume(dims, 6, 60, (15.0, 40.0), 8, 0.6, 4242)
    # volume layout of make_volume: voxel index = x + X (y + Y z) -> array [x, y, z, vol]
    data = v.dwi.reshape(dims[2], dims[1], dims[0], -1).transpose(2, 1, 0, 3)
    mask = v.mask.reshape(dims[2], dims[1], dims[0]).transpose(2, 1, 0)
    scale = 0.25
    raw = np.round(data / scale)
    kv = {"dw_scheme": mif.scheme_to_text(v.grad), "pe_scheme": "0,1,0,0.05", "TotalReadoutTime": "0.05",
          "command_history": "synthetic"}
    p_dwi, p_mask = str(tmp_path / "dwi.mif"), str(tmp_path / "mask.mif")
    # int16 on file with the intensity scaling in the header (value = 0 + scale * stored)
    img = mif.Image(data=raw, vox=[2.0, 2.0, 2.0, 1.0], transform=np.eye(4)[:3],
                    keyval={**kv, "scaling": f"0,{scale}"})
    mif.write(p_dwi, img, layout=[-2, 3, 4, 1], datatype="Int16LE")
    mif.write(p_mask, mif.Image(data=mask.astype(np.float64), vox=[2.0, 2.0, 2.0]), datatype="UInt8")
    resp = tmp_path / "response.txt"
    resp.write_text(" ".join(str(c) for c in synth.RESPONSE) + "\n")
    out_path = str(tmp_path / "fod.mif")
    assert run(["csd", p_dwi, str(resp), out_path, "-mask", p_mask, "-lmax", "8"]) == 0
    fod = mif.read(out_path)
    assert fod.data.shape == dims + (45,)
    assert fod.layout[3] == 1 and fod.datatype.startswith("Float32")
    assert "dw_scheme" not in fod.keyval and "pe_scheme" not in fod.keyval and "TotalReadoutTime" not in fod.keyval
    np.testing.assert_allclose(mif.parse_scheme(fod.keyval["prior_dw_scheme"]), v.grad)
    assert fod.keyval["command_history"] == "synthetic"
    # the same signals through the library directly (voxel order x fastest)
    s = csd.make_shared(v.grad, synth.RESPONSE, lmax=8)
    sig = (np.round(data / scale) * scale).astype(np.float32)
    flat = np.ascontiguousarray(sig.transpose(2, 1, 0, 3).reshape(-1, 66))
    direct = csd.dwi2fod_csd_host_phased(s, flat, v.mask)
    got = fod.data.transpose(2, 1, 0, 3).reshape(-1, 45)
    np.testing.assert_array_equal(got, direct["fod"])
    assert not got[v.mask == 0].any()
    idx = np.nonzero(v.mask)[0][:400]
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(flat[idx].astype(np.float64))
    rel = np.abs(got[idx] - ref["F"]).max(1) / np.abs(ref["F"]).max(1)
    assert np.percentile(rel, 99) <= 1e-4
    with pytest.raises(SystemExit, match="already exists"):
        run(["csd", p_dwi, str(resp), out_path])


def test_dwi2fod_csd_shells_option(cuda, hr_dirs, tmp_path):
    """-shells on a two-shell image: the csd branch deconvolves the chosen
    shell only (csd.h:64), so the FODs equal the oracle's on the image cut
    down to the b=0 volumes and that shell."""
    d1, d3 = synth.fibonacci_hemisphere(60), synth.fibonacci_hemisphere(45)
    grad = np.array([[0, 0, 0, 0]] * 6 + [[*d, 1000.0] for d in d1] + [[*d, 3000.0] for d in d3], np.float64)
    grad = grad[np.random.default_rng(8).permutation(len(grad))]
    dims = (9, 8, 7)
    n = int(np.prod(dims))
    sig = synth.voxel_signals(np.random.default_rng(9), grad, n, 30.0)
    data = sig.reshape(dims[2], dims[1], dims[0], -1).transpose(2, 1, 0, 3)
    p_dwi = str(tmp_path / "dwi.mif")
    mif.write(p_dwi, mif.Image(data=data.astype(np.float64), vox=[2.0, 2.0, 2.0, 1.0], transform=np.eye(4)[:3],
                               keyval={"dw_scheme": mif.scheme_to_text(grad)}), datatype="Float32LE")
    resp = tmp_path / "response.txt"
    resp.write_text(" ".join(str(c) for c in synth.RESPONSE) + "\n")
    for b in (1000.0, 3000.0):
        out_path = str(tmp_path / f"fod{int(b)}.mif")
        assert run(["csd", p_dwi, str(resp), out_path, "-shells", str(int(b))]) == 0
        got = mif.read(out_path).data.transpose(2, 1, 0, 3).reshape(-1, 45)
        keep = np.nonzero((grad[:, 3] == 0) | (grad[:, 3] == b))[0]
        ref = O.OracleShared(grad[keep], synth.RESPONSE, hr_dirs).solve(sig[:, keep].astype(np.float64))
        rel = np.abs(got - ref["F"]).max(1) / np.abs(ref["F"]).max(1)
        assert np.percentile(rel, 99) <= 1e-4, (b, np.percentile(rel, 99))
    with pytest.raises(SystemExit, match="2 non b=0 shells"):
        run(["csd", p_dwi, str(resp), str(tmp_path / "x.mif"), "-shells", "1000,3000"])
