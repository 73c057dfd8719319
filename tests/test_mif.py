"""MRtrix image files and text matrices (mrtrix3_b200/mif.py) on the CPU:
round trips over layouts / datatypes / compression, images written by hand
from the format's documented rules (docs/getting_started/image_data.rst:
355-470), the Bit datatype's bit order (core/raw.h:27, 176), separate
header / data files, and the delimited text loader."""
import gzip

import numpy as np
import pytest

from mrtrix3_b200 import mif
from mrtrix3_b200.dwi2fod import output_layout, run


@pytest.mark.parametrize("layout", [[1, 2, 3, 4], [-1, 3, 2, 4], [4, 3, 2, 1], [2, -4, 1, -3]])
@pytest.mark.parametrize("dtype", ["Float32LE", "Float32BE", "Float64LE", "Int16LE", "UInt8"])
@pytest.mark.parametrize("ext", [".mif", ".mif.gz"])
def test_round_trip(tmp_path, layout, dtype, ext):
    rng = np.random.default_rng(len(dtype) + sum(layout))
    if dtype.startswith("Float"):
        data = rng.normal(size=(5, 4, 3, 7))
    else:
        data = rng.integers(0, 100, size=(5, 4, 3, 7)).astype(np.float64)
    grad = np.c_[rng.normal(size=(7, 3)), rng.integers(0, 3000, size=7)]
    img = mif.Image(data=data, vox=[1.5, 2.0, 2.5, float("nan")],
                    transform=np.arange(12, dtype=float).reshape(3, 4),
                    keyval={"dw_scheme": mif.scheme_to_text(grad), "comments": "first\nsecond"})
    p = str(tmp_path / ("x" + ext))
    mif.write(p, img, layout=layout, datatype=dtype)
    back = mif.read(p)
    assert back.data.shape == data.shape
    np.testing.assert_allclose(back.data, data.astype(mif._dtype(dtype)), rtol=0, atol=0)
    assert back.layout == layout
    assert back.vox[:3] == [1.5, 2.0, 2.5]
    np.testing.assert_array_equal(back.transform, img.transform)
    np.testing.assert_array_equal(mif.parse_scheme(back.keyval["dw_scheme"]), grad)
    assert back.keyval["comments"] == "first\nsecond"


def _hand_written(body: bytes, header_lines, path):
    head = "mrtrix image\n" + "".join(l + "\n" for l in header_lines)
    off = len(head) + len("file: . 000\nEND\n")
    head += f"file: . {off:03d}\nEND\n"
    assert len(head) == off
    with open(path, "wb") as f:
        f.write(head.encode() + body)


def test_documented_layout_and_scaling(tmp_path):
    # dim 3 x 2, y fastest ("+1,+0" ranks x second), x stored right to left:
    # file order is (x=2,y=0) (x=2,y=1) (x=1,y=0) ... ; values = offset + scale * raw
    raw = np.array([20, 21, 10, 11, 0, 1], np.int16)
    p = tmp_path / "h.mif"
    _hand_written(raw.astype("<i2").tobytes(),
                  ["dim: 3,2", "vox: 1,1", "layout: -1,+0", "datatype: Int16LE", "scaling: 5,2",
                   "MyKey: a", "MyKey: b"], p)
    img = mif.read(str(p))
    expect = 5 + 2 * np.array([[0, 1], [10, 11], [20, 21]], np.float64)
    np.testing.assert_array_equal(img.data, expect)
    assert img.keyval["MyKey"] == "a\nb"


def test_bit_datatype_msb_first(tmp_path):
    bits = np.array([1, 0, 0, 0, 0, 0, 0, 1, 1, 1], bool)  # 10 voxels, x fastest
    packed = np.packbits(bits, bitorder="big").tobytes()
    p = tmp_path / "m.mif"
    _hand_written(packed, ["dim: 10", "vox: 1", "layout: +0", "datatype: Bit"], p)
    np.testing.assert_array_equal(mif.read(str(p)).data, bits)


def test_separate_header_and_data(tmp_path):
    data = np.arange(24, dtype="<f4").reshape(2, 3, 4)   # x slowest on file: layout +2,+1,+0
    (tmp_path / "d.dat").write_bytes(b"\0" * 8 + data.tobytes())
    (tmp_path / "d.mih").write_text("mrtrix image\ndim: 2,3,4\nvox: 1,1,1\nlayout: +2,+1,+0\n"
                                    "datatype: Float32LE\nfile: d.dat 8\nEND\n")
    np.testing.assert_array_equal(mif.read(str(tmp_path / "d.mih")).data, data)


def test_gz_hand_written(tmp_path):
    p = tmp_path / "g.mif"
    _hand_written(np.array([1.5, -2.0], "<f8").tobytes(), ["dim: 2", "vox: 3", "layout: +0", "datatype: Float64LE"], p)
    gz = tmp_path / "g.mif.gz"
    gz.write_bytes(gzip.compress(p.read_bytes()))
    np.testing.assert_array_equal(mif.read(str(gz)).data, [1.5, -2.0])


@pytest.mark.parametrize("header,msg", [
    ("mrtrix image\nvox: 1\nlayout: +0\ndatatype: Float32\nfile: . 0\nEND\n", "dim"),
    ("mrtrix image\ndim: 2\nlayout: +0\ndatatype: Float32\nfile: . 0\nEND\n", "vox"),
    ("mrtrix image\ndim: 2\nvox: 1\nlayout: +0\ndatatype: CFloat32\nfile: . 0\nEND\n", "datatype"),
    ("not an image\n", "mrtrix image"),
])
def test_header_errors(tmp_path, header, msg):
    p = tmp_path / "bad.mif"
    p.write_bytes(header.encode())
    with pytest.raises(ValueError, match=msg):
        mif.read(str(p))


def test_text_matrices(tmp_path):
    p = tmp_path / "r.txt"
    p.write_text("# response\n1700, -700;240\t-60 10  # trailing\n")
    np.testing.assert_array_equal(mif.load_vector(str(p)), [1700, -700, 240, -60, 10])
    p.write_text("1\n2\n3\n")
    np.testing.assert_array_equal(mif.load_vector(str(p)), [1, 2, 3])
    p.write_text("1 2\n3 4\n")
    with pytest.raises(ValueError, match="matrix, not vector"):
        mif.load_vector(str(p))
    p.write_text("1 2\n3\n")
    with pytest.raises(ValueError):
        mif.load_matrix(str(p))


def test_output_layout_keeps_spatial_order():
    assert output_layout([1, 2, 3, 4], 4) == [2, 3, 4, 1]
    assert output_layout([-1, 3, 2, 4], 4) == [-2, 4, 3, 1]
    assert output_layout([4, 3, 2, 1], 4) == [4, 3, 2, 1]


def test_cli_rejects_other_algorithms_and_arguments():
    with pytest.raises(SystemExit, match="usage"):
        run(["sdeconv", "a", "b", "c"])
    with pytest.raises(SystemExit, match="pairs"):
        run(["msmt_csd", "a", "b", "c", "d"])
    with pytest.raises(SystemExit, match="single input response"):
        run(["csd", "a", "b"])
    with pytest.raises(SystemExit, match="unknown option"):
        run(["csd", "a", "b", "c", "-bogus"])


def test_fsl_bvecs_bvals_import(tmp_path):
    """DWI::load_bvecs_bvals (core/dwi/gradient.cpp:127-200): rows or
    columns, the first axis negated for a transform with positive
    determinant, rotation into scanner space, NaN rows as b=0, errors."""
    bvecs = np.array([[1.0, 0.0, 0.0, np.nan], [0.0, 1.0, 0.0, np.nan], [0.0, 0.0, 1.0, np.nan]])
    bvals = np.array([1000.0, 2000.0, 3000.0, 0.0])
    pv, pb = str(tmp_path / "bvecs"), str(tmp_path / "bvals")
    np.savetxt(pv, bvecs)
    np.savetxt(pb, bvals[None, :])
    # identity transform (det 1 > 0): x negated
    g = mif.load_bvecs_bvals(pv, pb, np.eye(4)[:3], 4)
    np.testing.assert_allclose(g[:3], [[-1, 0, 0, 1000], [0, 1, 0, 2000], [0, 0, 1, 3000]])
    np.testing.assert_array_equal(g[3], 0.0)
    # a transform with negative determinant (x flipped): no negation, rotation applied
    T = np.diag([-1.0, 1.0, 1.0, 1.0])[:3]
    g2 = mif.load_bvecs_bvals(pv, pb, T, 4)
    np.testing.assert_allclose(g2[:3, :3], [[-1, 0, 0], [0, 1, 0], [0, 0, 1]])
    # a rotation of 90 degrees about z (det 1): x negated, then rotated
    Rz = np.array([[0.0, -1.0, 0.0, 5.0], [1.0, 0.0, 0.0, 6.0], [0.0, 0.0, 1.0, 7.0]])
    g3 = mif.load_bvecs_bvals(pv, pb, Rz, 4)
    np.testing.assert_allclose(g3[0, :3], Rz[:, :3] @ [-1.0, 0.0, 0.0])
    # column layout accepted; size checks
    np.savetxt(pv, bvecs.T)
    np.savetxt(pb, bvals[:, None])
    np.testing.assert_allclose(mif.load_bvecs_bvals(pv, pb, np.eye(4)[:3], 4), g)
    with pytest.raises(ValueError, match="same number of diffusion directions as DW-image"):
        mif.load_bvecs_bvals(pv, pb, None, 5)
    # a NaN bval with a valid direction is corrupt
    bv = bvals.copy()
    bv[0] = np.nan
    np.savetxt(pb, bv[None, :])
    with pytest.raises(ValueError, match="NaN present in bval"):
        mif.load_bvecs_bvals(pv, pb, None, 4)
    # the CLI helper: -grad and -fslgrad together are refused
    img = mif.Image(data=np.zeros((2, 2, 2, 4)), vox=[1.0] * 4, transform=np.eye(4)[:3])
    with pytest.raises(ValueError, match="NOT both"):
        mif.dw_scheme(img, {"-grad": "g.txt", "-fslgrad": (pv, pb)})
