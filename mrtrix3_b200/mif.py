"""MRtrix image files (.mif, .mif.gz, .mih + data) and text matrices.

The format (docs/getting_started/image_data.rst:355-470 of MRtrix3): a text
header opening with ``mrtrix image`` and closing with ``END``, one
``key: value`` per line in between (a key may repeat; its lines accumulate,
as ``read_mrtrix_header`` does in core/formats/mrtrix_utils.h:60-136), then
the binary data.  Required keys: ``dim``, ``vox``, ``layout``, ``datatype``,
``file``; optional: ``transform`` (three rows of four), ``scaling``
(offset, scale).  ``layout`` gives, per axis, the sign of its stride and
its rank from fastest (0) to slowest; a negative stride stores the axis
reversed.  Everything else (``dw_scheme`` among it) is kept as text.

An image is held as a numpy array in axis order (x, y, z, ...): voxel
[i, j, k] is ``data[i, j, k]``, whatever the order on file.
"""
from __future__ import annotations

import dataclasses
import gzip
import io
import os
import re

import numpy as np

_TYPES = {
    "int8": ("i1", None), "uint8": ("u1", None),
    "int16": ("i2", "="), "uint16": ("u2", "="), "int32": ("i4", "="), "uint32": ("u4", "="),
    "int64": ("i8", "="), "uint64": ("u8", "="), "float32": ("f4", "="), "float64": ("f8", "="),
}


def _dtype(spec: str):
    """numpy dtype of an MRtrix datatype specifier (case-insensitive); None for Bit."""
    s = spec.strip().lower()
    if s == "bit":
        return None
    order = "="
    if s.endswith("le"):
        order, s = "<", s[:-2]
    elif s.endswith("be"):
        order, s = ">", s[:-2]
    if s not in _TYPES:
        raise ValueError(f"unsupported MRtrix datatype \"{spec}\"")
    code, _ = _TYPES[s]
    return np.dtype(code if code.endswith("1") else order + code)


def _spec(dt: np.dtype) -> str:
    names = {"i1": "Int8", "u1": "UInt8", "i2": "Int16", "u2": "UInt16", "i4": "Int32", "u4": "UInt32",
             "i8": "Int64", "u8": "UInt64", "f4": "Float32", "f8": "Float64"}
    dt = np.dtype(dt)
    base = names[dt.kind + str(dt.itemsize)]
    if dt.itemsize == 1:
        return base
    little = dt.byteorder == "<" or (dt.byteorder in "=|" and np.little_endian)
    return base + ("LE" if little else "BE")


@dataclasses.dataclass
class Image:
    data: np.ndarray                      # axis order x, y, z, ...
    vox: list                             # voxel sizes, one per axis
    transform: np.ndarray | None = None   # 3 x 4 (scanner space)
    keyval: dict = dataclasses.field(default_factory=dict)  # other keys: name -> text (lines joined by "\n")
    layout: list | None = None            # as read: signed stride rank per axis ("+0" fastest)
    datatype: str = "Float32LE"

    @property
    def dim(self):
        return list(self.data.shape)


def _parse_layout(value: str, ndim: int):
    items = [v.strip() for v in value.split(",")]
    if len(items) != ndim:
        raise ValueError("layout does not match the image dimensions")
    out = []
    for it in items:
        m = re.fullmatch(r"([+-]?)(\d+)", it)
        if not m:
            raise ValueError(f"invalid layout entry \"{it}\"")
        out.append((-1 if m.group(1) == "-" else 1, int(m.group(2))))
    ranks = sorted(r for _, r in out)
    if ranks != list(range(ndim)):
        raise ValueError("layout ranks must be a permutation of 0..ndim-1")
    return out


def _read_header(f):
    first = f.readline().decode("latin-1").strip()
    if first != "mrtrix image":
        raise ValueError("not an MRtrix image (first line is not \"mrtrix image\")")
    keys: dict[str, list[str]] = {}
    order: list[str] = []
    while True:
        line = f.readline()
        if not line:
            raise ValueError("MRtrix header ended without END")
        line = line.decode("latin-1").rstrip("\r\n")
        if line.strip() == "END":
            break
        if not line.strip():
            continue
        if ":" not in line:
            raise ValueError(f"malformed MRtrix header line \"{line}\"")
        k, v = line.split(":", 1)
        k, v = k.strip(), v.strip()
        if not k or not v:
            continue
        if k not in keys:
            keys[k] = []
            order.append(k)
        keys[k].append(v)
    return keys, order


def read(path: str) -> Image:
    """Load a .mif / .mif.gz / .mih image (voxel values scaled by ``scaling``)."""
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rb") as fh:
        raw = fh.read()
    f = io.BytesIO(raw)
    keys, order = _read_header(f)
    lk = {k.lower(): k for k in keys}

    def req(name):
        if name not in lk:
            raise ValueError(f"missing \"{name}\" specification for MRtrix image \"{path}\"")
        return keys[lk[name]]

    dim = [int(v) for v in req("dim")[0].split(",")]
    if any(d < 1 for d in dim):
        raise ValueError(f"invalid dimensions for MRtrix image \"{path}\"")
    vox = [float(v) for v in req("vox")[0].split(",")]
    if len(vox) < min(3, len(dim)):
        raise ValueError(f"too few entries in \"vox\" specification for MRtrix image \"{path}\"")
    layout = _parse_layout(req("layout")[0], len(dim))
    dtspec = req("datatype")[0]
    dt = _dtype(dtspec)
    # data location(s)
    chunks = []
    for entry in req("file"):
        parts = entry.rsplit(None, 1)
        name, offset = (parts[0], int(parts[1])) if len(parts) == 2 else (parts[0], 0)
        if name == ".":
            chunks.append(raw[offset:])
        else:
            dpath = os.path.join(os.path.dirname(path), name)
            with (gzip.open if dpath.endswith(".gz") else open)(dpath, "rb") as dh:
                dh.seek(offset)
                chunks.append(dh.read())
    blob = b"".join(chunks)
    n = int(np.prod(dim))
    if dt is None:  # Bit: most significant bit first within each byte (core/raw.h)
        bits = np.unpackbits(np.frombuffer(blob, np.uint8, count=(n + 7) // 8), bitorder="big")[:n]
        flat = bits.astype(bool)
    else:
        flat = np.frombuffer(blob, dt, count=n)
    # on file the fastest axis is the one of rank 0: reshape slowest-first, then
    # transpose to x, y, z, ... and reverse the axes stored with negative strides
    axes_fast_to_slow = sorted(range(len(dim)), key=lambda a: layout[a][1])
    arr = flat.reshape([dim[a] for a in reversed(axes_fast_to_slow)])
    arr = np.transpose(arr, [list(reversed(axes_fast_to_slow)).index(a) for a in range(len(dim))])
    for a, (sign, _) in enumerate(layout):
        if sign < 0:
            arr = np.flip(arr, axis=a)
    arr = np.ascontiguousarray(arr)
    if "scaling" in lk:
        off, scale = (float(v) for v in keys[lk["scaling"]][0].split(","))
        if off != 0.0 or scale != 1.0:
            arr = off + scale * arr.astype(np.float64)
    transform = None
    if "transform" in lk:
        rows = [[float(v) for v in r.split(",")] for r in keys[lk["transform"]]]
        if len(rows) < 3 or any(len(r) != 4 for r in rows[:3]):
            raise ValueError(f"invalid \"transform\" specification for MRtrix image \"{path}\"")
        transform = np.array(rows[:3], np.float64)
    skip = {"dim", "vox", "layout", "datatype", "file", "transform", "scaling"}
    kv = {k: "\n".join(keys[k]) for k in order if k.lower() not in skip}
    return Image(data=arr, vox=vox[:len(dim)], transform=transform, keyval=kv,
                 layout=[s * (r + 1) for s, r in layout], datatype=dtspec)


def write(path: str, img: Image, layout=None, datatype: str | None = None):
    """Write a .mif (or .mif.gz) image.  ``layout``: signed 1-based stride
    ranks per axis (e.g. [+2, +3, +4, +1] stores axis 3 fastest); default:
    the image's own, else x fastest.  ``datatype``: an MRtrix specifier
    (default Float32 in native byte order)."""
    data = np.asarray(img.data)
    nd = data.ndim
    if layout is None:
        layout = img.layout if img.layout and len(img.layout) == nd else list(range(1, nd + 1))
    if sorted(abs(s) for s in layout) != list(range(1, nd + 1)):
        raise ValueError("layout must rank the axes 1..ndim with signs")
    dt = _dtype(datatype) if datatype else np.dtype("=f4")
    if dt is None:
        raise ValueError("writing Bit images is not supported")
    spec = datatype if datatype else _spec(np.dtype("=f4"))
    arr = data
    for a, s in enumerate(layout):
        if s < 0:
            arr = np.flip(arr, axis=a)
    fast_to_slow = sorted(range(nd), key=lambda a: abs(layout[a]))
    arr = np.transpose(arr, list(reversed(fast_to_slow)))
    payload = np.ascontiguousarray(arr.astype(dt)).tobytes()
    lines = ["mrtrix image", "dim: " + ",".join(str(d) for d in data.shape),
             "vox: " + ",".join(repr(float(v)) for v in (list(img.vox) + [1.0] * nd)[:nd]),
             "layout: " + ",".join(("+" if s > 0 else "-") + str(abs(s) - 1) for s in layout),
             "datatype: " + spec]
    if img.transform is not None:
        for r in np.asarray(img.transform)[:3]:
            lines.append("transform: " + ",".join(repr(float(v)) for v in r))
    for k, v in img.keyval.items():
        for line in str(v).split("\n"):
            lines.append(f"{k}: {line}")
    head = "\n".join(lines) + "\nfile: . "
    # the offset is written in the header itself: grow it until it fits, and
    # align the data to 16 bytes
    offset = len(head) + 16
    while True:
        text = head + str(offset) + "\nEND\n"
        if len(text) <= offset:
            break
        offset = len(text) + 16
    offset = (offset + 15) // 16 * 16
    text = (head + str(offset) + "\nEND\n").encode("latin-1")
    text = text + b"\0" * (offset - len(text))
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "wb") as fh:
        fh.write(text)
        fh.write(payload)


def load_matrix(path: str) -> np.ndarray:
    """Delimited numeric text (core/math/math.h:148-205): '#' starts a comment,
    entries separated by spaces, commas, semicolons or tabs; rows must agree."""
    rows = []
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            rows.append([float(v) for v in re.split(r"[ ,;\t]+", line) if v])
    if not rows:
        raise ValueError(f"no data in file \"{path}\"")
    if any(len(r) != len(rows[0]) for r in rows):
        raise ValueError(f"rows of different length in file \"{path}\"")
    return np.array(rows, np.float64)


def load_vector(path: str) -> np.ndarray:
    """A single row or column (core/math/math.h:325-334)."""
    m = load_matrix(path)
    if m.shape[1] == 1:
        return m[:, 0]
    if m.shape[0] > 1:
        raise ValueError(f"file \"{path}\" contains matrix, not vector")
    return m[0]


def scheme_to_text(grad: np.ndarray) -> str:
    """A gradient table as header text: one "x,y,z,b" row per line."""
    return "\n".join(",".join(repr(float(v)) for v in row) for row in np.asarray(grad))


def parse_scheme(text: str) -> np.ndarray:
    return np.array([[float(v) for v in re.split(r"[ ,;\t]+", line.strip()) if v]
                     for line in text.split("\n") if line.strip()], np.float64)


def load_bvecs_bvals(bvecs_path: str, bvals_path: str, transform=None, n_volumes: int | None = None) -> np.ndarray:
    """An FSL bvecs / bvals pair as an [n][4] gradient table in scanner
    space (DWI::load_bvecs_bvals, core/dwi/gradient.cpp:127-200): bvals one
    row (or column), bvecs three rows (or columns), both one entry a volume;
    the bvecs are in the image axes of a left-handed frame, so the first is
    negated when the transform's 3x3 part has a positive determinant, then
    rotated by that part; rows with NaN become b=0 rows (a NaN bval with a
    valid direction, or a NaN direction with b > 0, is an error)."""
    try:
        bvals = load_matrix(bvals_path)
        bvecs = load_matrix(bvecs_path)
    except (OSError, ValueError) as e:
        raise ValueError(f"Unable to import files \"{bvecs_path}\" and \"{bvals_path}\" as FSL bvecs/bvals pair "
                         f"({e})")
    if bvals.shape[0] != 1:
        if bvals.shape[1] == 1:
            bvals = bvals.T
        else:
            raise ValueError(f"bvals file must contain 1 row or column only (file \"{bvals_path}\" has "
                             f"{bvals.shape[0]})")
    if bvecs.shape[0] != 3:
        if bvecs.shape[1] == 3:
            bvecs = bvecs.T
        else:
            raise ValueError(f"bvecs file must contain exactly 3 rows or columns (file \"{bvecs_path}\" has "
                             f"{bvecs.shape[0]})")
    if bvals.shape[1] != bvecs.shape[1]:
        raise ValueError("bvecs and bvals files must have same number of diffusion directions")
    if n_volumes is not None and bvals.shape[1] != n_volumes:
        raise ValueError(f"bvecs and bvals files must have same number of diffusion directions as DW-image "
                         f"(gradients: {bvecs.shape[1]}, image: {n_volumes})")
    R = np.eye(3) if transform is None else np.asarray(transform, np.float64)[:3, :3]
    bvecs = bvecs.copy()
    if np.linalg.det(R) > 0.0:
        bvecs[0] *= -1.0
    grad = np.zeros((bvecs.shape[1], 4))
    grad[:, :3] = (R @ bvecs).T
    grad[:, 3] = bvals[0]
    for n in range(len(grad)):
        zero = False
        if np.isnan(grad[n, 3]):
            if np.sum(grad[n, :3] ** 2) > 0.0:
                raise ValueError("Corrupt content in bvecs/bvals data (NaN present in bval but valid direction in "
                                 "bvec)")
            zero = True
        if np.isnan(grad[n, :3]).any():
            if grad[n, 3] > 0.0:
                raise ValueError("Corrupt content in bvecs/bvals data (NaN bvec direction but non-zero value in "
                                 "bval)")
            zero = True
        if zero:
            grad[n] = 0.0
    return grad


def dw_scheme(img: Image, opt: dict) -> np.ndarray:
    """The gradient table of a DW image (DWI::get_raw_DW_scheme,
    gradient.cpp:250-273): -grad file, -fslgrad (bvecs, bvals), else the
    header's dw_scheme."""
    if "-grad" in opt and "-fslgrad" in opt:
        raise ValueError("Diffusion gradient table can be provided using either -grad or -fslgrad option, but NOT "
                         "both")
    if "-grad" in opt:
        return load_matrix(opt["-grad"])
    if "-fslgrad" in opt:
        bvecs, bvals = opt["-fslgrad"]
        return load_bvecs_bvals(bvecs, bvals, img.transform, img.data.shape[3] if img.data.ndim > 3 else 1)
    if "dw_scheme" in img.keyval:
        return parse_scheme(img.keyval["dw_scheme"])
    raise ValueError("no diffusion encoding information found in image")
