"""Regenerates sh2peaks_seeds_60.txt from an MRtrix3 source tree.

The 60 [azimuth, elevation] seed directions from which sh2peaks starts its
Newton searches (MRtrix3 cmd/sh2peaks.cpp, ``default_directions``) decide
which peaks are found, so they are shipped verbatim as text (the decimal
literals copied unchanged; the reference holds them as float).  MPL-2.0
licensed by the MRtrix3 contributors; see the header line of the file.

Usage: python extract_sh2peaks_seeds.py [path-to-mrtrix3-tree]
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    src = open(os.path.join(ref, "cmd/sh2peaks.cpp")).read()
    start = src.index("default_directions [] = {")
    body = src[start:src.index("};", start)].split("{", 1)[1]
    vals = re.findall(r"-?\d+\.\d+(?:[eE]-?\d+)?|-?\d+(?:[eE]-?\d+)?", body)
    assert len(vals) == 120, len(vals)
    out = os.path.join(HERE, "sh2peaks_seeds_60.txt")
    with open(out, "w") as f:
        f.write("# 60 sh2peaks seed directions [azimuth elevation] (radians).\n")
        f.write("# From MRtrix3 cmd/sh2peaks.cpp (MPL-2.0, (c) the MRtrix3 contributors).\n")
        for i in range(60):
            f.write(f"{vals[2*i]} {vals[2*i+1]}\n")
    print("wrote", out)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MRTRIX_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <MRtrix3 source tree>  (or set MRTRIX_REF)")
    main(root)
