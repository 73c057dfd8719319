"""Regenerates tessellation_1281.txt and tessellation_1281_adjacency.txt.

The 1281 [azimuth, elevation] directions of fod2fixel's FMLS segmenter
(MRtrix3 src/dwi/directions/predefined.cpp, tesselation_1281_data; accessor
predefined.h:67) are data the segmentation depends on bit for bit, so they
are shipped verbatim as text (decimal literals copied unchanged).  The table
is MPL-2.0 licensed by the MRtrix3 contributors; see the header line of the
generated file.  The adjacency file holds, per direction, its neighbours on
the convex hull of the directions and their antipodes, as
mrtrix3_b200.directions.hull_adjacency computes them (a restatement of
Set::initialise_adjacency, src/dwi/directions/set.cpp:83-318), so that
programs read it instead of rebuilding the hull.

Usage: python extract_tessellation_1281.py [path-to-mrtrix3-tree]
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    src = open(os.path.join(ref, "src/dwi/directions/predefined.cpp")).read()
    start = src.index("tesselation_1281_data[] = {")
    body = src[start:src.index("};", start)]
    vals = re.findall(r"-?\d+\.\d+(?:[eE]-?\d+)?|-?\d+(?:[eE]-?\d+)?", body.split("{", 1)[1])
    assert len(vals) == 2 * 1281, len(vals)
    out = os.path.join(HERE, "tessellation_1281.txt")
    with open(out, "w") as f:
        f.write("# 1281 tessellation directions [azimuth elevation] (radians).\n")
        f.write("# From MRtrix3 src/dwi/directions/predefined.cpp (MPL-2.0, (c) the MRtrix3 contributors).\n")
        for i in range(1281):
            f.write(f"{vals[2*i]} {vals[2*i+1]}\n")
    print("wrote", out)
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from mrtrix3_b200 import directions
    adj = directions.hull_adjacency(directions.unit_vectors(directions.load_tessellation_1281()))
    out2 = os.path.join(HERE, "tessellation_1281_adjacency.txt")
    with open(out2, "w") as f:
        f.write("# neighbours of each of the 1281 tessellation directions (0-based, ascending), one line each\n")
        for a in adj:
            f.write(" ".join(str(int(j)) for j in a) + "\n")
    print("wrote", out2)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MRTRIX_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <MRtrix3 source tree>  (or set MRTRIX_REF)")
    main(root)
