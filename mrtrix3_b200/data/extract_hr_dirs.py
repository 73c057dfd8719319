"""Regenerates electrostatic_repulsion_300.txt from an MRtrix3 source tree.

The 300 [azimuth, elevation] constraint directions that CSD projects onto
(MRtrix3 src/dwi/directions/predefined.cpp:92-393, accessor predefined.h:51)
are data the results depend on bit for bit, so they are shipped verbatim as
text (the decimal literals are copied unchanged, so strtod on either side
yields the same doubles).  The table is MPL-2.0 licensed by the MRtrix3
contributors; see the header line of the generated file.

Usage: python extract_hr_dirs.py [path-to-mrtrix3-tree]
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    src = open(os.path.join(ref, "src/dwi/directions/predefined.cpp")).read()
    start = src.index("electrostatic_repulsion_300_data[] = {")
    body = src[start:src.index("};", start)]
    vals = re.findall(r"-?\d+\.\d+(?:[eE]-?\d+)?|-?\d+(?:[eE]-?\d+)?", body.split("{", 1)[1])
    assert len(vals) == 600, len(vals)
    out = os.path.join(HERE, "electrostatic_repulsion_300.txt")
    with open(out, "w") as f:
        f.write("# 300 electrostatic-repulsion directions [azimuth elevation] (radians).\n")
        f.write("# From MRtrix3 src/dwi/directions/predefined.cpp (MPL-2.0, (c) the MRtrix3 contributors).\n")
        for i in range(300):
            f.write(f"{vals[2*i]} {vals[2*i+1]}\n")
    print("wrote", out)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MRTRIX_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <MRtrix3 source tree>  (or set MRTRIX_REF)")
    main(root)
