"""Extracts the ICLS solver's golden vectors from the reference's unit test
(testing/cmd/testing_unit_tests_icls.cpp: a 100 x 50 problem with 290
inequality and 10 equality constraints and four solutions computed with
Matlab's quadprog) into tests/golden/icls_golden.npz.

    python tests/golden/make_icls_golden.py [reference root]

The arrays are read as text; the matrices are stored column-major there
(Eigen::Map of a plain array) and are saved here in numpy (row-major) order.
"""
import os
import re
import sys

import numpy as np

SIZES = {"num_sig": 100, "num_coef": 50, "num_ineq": 290, "num_eq": 10}
SHAPES = {
    "problem_matrix": ("num_sig", "num_coef"),
    "inequality_constraint_matrix": ("num_ineq", "num_coef"),
    "equality_constraint_matrix": ("num_eq", "num_coef"),
    "problem_vector": ("num_sig",),
    "inequality_constraint_vector": ("num_ineq",),
    "equality_constraint_vector": ("num_eq",),
    "solution": ("num_coef",),
    "solution_no_eq": ("num_coef",),
    "solution_zero": ("num_coef",),
    "solution_no_eq_zero": ("num_coef",),
}


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MRTRIX_REF")
    if not root:
        sys.exit("usage: python make_icls_golden.py <MRtrix3 source tree>  (or set MRTRIX_REF)")
    src = open(os.path.join(root, "testing", "cmd", "testing_unit_tests_icls.cpp")).read()
    for k, v in SIZES.items():
        m = re.search(r"const size_t %s = (\d+);" % k, src)
        assert m and int(m.group(1)) == v, k
    out = {}
    for name, shape in SHAPES.items():
        m = re.search(r"double %s_data\[\] = \{([^}]*)\};" % name, src)
        assert m, name
        vals = np.array([float(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()], np.float64)
        dims = tuple(SIZES[d] for d in shape)
        assert vals.size == int(np.prod(dims)), (name, vals.size, dims)
        out[name] = vals.reshape(dims, order="F")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "icls_golden.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}")


if __name__ == "__main__":
    main()
