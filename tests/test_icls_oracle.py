"""The FP64 ICLS restatement (oracle/icls_ref.py) against the reference's own
golden vectors (testing/cmd/testing_unit_tests_icls.cpp, solutions from
Matlab's quadprog; fixture tests/golden/icls_golden.npz), with the
reference's acceptance test isApprox(x, solution, 1e-6).  CPU only."""
import os

import numpy as np
import pytest

from oracle import icls_ref as R

G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "icls_golden.npz"))


def _solve(P):
    x, niter = R.solve(P, G["problem_vector"])
    assert niter <= P.max_niter
    return x


def test_ineq_and_eq_with_vectors():
    P = R.Problem.with_equalities(G["problem_matrix"], G["inequality_constraint_matrix"],
                                  G["equality_constraint_matrix"], G["inequality_constraint_vector"],
                                  G["equality_constraint_vector"])
    assert R.is_approx(_solve(P), G["solution"], 1e-6)


def test_ineq_and_eq_zero_vectors():
    P = R.Problem.with_equalities(G["problem_matrix"], G["inequality_constraint_matrix"],
                                  G["equality_constraint_matrix"])
    assert R.is_approx(_solve(P), G["solution_zero"], 1e-6)


def test_ineq_with_vector():
    P = R.Problem(G["problem_matrix"], G["inequality_constraint_matrix"], G["inequality_constraint_vector"])
    assert R.is_approx(_solve(P), G["solution_no_eq"], 1e-6)


def test_ineq_zero_vector():
    P = R.Problem(G["problem_matrix"], G["inequality_constraint_matrix"])
    assert R.is_approx(_solve(P), G["solution_no_eq_zero"], 1e-6)


def test_stacked_constraints_with_num_eq():
    A = np.vstack([G["inequality_constraint_matrix"], G["equality_constraint_matrix"]])
    t = np.concatenate([G["inequality_constraint_vector"], G["equality_constraint_vector"]])
    P = R.Problem(G["problem_matrix"], A, t, num_eq=10)
    assert R.is_approx(_solve(P), G["solution"], 1e-6)


def test_kkt_of_the_solution():
    """Independent of the golden data: the solution satisfies the
    optimality conditions of min ||Hx - b||^2 s.t. A x >= t."""
    H, A, t, b = G["problem_matrix"], G["inequality_constraint_matrix"], G["inequality_constraint_vector"], \
        G["problem_vector"]
    P = R.Problem(H, A, t)
    x = _solve(P)
    r = A @ x - t
    assert r.min() > -1e-9
    act = np.nonzero(r < 1e-8)[0]
    # stationarity: H^T (H x - b) = A_act^T mu with mu >= 0
    g = H.T @ (H @ x - b)
    mu, *_ = np.linalg.lstsq(A[act].T, g, rcond=None)
    assert np.linalg.norm(A[act].T @ mu - g) < 1e-8 * max(1.0, np.linalg.norm(g))
    assert mu.min() > -1e-8


def test_unconstrained_when_feasible():
    rng = np.random.default_rng(0)
    H = rng.normal(size=(40, 10))
    b = rng.normal(size=40)
    x_ls = np.linalg.lstsq(H, b, rcond=None)[0]
    A = np.eye(10)
    t = x_ls - 1.0  # every constraint slack at the least-squares solution
    x, niter = R.solve(R.Problem(H, A, t), b)
    assert niter == 0
    np.testing.assert_allclose(x, x_ls, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_nonnegative_least_squares_matches_scipy(seed):
    from scipy.optimize import nnls
    rng = np.random.default_rng(seed)
    H = rng.normal(size=(60, 20))
    b = rng.normal(size=60)
    x, _ = R.solve(R.Problem(H, np.eye(20)), b)
    ref, _ = nnls(H, b)
    np.testing.assert_allclose(x, ref, atol=1e-9)


def test_c_restatement_matches_python():
    """oracle/icls_oracle.c (the CPU baseline) against the numpy restatement:
    the golden problem and non-negative least squares, several threads."""
    P = R.Problem.with_equalities(G["problem_matrix"], G["inequality_constraint_matrix"],
                                  G["equality_constraint_matrix"], G["inequality_constraint_vector"],
                                  G["equality_constraint_vector"])
    x, it = R.solve_batch_c(P, G["problem_vector"][None, :], nthreads=1)
    assert R.is_approx(x[0], G["solution"], 1e-6)
    rng = np.random.default_rng(4)
    H = rng.normal(size=(60, 20))
    Q = R.Problem(H, np.eye(20))
    b = rng.normal(size=(40, 60))
    xc, itc = R.solve_batch_c(Q, b, nthreads=4)
    for i in range(len(b)):
        xp, itp = R.solve(Q, b[i])
        np.testing.assert_allclose(xc[i], xp, atol=1e-10)
        assert itc[i] == itp
