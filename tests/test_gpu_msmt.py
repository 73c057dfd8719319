"""The batched GPU ICLS solver (csd_icls_create / csd_icls_solve) and
multi-shell multi-tissue CSD on it, against the reference's golden ICLS
vectors (testing/cmd/testing_unit_tests_icls.cpp, with its isApprox 1e-6
test) and the FP64 restatements (oracle/icls_ref.py, oracle/msmt_ref.py).
Outputs are float32: tolerances are relative to the voxel's largest
parameter, 1e-5 (p99) and 1e-4 (max)."""
import os

import numpy as np
import pytest

from mrtrix3_b200 import msmt, synth
from oracle import icls_ref, msmt_ref

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "icls_golden.npz"))
RESP = [synth.MSMT_RESPONSES["wm"], synth.MSMT_RESPONSES["gm"], synth.MSMT_RESPONSES["csf"]]


def _rows(cuda, b, n):
    import torch
    return torch.from_numpy(np.tile(np.asarray(b, np.float32), (n, 1))).to(cuda)


@pytest.mark.parametrize("case", ["eq_t", "eq_zero", "ineq_t", "ineq_zero", "stacked"])
def test_icls_golden_vectors(cuda, case):
    G = GOLD
    H, Ai, Ae = G["problem_matrix"], G["inequality_constraint_matrix"], G["equality_constraint_matrix"]
    ti, te = G["inequality_constraint_vector"], G["equality_constraint_vector"]
    if case == "eq_t":
        P, want = msmt.ICLSProblem(H, np.vstack([Ai, Ae]), np.concatenate([ti, te]), num_eq=10), G["solution"]
    elif case == "eq_zero":
        P, want = msmt.ICLSProblem(H, np.vstack([Ai, Ae]), None, num_eq=10), G["solution_zero"]
    elif case == "ineq_t":
        P, want = msmt.ICLSProblem(H, Ai, ti), G["solution_no_eq"]
    elif case == "ineq_zero":
        P, want = msmt.ICLSProblem(H, Ai), G["solution_no_eq_zero"]
    else:
        A = np.vstack([Ai, Ae])
        P, want = msmt.ICLSProblem(H, A, np.concatenate([ti, te]), num_eq=10), G["solution"]
    # the problem vector is stored in float32 for the device: compare with the
    # oracle on the same rounded vector, and with the golden solution
    b32 = G["problem_vector"].astype(np.float32)
    x, it = P.solve(_rows(cuda, b32, 37))
    x = x.cpu().numpy().astype(np.float64)
    it = it.cpu().numpy()
    assert (it >= 0).all() and (it == it[0]).all()
    for row in x:
        assert icls_ref.is_approx(row, want, 1e-5)  # float32 b and x: the golden 1e-6 holds in FP64 (CPU test)
    ref = icls_ref.Problem(H, np.vstack([Ai, Ae]) if case in ("eq_t", "eq_zero", "stacked") else Ai,
                           None if case in ("eq_zero", "ineq_zero") else
                           (np.concatenate([ti, te]) if case in ("eq_t", "stacked") else ti),
                           num_eq=10 if case in ("eq_t", "eq_zero", "stacked") else 0)
    xr, itr = icls_ref.solve(ref, b32.astype(np.float64))
    assert icls_ref.is_approx(x[0], xr, 1e-6)
    assert it[0] == itr


@pytest.mark.parametrize("seed", [0, 1])
def test_icls_batch_of_different_problems_vectors(cuda, seed):
    """Non-negative least squares, one right-hand side a row."""
    import torch
    rng = np.random.default_rng(seed)
    H = rng.normal(size=(60, 20))
    P = msmt.ICLSProblem(H, np.eye(20))
    ref = icls_ref.Problem(H, np.eye(20))
    b = rng.normal(size=(257, 60)).astype(np.float32)
    x, it = P.solve(torch.from_numpy(b).to(cuda))
    x, it = x.cpu().numpy(), it.cpu().numpy()
    same = 0
    for i in range(len(b)):
        xr, itr = icls_ref.solve(ref, b[i].astype(np.float64))
        assert np.max(np.abs(x[i] - xr)) <= 1e-5 * max(1.0, np.abs(xr).max())
        # with tol = 0 the last round stops on the sign of a multiplier's
        # residual that is zero in exact arithmetic: rounding may add a round
        # that changes nothing
        assert abs(int(it[i]) - int(itr)) <= 1
        same += it[i] == itr
    assert same >= 0.8 * len(b)


def _msmt_case(n, seed):
    s = msmt.MSMTShared(synth.msmt_scheme())
    s.set_responses(RESP)
    s.init()
    P = msmt_ref.problem(s.grad, s.shells, RESP, [8, 0, 0], s.HR_dirs)
    rng = np.random.default_rng(seed)
    truth = synth.msmt_truth(rng, n)
    clean = truth @ P.H.T
    sigma = rng.uniform(1000.0 / 40, 1000.0 / 15, n)
    dwi = synth.rician(rng, clean, sigma).astype(np.float32)
    return s, P, dwi


def _rel(x, r):
    return np.abs(x - r).max(1) / np.maximum(np.abs(r).max(1), 1e-30)


def test_msmt_matches_oracle(cuda):
    import torch
    s, P, dwi = _msmt_case(3000, 21)
    x, it = s.solve(torch.from_numpy(dwi).to(cuda))
    torch.cuda.synchronize()
    x, it = x.cpu().numpy().astype(np.float64), it.cpu().numpy()
    assert x.shape == (3000, 47) and (it >= 1).any()
    idx = np.arange(0, 3000, 10)
    xr, itr = msmt_ref.solve(P, dwi[idx].astype(np.float64))
    rel = _rel(x[idx], xr)
    assert np.percentile(rel, 99) <= 1e-5 and rel.max() <= 1e-4
    assert np.mean(it[idx] == itr) >= 0.9
    assert (it <= s.max_niter()).all()
    wm, gm, csf = s.split(x)
    assert wm.shape[1] == 45 and gm.shape[1] == 1 and csf.shape[1] == 1


def test_msmt_mask_nonfinite_and_layout(cuda):
    import torch
    s, P, dwi = _msmt_case(300, 22)
    dwi[7, 3] = np.nan
    mask = np.ones(300, np.uint8)
    mask[::3] = 0
    # volume-major storage: voxel stride 1, volume stride n
    d = torch.from_numpy(np.ascontiguousarray(dwi.T)).to(cuda).t()
    x, it = s.solve(d, mask=torch.from_numpy(mask).to(cuda))
    x, it = x.cpu().numpy().astype(np.float64), it.cpu().numpy()
    assert not x[mask == 0].any() and (it[mask == 0] == 0).all()
    assert np.isnan(x[7]).all()
    live = np.nonzero(mask)[0]
    live = live[(live != 7)][:60]
    xr, _ = msmt_ref.solve(P, dwi[live].astype(np.float64))
    assert _rel(x[live], xr).max() <= 1e-4


def test_icls_active_sets_beyond_the_shared_memory_rows(cuda):
    """Non-negative least squares whose unconstrained solution is negative
    almost everywhere: 60-80 active constraints, so the factor's rows past
    the 48 kept in shared memory (and the Givens removals across that
    boundary) are exercised."""
    import torch
    rng = np.random.default_rng(9)
    H = rng.normal(size=(150, 80))
    P = msmt.ICLSProblem(H, np.eye(80))
    ref = icls_ref.Problem(H, np.eye(80))
    u = rng.uniform(0.5, 1.5, size=(33, 80))
    u[:, ::7] *= -1.0  # a few coordinates stay free
    b = (-(u @ H.T) + rng.normal(scale=0.05, size=(33, 150))).astype(np.float32)
    x, it = P.solve(torch.from_numpy(b).to(cuda))
    x, it = x.cpu().numpy(), it.cpu().numpy()
    big = 0
    for i in range(len(b)):
        tr = []
        xr, itr = icls_ref.solve(ref, b[i].astype(np.float64), trace=tr)
        big += max(len(t) for t in tr) > 48
        assert np.max(np.abs(x[i] - xr)) <= 1e-5 * max(1.0, np.abs(xr).max())
        assert abs(int(it[i]) - int(itr)) <= 1
    assert big == len(b)


def test_dwi2fod_msmt_csd_command_line(cuda, tmp_path):
    """``dwi2fod msmt_csd`` on .mif files: one output per tissue (float32,
    SH axis contiguous, the gradient table in prior_dw_scheme), equal voxel
    for voxel to the library call, near the oracle; -mask, -lmax and
    -predicted_signal."""
    import torch
    from mrtrix3_b200 import mif
    from mrtrix3_b200.dwi2fod import run
    s, P, dwi = _msmt_case(7 * 6 * 5, 23)
    dims = (7, 6, 5)
    data = dwi.reshape(dims[2], dims[1], dims[0], -1).transpose(2, 1, 0, 3)
    mask = np.ones(dims[::-1], np.uint8)
    mask[0, 0, :] = 0
    p_dwi, p_mask = str(tmp_path / "dwi.mif"), str(tmp_path / "mask.mif")
    mif.write(p_dwi, mif.Image(data=data, vox=[2.0, 2.0, 2.0, 1.0], transform=np.eye(4)[:3],
                               keyval={"dw_scheme": mif.scheme_to_text(s.grad), "pe_scheme": "0,1,0,0.05"}),
              layout=[-2, 3, 4, 1])
    mif.write(p_mask, mif.Image(data=mask.transpose(2, 1, 0).astype(np.float64), vox=[2.0, 2.0, 2.0]),
              datatype="UInt8")
    resp = []
    for k in ("wm", "gm", "csf"):
        f = tmp_path / f"{k}.txt"
        np.savetxt(f, synth.MSMT_RESPONSES[k])
        resp.append(str(f))
    outs = [str(tmp_path / f"{k}.mif") for k in ("wm", "gm", "csf")]
    pred_path = str(tmp_path / "pred.mif")
    args = ["msmt_csd", p_dwi, resp[0], outs[0], resp[1], outs[1], resp[2], outs[2], "-mask", p_mask,
            "-predicted_signal", pred_path]
    assert run(args) == 0
    imgs = [mif.read(o) for o in outs]
    assert [i.data.shape[3] for i in imgs] == [45, 1, 1]
    for i in imgs:
        assert i.layout[3] == 1 and i.datatype.startswith("Float32")
        assert "dw_scheme" not in i.keyval and i.keyval["pe_scheme"] == "0,1,0,0.05"
        np.testing.assert_allclose(mif.parse_scheme(i.keyval["prior_dw_scheme"]), s.grad)
    got = np.concatenate([i.data.transpose(2, 1, 0, 3).reshape(-1, i.data.shape[3]) for i in imgs], axis=1)
    flat_mask = mask.reshape(-1)
    x, _ = s.solve(torch.from_numpy(dwi).to(cuda), mask=torch.from_numpy(flat_mask).to(cuda))
    # the command line re-reads the scheme from the header text and normalises
    # it again: the problem differs from this one's in the last bits only
    xd = x.cpu().numpy()
    assert np.all(np.abs(got - xd) <= 1e-6 * np.abs(xd).max(1, keepdims=True))
    assert not got[flat_mask == 0].any()
    live = np.nonzero(flat_mask)[0][:40]
    xr, _ = msmt_ref.solve(P, dwi[live].astype(np.float64))
    assert _rel(got[live], xr).max() <= 1e-4
    pred = mif.read(pred_path).data.transpose(2, 1, 0, 3).reshape(-1, dwi.shape[1]).astype(np.float64)
    want = xr @ P.H.T
    assert np.abs(pred[live] - want).max() <= 1e-4 * np.abs(want).max()
    assert not pred[flat_mask == 0].any()
    # -lmax per tissue, and the argument rules
    assert run(args[:8] + ["-lmax", "6,0,0", "-force"]) == 0
    assert mif.read(outs[0]).data.shape[3] == 28
    with pytest.raises(SystemExit, match="pairs"):
        run(["msmt_csd", p_dwi, resp[0], outs[0], resp[1]])
    with pytest.raises(SystemExit, match="already exists"):
        run(args[:8])


@pytest.mark.parametrize("tissues,lmax", [(("gm", "csf"), None), (("wm", "gm", "csf"), [10, 0, 0]),
                                          (("wm", "csf"), [6, 0])])
def test_msmt_tissue_sets(cuda, tissues, lmax):
    """Isotropic tissues only (2 parameters, 2 constraints), white matter at
    lmax 10 (its response padded with zeros), two tissues."""
    import torch
    resp = [synth.MSMT_RESPONSES[k] for k in tissues]
    s = msmt.MSMTShared(synth.msmt_scheme())
    if lmax:
        s.parse_cmdline_options(lmax=lmax)
    s.set_responses(resp)
    s.init()
    want_lmax = lmax or [0] * len(tissues)
    assert s.lmax == want_lmax
    pad = [np.pad(r, ((0, 0), (0, max(0, L // 2 + 1 - r.shape[1]))))[:, :L // 2 + 1] for r, L in zip(resp, want_lmax)]
    P = msmt_ref.problem(s.grad, s.shells, pad, want_lmax, s.HR_dirs)
    rng = np.random.default_rng(31)
    truth = synth.msmt_truth(rng, 200)
    cols = {"wm": list(range(45)), "gm": [45], "csf": [46]}
    x_true = np.zeros((200, P.H.shape[1]))
    c0 = 0
    for k, L in zip(tissues, want_lmax):
        n = (L + 1) * (L + 2) // 2
        src = truth[:, cols[k]]
        x_true[:, c0:c0 + min(n, src.shape[1])] = src[:, :n]
        c0 += n
    dwi = synth.rician(rng, x_true @ P.H.T, 30.0).astype(np.float32)
    x, it = s.solve(torch.from_numpy(dwi).to(cuda))
    x = x.cpu().numpy().astype(np.float64)
    idx = np.arange(0, 200, 4)
    xr, itr = msmt_ref.solve(P, dwi[idx].astype(np.float64))
    assert _rel(x[idx], xr).max() <= 1e-4
    assert (it.cpu().numpy() >= 0).all()


def test_msmt_host_buffers_equal_device_call(cuda):
    """csd_icls_solve_host (host arrays, staged through the device) gives the
    device call's results bit for bit, with the mask and predicted signal."""
    import torch
    s, P, dwi = _msmt_case(500, 24)
    mask = (np.arange(500) % 5 != 0).astype(np.uint8)
    x_h, it_h, pred_h = s.solve_host(dwi, mask, predicted=True)
    pred_d = torch.empty((500, dwi.shape[1]), dtype=torch.float32, device=cuda)
    x_d, it_d = s.solve(torch.from_numpy(dwi).to(cuda), mask=torch.from_numpy(mask).to(cuda), predicted=pred_d)
    np.testing.assert_array_equal(x_h, x_d.cpu().numpy())
    np.testing.assert_array_equal(it_h, it_d.cpu().numpy())
    np.testing.assert_array_equal(pred_h, pred_d.cpu().numpy())
    assert not x_h[mask == 0].any()


def test_msmt_shell_subset(cuda):
    """-shells 0,1000,3000: the volumes of the other shell take no part
    (their rows of the forward matrix are zero, as in the reference)."""
    import torch
    resp = [r[[0, 1, 3]] for r in RESP]
    s = msmt.MSMTShared(synth.msmt_scheme(), shells=[0, 1000, 3000])
    assert [len(v) for v in s.shells] == [6, 30, 60]
    s.set_responses(resp)
    s.init()
    assert not s.C[s.grad[:, 3] == 2000.0].any()
    P = msmt_ref.problem(s.grad, s.shells, resp, [8, 0, 0], s.HR_dirs)
    rng = np.random.default_rng(25)
    full = msmt_ref.problem(s.grad, msmt.cluster_shells(s.grad[:, 3]), RESP, [8, 0, 0], s.HR_dirs)
    dwi = synth.rician(rng, synth.msmt_truth(rng, 200) @ full.H.T, 25.0).astype(np.float32)
    x, _ = s.solve(torch.from_numpy(dwi).to(cuda))
    idx = np.arange(0, 200, 5)
    xr, _ = msmt_ref.solve(P, dwi[idx].astype(np.float64))
    assert _rel(x.cpu().numpy()[idx].astype(np.float64), xr).max() <= 1e-4
