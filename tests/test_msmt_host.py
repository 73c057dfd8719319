"""Host set-up of multi-shell multi-tissue CSD (mrtrix3_b200/msmt.py) against
the FP64 restatement (oracle/msmt_ref.py) and the shell rules; the oracle's
solutions against the optimality conditions.  CPU only."""
import numpy as np
import pytest

from mrtrix3_b200 import msmt, synth
from oracle import icls_ref, msmt_ref

RESP = [synth.MSMT_RESPONSES["wm"], synth.MSMT_RESPONSES["gm"], synth.MSMT_RESPONSES["csf"]]


def _shared(lmax=None):
    s = msmt.MSMTShared(synth.msmt_scheme())
    if lmax is not None:
        s.parse_cmdline_options(lmax=lmax)
    s.set_responses(RESP)
    return s.init(upload=False)


def test_shells_of_the_scheme():
    g = synth.msmt_scheme(6, (30, 45, 60))
    shells = msmt.cluster_shells(g[:, 3])
    assert [len(v) for v in shells] == [6, 30, 45, 60]
    assert list(shells[0]) == list(range(6)) and list(shells[3]) == list(range(81, 141))
    # b-values jittered within the clustering distance still form one shell each
    g2 = g.copy()
    g2[6:, 3] += np.random.default_rng(0).uniform(-30, 30, len(g) - 6)
    assert [len(v) for v in msmt.cluster_shells(g2[:, 3])] == [6, 30, 45, 60]
    # a volume with no neighbours is left out
    g3 = np.vstack([g, [[1.0, 0.0, 0.0, 5000.0]]])
    assert sum(len(v) for v in msmt.cluster_shells(g3[:, 3])) == len(g)


def test_scheme_normalisation():
    g = synth.msmt_scheme()
    g2 = g.copy()
    g2[6:, :3] *= 2.0  # |g| = 2: directions normalised, b scaled by |g|^2
    n = msmt.normalise_scheme(g2)
    np.testing.assert_allclose(n[6:, :3], g[6:, :3], atol=1e-15)
    np.testing.assert_allclose(n[6:, 3], 4.0 * g[6:, 3])


@pytest.mark.parametrize("lmax", [None, [8, 0, 0], [6, 0, 0], [4, 2, 0]])
def test_forward_and_constraint_matrices_match_oracle(lmax):
    s = _shared(lmax)
    want_lmax = lmax or [8, 0, 0]
    assert s.lmax == want_lmax
    resp = [np.pad(r, ((0, 0), (0, max(0, L // 2 + 1 - r.shape[1]))))[:, :L // 2 + 1]
            for r, L in zip(RESP, want_lmax)]
    C = msmt_ref.forward_matrix(s.grad, s.shells, resp, want_lmax)
    A = msmt_ref.constraint_matrix(s.HR_dirs, want_lmax)
    assert s.C.shape == C.shape and s.A.shape == A.shape
    assert np.max(np.abs(s.C - C)) <= 1e-9 * np.max(np.abs(C))
    assert np.max(np.abs(s.A - A)) <= 1e-12


def test_response_rules():
    s = msmt.MSMTShared(synth.msmt_scheme())
    wm = np.hstack([RESP[0], np.zeros((4, 3))])  # trailing zero columns are clipped
    s.set_responses([wm, RESP[1]])
    assert s.lmax_response == [8, 0]
    s.init(upload=False)
    assert s.nparams() == [45, 1]
    with pytest.raises(ValueError, match="number of shells"):
        bad = msmt.MSMTShared(synth.msmt_scheme())
        bad.set_responses([RESP[0][:3]])
        bad.init(upload=False)
    with pytest.raises(ValueError, match="does not match number of tissues"):
        bad = msmt.MSMTShared(synth.msmt_scheme())
        bad.parse_cmdline_options(lmax=[8, 0])
        bad.set_responses(RESP)
        bad.init(upload=False)
    with pytest.raises(ValueError, match="non-negative even"):
        bad = msmt.MSMTShared(synth.msmt_scheme())
        bad.parse_cmdline_options(lmax=[7, 0, 0])
        bad.set_responses(RESP)
        bad.init(upload=False)


def test_oracle_solutions_are_optimal():
    """The oracle's MSMT solutions satisfy the optimality conditions of
    min ||C x - b||^2 + (regularisation) s.t. A x >= 0."""
    s = _shared()
    P = msmt_ref.problem(s.grad, s.shells, [RESP[0], RESP[1], RESP[2]], [8, 0, 0], s.HR_dirs)
    rng = np.random.default_rng(3)
    truth = synth.msmt_truth(rng, 12)
    clean = truth @ P.H.T
    dwi = synth.rician(rng, clean, 20.0)
    x, it = msmt_ref.solve(P, dwi)
    assert (it <= P.max_niter).all()
    A = msmt_ref.constraint_matrix(s.HR_dirs, [8, 0, 0])
    for xi, b in zip(x, dwi):
        r = A @ xi
        assert r.min() > -1e-6 * np.abs(r).max()
        # stationarity of the regularised objective: H^T (H x - b) + reg x = A_act^T mu, mu >= 0
        HtH = P.H.T @ P.H
        reg = 1e-10 * np.max(np.diag(HtH))
        g = HtH @ xi - P.H.T @ b + reg * xi
        act = np.nonzero(r < 1e-7 * np.abs(r).max())[0]
        mu, *_ = np.linalg.lstsq(A[act].T, g, rcond=None)
        assert np.linalg.norm(A[act].T @ mu - g) <= 1e-6 * np.linalg.norm(P.H.T @ b)
        assert mu.min() >= -1e-6 * np.abs(mu).max()
    # noiseless pure grey matter / CSF voxels are recovered
    for i in (0, 5):
        xi, _ = icls_ref.solve(P, clean[i])
        np.testing.assert_allclose(xi[-2:], truth[i, -2:], atol=1e-6 * np.abs(truth[i]).max())


def test_icls_create_rejects_bad_problems():
    """Argument checks of csd_icls_create run before any device work."""
    import ctypes

    from mrtrix3_b200 import csd
    h = ctypes.c_void_p()
    H = np.ones((4, 2))
    A = np.ones((3, 2))
    L = csd.lib()
    for args in [(H.ctypes.data, 4, 0, A.ctypes.data, 3, None, 0, 0.0, 0.0, 0, 0.0),    # no parameters
                 (H.ctypes.data, 4, 2, A.ctypes.data, 3, None, 4, 0.0, 0.0, 0, 0.0),    # more equalities than rows
                 (H.ctypes.data, 4, 2, A.ctypes.data, 3, None, 0, -1.0, 0.0, 0, 0.0),   # negative regularisation
                 (H.ctypes.data, 4, 2, A.ctypes.data, 3, None, 0, 0.0, 0.0, 0, -1.0),   # negative tolerance
                 (H.ctypes.data, 4, 300, A.ctypes.data, 3, None, 0, 0.0, 0.0, 0, 0.0)]:  # too many parameters
        assert L.csd_icls_create(*args, ctypes.byref(h)) == csd.CSD_ERR_INVALID
        assert not h.value


def test_top_threshold_rule():
    """mrthreshold -top N: the value at index size - N of the sorted finite
    values, voxels >= it selected (ties at the threshold all kept)."""
    from mrtrix3_b200.dwi2response import top_threshold
    v = np.array([0.1, 0.5, np.nan, 0.3, 0.9, 0.5, 0.0])
    assert top_threshold(v, 2) == 0.5
    assert np.sum(v >= top_threshold(v, 2)) == 3  # the tie at 0.5 keeps both
    assert top_threshold(v, 6) == 0.0
    with pytest.raises(SystemExit, match="less than number of voxels"):
        top_threshold(v, 7)


def test_dwi2response_argument_errors(tmp_path):
    from mrtrix3_b200.dwi2response import run
    with pytest.raises(SystemExit, match="usage"):
        run(["dhollander", "a.mif", "r.txt"])
    with pytest.raises(SystemExit, match="wrong number of arguments"):
        run(["manual", "a.mif", "r.txt"])
    with pytest.raises(SystemExit, match="-mask is required"):
        run(["fa", "a.mif", str(tmp_path / "r.txt")])
    out = tmp_path / "r.txt"
    out.write_text("1\n")
    with pytest.raises(SystemExit, match="already exists"):
        run(["fa", "a.mif", str(out), "-mask", "m.mif"])


def test_shell_selection_rules():
    """Shells::select_shells with -shells (dwi/shells.cpp:100-215): exact
    range, within 1 of a mean, nearest in standard deviations, the
    ambiguity rule (the last shell's verdict, as there), b=0, repeats."""
    g = msmt.normalise_scheme(synth.msmt_scheme())
    sh = msmt.cluster_shells(g[:, 3])
    assert msmt.select_shells(g[:, 3], sh, [0, 3000]) == [0, 3]
    assert msmt.select_shells(g[:, 3], sh, [2000.5]) == [2]
    assert msmt.select_shells(g[:, 3], sh, [1000, 2000]) == [1, 2]
    with pytest.raises(ValueError, match="robustly"):
        msmt.select_shells(g[:, 3], sh, [2100])
    with pytest.raises(ValueError, match="more than once"):
        msmt.select_shells(g[:, 3], sh, [1000, 1000.4])
    with pytest.raises(ValueError, match="b=0 shell more than once"):
        msmt.select_shells(g[:, 3], sh, [0, 5])
    with pytest.raises(ValueError, match="negative"):
        msmt.select_shells(g[:, 3], sh, [-1])
    g2 = g.copy()
    g2[6:, 3] += np.random.default_rng(0).uniform(-40, 40, len(g) - 6)
    sh2 = msmt.cluster_shells(g2[:, 3])
    assert msmt.select_shells(g2[:, 3], sh2, [1000, 3000]) == [1, 3]
    # a shell's "max" is its last volume's b-value (shells.cpp:63-64)
    mean, sd, lo, hi = msmt._shell_stats(g2[:, 3], sh2[1])
    assert lo == g2[sh2[1], 3].min() and hi == max(lo, g2[sh2[1][-1], 3])
    # the multi-tissue set-up keeps only the selected shells
    s = msmt.MSMTShared(synth.msmt_scheme(), shells=[0, 3000])
    assert [len(v) for v in s.shells] == [6, 60]


@pytest.mark.parametrize("lmax", [0, 2, 8, 10, 12])
def test_amp2response_host_transforms_match_oracle(lmax):
    """ZSH::init_amp_transform / init_deriv_transform (ZSH.h:66-99) and the
    constraint matrix at 0..90 degrees (amp2response.cpp:337-344)."""
    from mrtrix3_b200 import amp2response as AR
    from oracle import amp2response_ref as AREF
    els = np.linspace(0.0, np.pi, 37)
    assert np.abs(AR.zonal_amp_transform(els, lmax) - AREF._zonal(els, lmax, 0)).max() <= 1e-12
    if lmax:
        d = AR.zonal_deriv_transform(els, lmax)
        dr = AREF._zonal(els, lmax, 1)
        assert np.abs(d[:, 1:] - dr[:, 1:]).max() <= 1e-12 and not d[:, 0].any()
        C = AR.constraint_matrix(lmax)
        assert C.shape == (182, lmax // 2 + 1)
        assert np.abs(C - AREF.constraints(lmax)).max() <= 1e-12
