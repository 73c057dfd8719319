"""GPU parity across signal and response scales.

The reference's answer is exactly scale-covariant: scaling the signal by
alpha and the response by beta scales the FOD by alpha / beta
(csd.h:102-198: M and HR_trans grow with the response, the constraint
multiplier 50 r0 / 300 with its l = 0 term, b = M^T S with both).  The GPU
path splits its FP32 constraint tables and FODs into FP16 hi + lo halves for
the tensor cores, so it has to keep those halves inside FP16's range at
every scale a caller can hand it: raw scanner units (responses of 1e5 and
more), normalised data (1e-3), and dwi2response tournier's first-round
response "1 -1 1" on a signal of ~1500.  Each case is checked against the
FP64 oracle on the same scaled inputs with the usual bar (p99 relative error
<= 1e-4, >= 99.5% of voxels on the oracle's final negative set), for the
persistent kernel and for the phased method, plain and warm-started.
"""
import os

import numpy as np
import pytest

from mrtrix3_b200 import csd, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P99_TOL = 1e-4
MATCH_TOL = 0.995
WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mrtrix3_b200", "data",
                       "warmstart_c5.npz")

# (signal scale, response scale); alpha / beta is the FOD's scale
CASES = [(1.0, 1.0), (1e-3, 1e-3), (1e3, 1e3), (1e5, 1e5), (1e-4, 1.0), (1e4, 1.0), (1.0, 1e-3), (1.0, 1e2)]


def _volume():
    # the benchmark's scheme (6 b=0 + 60 DW), a small number of voxels
    grad = synth.config5_scheme()
    rng = np.random.default_rng(77)
    return grad, synth.voxel_signals(rng, grad, 1536, (15.0, 40.0))


def _rel(fod, F):
    den = np.abs(F).max(axis=1)
    return np.abs(fod.astype(np.float64) - F).max(axis=1) / np.where(den > 0, den, 1.0)


def _check(out, ref, label):
    r = _rel(out["fod"], ref["F"])
    m = np.all(out["negmask"].view(np.uint32) == ref["negmask"], axis=1)
    assert np.all(np.isfinite(out["fod"])), label
    assert np.percentile(r, 99) <= P99_TOL, (label, np.percentile(r, 99), r.max())
    assert m.mean() >= MATCH_TOL, (label, m.mean())


def _run_all(grad, dwi, response, hr_dirs, warm_net=None):
    import torch
    ref = O.OracleShared(grad, response, hr_dirs).solve(dwi)
    s = csd.make_shared(grad, response)
    d = torch.from_numpy(np.ascontiguousarray(dwi)).cuda()
    outs = {}
    o = csd.dwi2fod_csd(s, d, want_negmask=True)
    outs["persistent"] = {k: v.cpu().numpy() for k, v in o.items()}
    st = csd.State(s, d.shape[0])
    st.run(d)
    outs["phased_plain"] = st.fod()
    if warm_net is not None:
        st.run(d, warm=warm_net.predict(d))
        outs["phased_warm"] = st.fod()
    st.close()
    return ref, outs


@pytest.mark.parametrize("alpha,beta", CASES)
def test_scaled_signal_and_response(cuda, hr_dirs, alpha, beta):
    from mrtrix3_b200.warmstart import WarmStartNet
    grad, dwi = _volume()
    net = WarmStartNet.load(WEIGHTS) if alpha == beta else None  # the network sees S / S0: any alpha
    ref, outs = _run_all(grad, (dwi * alpha).astype(np.float32), synth.RESPONSE * beta, hr_dirs, net)
    for name, out in outs.items():
        _check(out, ref, f"{name} alpha={alpha} beta={beta}")


def test_tournier_first_round_response(cuda, hr_dirs):
    """dwi2response tournier starts from the response "1 -1 1" on the raw
    signal (tournier.py): FODs of ~1e3 times the usual size."""
    grad, dwi = _volume()
    ref, outs = _run_all(grad, dwi, np.array([1.0, -1.0, 1.0]), hr_dirs)
    for name, out in outs.items():
        _check(out, ref, f"{name} response 1 -1 1")
