"""GPU tests of the warm-start network: kernel gradients against the FP64 CPU
reference, training, and what the warm start gains over the plain method."""
import numpy as np
import pytest

from mrtrix3_b200 import csd, synth
from oracle import mlp_ref
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_gradients_match_cpu_oracle(cuda):
    """Forward logits and BCE gradients of every parameter tensor from the
    hand-written kernels agree with the FP64 reference (BF16 rounding
    emulated at the same storage points) to 1% relative L2."""
    import torch

    from mrtrix3_b200.warmstart import WarmStartNet
    grad = synth.config5_scheme()
    rng = np.random.default_rng(3)
    sig = synth.voxel_signals(rng, grad, 512, (15.0, 40.0))
    net = WarmStartNet(66, 256, 300, seed=5)
    net.fit_inputs(grad, sig)
    x = net.inputs(torch.from_numpy(sig).cuda())
    y = torch.from_numpy(rng.integers(0, 2 ** 32, size=(512, 10), dtype=np.uint64).astype(np.uint32).view(np.int32)).cuda()
    y[:, 9] &= (1 << 12) - 1
    p = net.get_params()
    xh = x.cpu().numpy().view(np.uint16).astype(np.uint32) << 16
    xh = xh.view(np.float32).astype(np.float64)
    Z, loss, g_ref = mlp_ref.forward_backward(p, xh, y.cpu().numpy().view(np.uint32), 66, 256, 300, bf16=True)
    z = net.logits(x)
    assert _rel(z, Z[:, :300]) < 1e-2
    g, l_gpu = net.gradients(x, y)
    assert abs(l_gpu - loss) <= 1e-3 * abs(loss)
    for name, (o, size) in net.layout().items():
        assert _rel(g[o:o + size], g_ref[o:o + size]) < 1e-2, name


def _labelled(n, seed):
    import torch
    grad = synth.config5_scheme()
    sig = synth.voxel_signals(np.random.default_rng(seed), grad, n, (15.0, 40.0))
    s = csd.make_shared(grad, synth.RESPONSE)
    d = torch.from_numpy(sig).cuda()
    o = csd.dwi2fod_csd(s, d, want_negmask=True)
    return grad, sig, s, d, o


def test_training_reduces_loss(cuda):
    from mrtrix3_b200.warmstart import WarmStartNet
    grad, sig, s, d, o = _labelled(32768, 21)
    net = WarmStartNet(66, 256, 300, seed=1)
    net.fit_inputs(grad, sig)
    losses = net.train(net.inputs(d), o["negmask"], epochs=4, batch=2048, lr=2e-3)
    assert losses[-1] < 0.8 * losses[0]
    assert losses[-1] < 0.45


def test_warm_start_gains_over_plain(cuda, hr_dirs):
    """Trained on 300k labelled voxels, the network's first sets cut the
    iterate() calls of a fresh volume, while the result stays on the FP64
    oracle within the parity bar (p99 rel err <= 1e-4, >= 99.5% same set)."""
    import torch

    from mrtrix3_b200.warmstart import train_warm_start
    grad = synth.config5_scheme()
    net, losses = train_warm_start(grad, n_train=400_000, epochs=10, batch=4096, seed=2)
    v = synth.make_volume((40, 40, 20), 6, 60, (15.0, 40.0), 8, 0.5, 9001)
    s = csd.make_shared(v.grad, synth.RESPONSE)
    d = torch.from_numpy(v.dwi).cuda()
    m = torch.from_numpy(v.mask).cuda()
    plain = csd.dwi2fod_csd(s, d, mask=m, want_negmask=True)
    warm_sets = net.predict(d, mask=m)
    warm = csd.dwi2fod_csd(s, d, mask=m, warm=warm_sets, want_negmask=True)
    torch.cuda.synchronize()
    inside = v.mask.astype(bool)
    it_plain = plain["iterations"].cpu().numpy()[inside].astype(float)
    it_warm = warm["iterations"].cpu().numpy()[inside].astype(float)
    # plain starts average ~5.4 iterate() calls; the learned first sets save
    # the early passes (the boundary directions still take their own steps)
    print(f"iterate() calls per voxel: plain {it_plain.mean():.3f}, warm {it_warm.mean():.3f}")
    assert it_warm.mean() <= it_plain.mean() - 0.6, (it_warm.mean(), it_plain.mean())
    idx = np.nonzero(inside)[0][:3000]
    ref = O.OracleShared(v.grad, synth.RESPONSE, hr_dirs).solve(v.dwi[idx])
    fod = warm["fod"].cpu().numpy()[idx].astype(np.float64)
    rel = np.abs(fod - ref["F"]).max(1) / np.abs(ref["F"]).max(1)
    match = np.mean(np.all(warm["negmask"].cpu().numpy()[idx].view(np.uint32) == ref["negmask"], axis=1))
    assert np.percentile(rel, 99) <= 1e-4
    assert match >= 0.995


def test_fused_inference_matches_layer_gemms(cuda):
    """csd_mlp_predict's fused tcgen05 kernel (inputs, three layers and the
    bit packing in one launch, accumulators in tensor memory) gives the sets
    of the one-GEMM-per-layer path: the logits differ only in FP32 summation
    order, so at most a few bits in 10^4 flip, masked-out voxels get empty
    sets, ragged last tiles are handled, and new weights are re-packed."""
    import os

    import torch

    from mrtrix3_b200 import autotune
    from mrtrix3_b200.warmstart import WarmStartNet
    here = os.path.dirname(os.path.abspath(__file__))
    net = WarmStartNet.load(os.path.join(here, "..", "mrtrix3_b200", "data", "warmstart_c5.npz"))
    grad = synth.config5_scheme()
    rng = np.random.default_rng(12)
    sig = synth.voxel_signals(rng, grad, 20_001, (15.0, 40.0))
    d = torch.from_numpy(sig).cuda()
    mask = torch.from_numpy((rng.random(len(sig)) < 0.5).astype(np.uint8)).cuda()

    def both(mk):
        out = {}
        try:
            for kind in (1, 2):
                autotune.set_knob(autotune.KNOB_INFER, kind)
                out[kind] = net.predict(d, mask=mk).cpu().numpy().view(np.uint32)
        finally:
            autotune.set_knob(autotune.KNOB_INFER, 0)
        return out

    for mk in (None, mask):
        o = both(mk)
        diff = np.unpackbits((o[1] ^ o[2]).view(np.uint8)).sum()
        assert diff <= 2e-4 * o[1].size * 32, diff
        if mk is not None:
            off = mask.cpu().numpy() == 0
            assert not o[2][off].any()
        assert o[2][:, -1].max() < (1 << (300 - 288))  # no bits past the 300 directions
        assert np.unpackbits(o[2].view(np.uint8)).mean() > 0.2  # the sets are not empty
    # new weights must reach the fused kernel
    p = net.get_params()
    net.set_params(p * np.float32(0.5))
    o = both(None)
    diff = np.unpackbits((o[1] ^ o[2]).view(np.uint8)).sum()
    assert diff <= 2e-4 * o[1].size * 32, diff
    net.set_params(p)
