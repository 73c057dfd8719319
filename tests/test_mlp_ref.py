"""CPU check of the FP64 warm-start network reference: its analytic
gradient equals a central finite difference of its loss."""
import numpy as np

from oracle import mlp_ref


def test_reference_gradient_finite_difference():
    rng = np.random.default_rng(0)
    n_in, H, n_out, n = 6, 8, 10, 7
    ld_in, ld_out = 16, 16
    sizes = [H * ld_in, H, H * H, H, ld_out * H, ld_out]
    p = rng.normal(scale=0.5, size=sum(sizes))
    P, _, _ = mlp_ref.unpack(p, n_in, H, n_out)
    # zero the padding the GPU layout keeps at zero
    o = 0
    W1 = p[o:o + H * ld_in].reshape(H, ld_in)
    W1[:, n_in:] = 0
    o = H * ld_in + H + H * H + H
    W3 = p[o:o + ld_out * H].reshape(ld_out, H)
    W3[n_out:] = 0
    p[o + ld_out * H + n_out:] = 0
    x = np.zeros((n, ld_in))
    x[:, :n_in] = rng.normal(size=(n, n_in))
    y = rng.integers(0, 2 ** 10, size=(n, 1)).astype(np.uint32)
    _, loss, g = mlp_ref.forward_backward(p, x, y, n_in, H, n_out, bf16=False)
    eps = 1e-6
    idx = rng.choice(len(p), 60, replace=False)
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        lp = mlp_ref.forward_backward(pp, x, y, n_in, H, n_out, bf16=False)[1]
        lm = mlp_ref.forward_backward(pm, x, y, n_in, H, n_out, bf16=False)[1]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.001953125, 3.14159, -2.5e-3], np.float32)
    r = mlp_ref.to_bf16(a)
    import torch
    t = torch.from_numpy(a).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(r, t)
