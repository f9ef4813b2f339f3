"""The perceptron on the tensor cores (tcgen05, BF16 x BF16 -> FP32 in tensor
memory) against the numpy oracle with the same BF16 rounding points.

Tolerances (norm-wise relative): forward outputs 1e-2; loss 1e-2; every
layer's weight and bias gradient 3e-2 -- BF16 intermediates round at the same
points on both sides, but the tensor cores accumulate in FP32 in their own
order, which can move a rounding boundary.
"""
import numpy as np
import pytest

from multilayersolver2024_b200.learned import Mlp
from oracle import mlp as M

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("B", [128, 300, 1024])
def test_forward_matches_oracle(gpu, B):
    net = Mlp(44, 7, n_hidden=128, n_hidden_layers=3, max_batch=1024, seed=1)
    p = net.get_params()
    x = np.random.default_rng(B).normal(0, 1, (B, 44)).astype(np.float32)
    y = net.forward(x)
    ref, _ = M.forward(p, net.layer_shapes(), x)
    assert _rel(y, ref) <= 1e-2


@pytest.mark.parametrize("B,hidden", [(256, 128), (200, 64)])
def test_gradient_matches_oracle(gpu, B, hidden):
    rng = np.random.default_rng(7)
    net = Mlp(44, 7, n_hidden=hidden, n_hidden_layers=3, max_batch=512, seed=2)
    p = net.get_params()
    x = rng.normal(0, 1, (B, 44)).astype(np.float32)
    t = rng.normal(0, 1, (B, 7)).astype(np.float32)
    loss, g = net.loss_grad(x, t)
    ref_loss, ref_g = M.loss_grad(p, net.layer_shapes(), x, t)
    assert abs(loss - ref_loss) <= 1e-2 * abs(ref_loss)
    o = 0
    for (n_out, n_in) in net.layer_shapes():
        for size in (n_out * n_in, n_out):
            assert _rel(g[o:o + size], ref_g[o:o + size]) <= 3e-2, (n_out, n_in, size)
            o += size


def test_training_reduces_loss(gpu):
    rng = np.random.default_rng(3)
    x = rng.normal(0, 1, (8192, 44)).astype(np.float32)
    A = rng.normal(0, 0.3, (44, 7))
    t = (np.tanh(x @ A) + 0.1 * np.sin(3 * x[:, :7])).astype(np.float32)
    net = Mlp(44, 7, max_batch=1024, seed=4)
    losses = net.train(x, t, batch=512, epochs=12, lr=2e-3)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.15 * losses[0], losses


def test_device_gelu_matches_erf_gelu(gpu):
    """The hidden activation on the device is GELU: a one-hidden-layer network
    with identity weights returns GELU(x) of the BF16-rounded inputs, within
    the BF16 rounding of the stored activation (and the tanh form's 1e-3)."""
    from scipy.special import erf
    n = 44
    net = Mlp(n, n, n_hidden=128, n_hidden_layers=1, max_batch=512, seed=3)
    W1 = np.zeros((128, n), np.float32)
    W1[np.arange(n), np.arange(n)] = 1.0
    W2 = np.zeros((n, 128), np.float32)
    W2[np.arange(n), np.arange(n)] = 1.0
    net.set_params(np.concatenate([W1.ravel(), np.zeros(128, np.float32), W2.ravel(), np.zeros(n, np.float32)]))
    x = np.linspace(-6.0, 6.0, 512 * n, dtype=np.float32).reshape(512, n)
    y = net.forward(x)
    xb = M.bf16(x)
    exact = 0.5 * xb * (1.0 + erf(xb / np.sqrt(2.0)))
    assert np.all(np.abs(y - exact) <= 1e-3 + 2.0 ** -8 * np.abs(exact))
    net.close()
