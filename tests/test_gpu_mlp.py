"""The tensor-core MLP (akb_mlp_*) against its FP64 oracle with the same
BF16 roundings: forward values, loss and parameter gradients (the gradient
check), and that Adam training drives the loss down."""
import numpy as np
import pytest

from oracle.oracle import OracleMLP

pytestmark = pytest.mark.gpu


def setup(nb=300, seed=0, width=256, nh=3):
    import torch
    from akantu_b200.surrogate import MLPSurrogate
    rng = np.random.default_rng(seed)
    net = MLPSurrogate(9, 9, width, nh, seed=seed)
    x = rng.uniform(-0.3, 0.3, (nb, 9))
    t = np.sin(3 * x) @ rng.normal(size=(9, 9)) + 0.1
    net.fit_scaling(x, t)
    X = torch.as_tensor(x, device="cuda")
    T = torch.as_tensor(t, device="cuda")
    sc = net.scaling
    O = OracleMLP(9, 9, width, nh, net.get_parameters(), sc["in_shift"], sc["in_scale"],
                  sc["out_shift"], sc["out_scale"])
    return net, X, T, x, t, O


def test_forward_matches_oracle():
    net, X, T, x, t, O = setup()
    y = net.forward_features(X).cpu().numpy()
    yo = O.forward(x, emulate_bf16=True)
    scale = np.abs(yo).max()
    assert np.abs(y - yo).max() <= 5e-3 * scale
    assert np.abs(y - yo).mean() <= 5e-4 * scale


def test_gradient_check_against_cpu():
    net, X, T, x, t, O = setup(nb=300, seed=1)
    loss, g = net.gradients_features(X, T)
    lo, go = O.gradients(x, t, emulate_bf16=True)
    assert loss == pytest.approx(lo, rel=2e-3)
    assert np.linalg.norm(g - go) <= 1e-2 * np.linalg.norm(go)
    # layer by layer: direction and size
    off = 0
    for k, n in net.layer_shapes():
        for size in (k * n, n):
            a, b = g[off:off + size], go[off:off + size]
            off += size
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
            assert cos >= 0.999
            assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-12
    # the FP64 gradient without roundings is close too
    _, g64 = O.gradients(x, t, emulate_bf16=False)
    assert np.linalg.norm(g - g64) <= 5e-2 * np.linalg.norm(g64)


def test_inference_equals_training_forward_and_partial_tiles():
    net, X, T, x, t, O = setup(nb=257, seed=2)
    y = net.forward_features(X).cpu().numpy()
    y1 = net.forward_features(X[100:101]).cpu().numpy()
    assert np.array_equal(y1[0], y[100])


def test_training_reduces_loss():
    net, X, T, x, t, O = setup(nb=4096, seed=3)
    l0, _ = net.gradients_features(X, T)
    losses = net.train(X, T, epochs=60, batch=1024, lr=2e-3, lr_final=1e-4)
    l1, _ = net.gradients_features(X, T)
    assert l1 <= 0.05 * l0 and losses[-1] < losses[0]
