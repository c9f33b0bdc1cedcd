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


def test_compute_then_apply_is_the_train_step():
    """akb_mlp_compute_gradients + akb_mlp_apply_gradients (the halves a
    data-parallel step all-reduces between) equal akb_mlp_train_step bit for
    bit, and the gradient view is the array the library reads."""
    import torch
    from akantu_b200.surrogate import MLPSurrogate
    rng = np.random.default_rng(12)
    x = torch.as_tensor(rng.normal(size=(1000, 10)), device="cuda")
    t = torch.as_tensor(rng.normal(size=(1000, 9)), device="cuda")
    a, b = MLPSurrogate(seed=4), MLPSurrogate(seed=4)
    for step in range(3):
        la = a.train_step_features(x, t, 1e-3)
        lb = b.compute_gradients(x, t)
        g = b.gradient_tensor()
        assert g.shape == (b.nb_parameters,) and bool(torch.isfinite(g).all())
        b.apply_gradients(1e-3)
        assert la == lb
    assert np.array_equal(a.get_parameters(), b.get_parameters())
    # a gradient scaled in place before the step changes it (the step reads the view)
    c = MLPSurrogate(seed=4)
    c.compute_gradients(x, t)
    c.gradient_tensor().mul_(0.0)
    p0 = c.get_parameters()
    c.apply_gradients(1e-3)
    torch.cuda.synchronize()
    assert np.array_equal(c.get_parameters(), p0)  # Adam with zero gradient: no move
    a.close(), b.close(), c.close()
