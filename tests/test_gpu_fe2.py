"""FE^2 on the GPU: macro model with the RVE-backed material, the surrogate
path with its envelope fallback, and dataset generation."""
import numpy as np
import pytest

from akantu_b200 import fe2

pytestmark = pytest.mark.gpu


def small_rve():
    vm, vf = fe2.sphere_inclusion_rve(8)
    mats = fe2.matrix_inclusion_materials()
    from akantu_b200.rve import SolidMechanicsModelRVE
    return SolidMechanicsModelRVE(8, vm, mats, tolerance=1e-5), mats, vf


def run_macro(provider, mats, vf, steps=12, cells=2):
    m = fe2.macro_block(provider.material(mats, [1 - vf, vf]), cells=cells)
    m.setTimeStep(0.8 * m.getStableTimeStep())
    for s in range(1, steps + 1):
        fe2.macro_step(m, s, ramp_steps=steps, stretch=0.05)
    u = m.getDisplacement().copy()
    m.close()
    return u


def test_fallback_everywhere_equals_plain_fe2():
    """A surrogate whose envelope excludes every point hands all of them to
    the RVEs: the result is the plain FE^2 result bit for bit."""
    from akantu_b200.surrogate import MLPSurrogate
    rve, mats, vf = small_rve()
    u_plain = run_macro(fe2.MaterialFE2(rve), mats, vf)
    net = MLPSurrogate()
    prov = fe2.MaterialFE2(rve, surrogate=net, amplitude=-1.0)
    u_fb = run_macro(prov, mats, vf)
    assert prov.stats["fallback"] == prov.stats["rve_solves"] > 0
    assert np.array_equal(u_plain, u_fb)
    assert np.abs(u_plain[:, 0]).max() == pytest.approx(0.05 * 1.0, rel=1e-12)


def test_plain_fe2_pulls_the_block():
    rve, mats, vf = small_rve()
    prov = fe2.MaterialFE2(rve)
    u = run_macro(prov, mats, vf, steps=12, cells=2)
    assert prov.stats["rve_solves"] == 12 * 8 * 8
    # the free faces contract laterally under the stretch
    assert np.isfinite(u).all() and np.abs(u[:, 1:]).max() > 0


def test_dataset_and_surrogate_error_metrics():
    import torch
    from akantu_b200.surrogate import MLPSurrogate
    rve, mats, vf = small_rve()
    X, Y, it, res = fe2.generate_dataset(rve, 600, seed=5, chunk=256)
    assert X.shape == (600, 9) and Y.shape == (600, 9)
    H = fe2.sample_gradients(600, seed=5)
    assert np.allclose(X[:, [0, 4, 8]].cpu().numpy(), H[:, [0, 1, 2], [0, 1, 2]])
    assert np.allclose(X[:, 1].cpu().numpy(), H[:, 1, 0])  # column-major features
    from akantu_b200.surrogate import scaled_features
    net = MLPSurrogate()
    x, y = scaled_features(X, Y)
    assert x.shape == (600, 10) and y.shape == (600, 9)
    r = torch.linalg.norm(X, dim=1)
    assert torch.allclose(torch.exp(x[:, 9]), r) and torch.allclose(y * r[:, None], Y)
    net.fit_scaling(x.cpu().numpy(), y.cpu().numpy())
    e = fe2.surrogate_error(net, X, Y)
    assert e["relative_l2"] > 0 and e["p99"] >= e["median"]
    net.train(x, y, epochs=30, batch=128, lr=2e-3)
    e2 = fe2.surrogate_error(net, X, Y)
    assert e2["relative_l2"] < e["relative_l2"]
    # small-strain samples: log-uniform magnitudes
    Hs = fe2.sample_small_gradients(1000, seed=2)
    rs = np.linalg.norm(Hs.reshape(-1, 9), axis=1)
    assert rs.min() >= 1e-4 * (1 - 1e-12) and rs.max() <= 0.3 * (1 + 1e-12)


def test_fused_stress_matches_the_eager_path():
    """akb_mlp_stress (features, network, |H| rescale and envelope list in one
    launch) against the same map written with torch around akb_mlp_forward:
    equal to rounding of the norm, and the listed points are exactly those
    outside the envelope."""
    import torch
    from akantu_b200.surrogate import MLPSurrogate
    net = MLPSurrogate(seed=3)
    rng = np.random.default_rng(4)
    n = 5000
    H = torch.as_tensor(rng.normal(0.0, 0.2, (n, 9)), device="cuda")
    H[:7] = 0.0  # |H| = 0: features at the clamp, P = 0
    x = np.asarray(H.cpu())
    net.fit_scaling(np.c_[x, np.log(np.maximum(np.linalg.norm(x, axis=1), 1e-8))],
                    rng.normal(0, 1, (n, 9)))
    ref = net.predict_flat(H)
    P = torch.empty_like(H)
    idx = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.full((1,), 77, dtype=torch.int32, device="cuda")
    amp, mind = 0.3, 0.5
    net.stress_into(H, P, envelope=(amp, mind), fallback=(idx, cnt))
    torch.cuda.synchronize()
    assert torch.equal(P[:7], torch.zeros_like(P[:7]))
    assert ((P - ref).abs().max() / ref.abs().max()).item() <= 1e-12
    F = torch.eye(3, dtype=H.dtype, device=H.device) + H.reshape(-1, 3, 3).transpose(1, 2)
    out = (H.abs().max(dim=1).values > amp) | (torch.linalg.det(F) < mind)
    k = int(cnt.item())
    assert k == int(out.sum()) > 0
    assert sorted(idx[:k].tolist()) == torch.nonzero(out).flatten().tolist()
    # without the envelope: the same stresses, no list
    P2 = torch.empty_like(H)
    net.stress_into(H, P2)
    assert torch.equal(P, P2)


def test_indexed_rve_solve_touches_only_listed_points():
    import torch
    rve, _, _ = small_rve()
    H = torch.as_tensor(fe2.sample_gradients(40, seed=6), device="cuda")
    Hc = H.transpose(1, 2).reshape(-1, 9).contiguous()
    pick = torch.tensor([3, 17, 0, 39, 22], dtype=torch.int32, device="cuda")
    idx = torch.zeros(40, dtype=torch.int32, device="cuda")
    idx[:5] = pick
    cnt = torch.tensor([5], dtype=torch.int32, device="cuda")
    P = torch.full((40, 9), 123.0, dtype=torch.float64, device="cuda")
    w = rve.zero_fluctuation(40)
    rve.solve_indexed(idx, cnt, Hc, P, w)
    ref = rve.solve(H[pick.long()])
    Pr = ref["stress"].transpose(1, 2).reshape(-1, 9)
    torch.cuda.synchronize()
    assert torch.equal(P[pick.long()], Pr)  # the same per-instance kernel body
    others = torch.ones(40, dtype=torch.bool, device="cuda")
    others[pick.long()] = False
    assert bool((P[others] == 123.0).all())
    assert bool((w[others] == 0).all()) and bool((w[pick.long()] != 0).any())
    # an empty list changes nothing
    cnt.zero_()
    P0 = P.clone()
    rve.solve_indexed(idx, cnt, Hc, P, w)
    torch.cuda.synchronize()
    assert torch.equal(P, P0)
