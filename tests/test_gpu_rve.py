"""Batched periodic RVE solves on the GPU against the FP64 oracle."""
import numpy as np
import pytest

from akantu_b200 import _abi, fe2
from tests.fe2_cases import lame, neohookean_P, oracle_rve, rve_case

pytestmark = pytest.mark.gpu


def gpu_rve(cells, vm, mats, **kw):
    from akantu_b200.rve import SolidMechanicsModelRVE
    return SolidMechanicsModelRVE(cells, vm, mats, **kw)


def test_fp64_rve_matches_oracle_step_for_step():
    """Same algorithm in FP64: after a fixed number of updates the stresses and
    fluctuations agree to rounding (colour order vs element order sums)."""
    vm, mats = rve_case(8)
    H = fe2.sample_gradients(3, seed=21)
    R = gpu_rve(8, vm, mats, precision=_abi.MODE_FP64, tolerance=-1.0, max_iterations=150)
    out = R.solve(H, R.zero_fluctuation(3))
    P = out["stress"].cpu().numpy()
    w = out["fluctuation"].cpu().numpy()
    assert (out["iterations"].cpu().numpy() == 150).all()
    O = oracle_rve(8, vm, mats)
    for k in range(3):
        Po, wo, it, r = O.solve(H[k], tolerance=-1.0, max_iterations=150, time_step_factor=0.6,
                                damping_factor=0.6)
        assert it == 150
        assert np.abs(P[k] - Po).max() <= 1e-10 * np.abs(Po).max()
        assert np.abs(w[k] - wo).max() <= 1e-9 * np.abs(wo).max()
        assert out["residual"][k].item() == pytest.approx(r, rel=1e-6)


def test_stress_of_given_state_matches_oracle():
    vm, mats = rve_case(8)
    H = fe2.sample_gradients(2, seed=4)
    rng = np.random.default_rng(0)
    w = 0.01 * rng.normal(size=(2, 512, 3))
    R = gpu_rve(8, vm, mats, precision=_abi.MODE_FP64)
    import torch
    P, f = R.stress(H, torch.as_tensor(w, device="cuda"))
    O = oracle_rve(8, vm, mats)
    for k in range(2):
        Po, fo = O.stress(H[k], w[k])
        assert np.abs(P[k].cpu().numpy() - Po).max() <= 1e-12 * np.abs(Po).max()
        assert np.abs(f[k].cpu().numpy() - fo).max() <= 1e-10 * np.abs(fo).max()


def test_fp32_rve_16_cells_matches_converged_oracle():
    vm, mats = rve_case(16)
    H = fe2.sample_gradients(4, seed=8)
    R = gpu_rve(16, vm, mats, tolerance=1e-5)
    out = R.solve(H)
    P = out["stress"].cpu().numpy()
    it = out["iterations"].cpu().numpy()
    assert (out["residual"].cpu().numpy() <= 1e-5).all() and (it < 2000).all()
    O = oracle_rve(16, vm, mats)
    for k in range(2):
        Po, _, ito, _ = O.solve(H[k], tolerance=1e-7, time_step_factor=0.6, damping_factor=0.6)
        assert np.abs(P[k] - Po).max() <= 2e-4 * np.abs(Po).max()


def test_homogeneous_and_identity_need_no_update():
    vm, mats = rve_case(16, homogeneous=True)
    R = gpu_rve(16, vm, mats)
    H = fe2.sample_gradients(8, seed=3)
    H[0] = 0.0
    out = R.solve(H)
    assert int(out["iterations"].max()) == 0
    lam, mu = lame(mats[0])
    P = out["stress"].cpu().numpy()
    assert np.abs(P[0]).max() == 0.0
    for k in range(1, 8):
        ref = neohookean_P(H[k], lam, mu)
        assert np.abs(P[k] - ref).max() <= 1e-5 * np.abs(ref).max()


def test_warm_start_and_batch_independence():
    vm, mats = rve_case(16)
    H = fe2.sample_gradients(32, seed=9)
    R = gpu_rve(16, vm, mats)
    w = R.zero_fluctuation(32)
    first = R.solve(H, w)
    P1 = first["stress"].clone()
    again = R.solve(H, w)  # restarts from the relaxed fluctuation
    assert int(again["iterations"].max()) <= 10
    assert float((again["stress"] - P1).abs().max()) <= 1e-4 * float(P1.abs().max())
    # one instance alone gives the same stress as inside the batch
    single = R.solve(H[5:6])
    assert np.array_equal(single["stress"].cpu().numpy()[0], P1.cpu().numpy()[5])


def test_rve_argument_errors():
    from akantu_b200._lib import AkbError
    vm, mats = rve_case(8)
    with pytest.raises(AkbError):
        gpu_rve(7, np.zeros(343, np.uint8), mats)  # odd cell count
    with pytest.raises(AkbError):
        gpu_rve(16, vm[:0].tolist() + [0] * 4096, mats, precision=_abi.MODE_FP64)  # too large
    bad = np.full(512, 5, np.uint8)
    with pytest.raises(AkbError):
        gpu_rve(8, bad, mats)
