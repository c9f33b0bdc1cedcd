"""Parity at the benchmark's full sizes (B200), where the CPU oracle would
take hours: the fused fast modes against the GPU reference-order mode (the
reference's operation order, bitwise equal to the oracle on every size the
oracle runs in tests/test_gpu_parity.py), on the same steps.

  cube_tet4 100^3 x 6 (6 M elements), its 1000 steps: FP64 <= 1e-10,
      FP32-bulk <= 1e-5 (displacement, relative to its maximum);
  block_hex8 128^3 neo-Hookean (2.1 M elements), its 2000 steps: FP64 <=
      1e-10, FP32-bulk <= 1e-5.
"""
import numpy as np
import pytest

from akantu_b200 import _abi, configs

pytestmark = pytest.mark.gpu


def _run(w, mode, steps):
    from akantu_b200.model import SolidMechanicsModel, material_from_dict
    m = SolidMechanicsModel(w["mesh"], [material_from_dict(mm) for mm in w["materials"]],
                            precision=mode)
    m.initFull()

    class F:
        set = m.setField
        set_blocked = m.setBlockedDOFs
        stable_time_step = m.getStableTimeStep
        set_time_step = m.setTimeStep
    dt = configs.setup_model(F, w)
    m.solveSteps(steps)
    u = np.array(m.getDisplacement())
    v = np.array(m.getVelocity())
    m.close()
    return dt, u, v


def _rel(x, ref):
    return np.abs(x - ref).max() / np.abs(ref).max()


@pytest.mark.parametrize("w", [
    lambda: configs.cube_tet4(100),
    lambda: configs.block_hex8(128, 1.28),
], ids=["cube_tet4_100", "block_hex8_128"])
def test_fast_modes_against_reference_order(w):
    w = w()
    steps = w["steps"]
    dt_r, u_r, v_r = _run(w, _abi.MODE_FP64_REFERENCE, steps)
    dt_f, u_f, v_f = _run(w, _abi.MODE_FP64, steps)
    assert dt_f == dt_r
    assert _rel(u_f, u_r) <= 1e-10 and _rel(v_f, v_r) <= 1e-10
    dt_s, u_s, _ = _run(w, _abi.MODE_FP32_BULK, steps)
    assert dt_s == dt_r
    assert _rel(u_s, u_r) <= 1e-5
