"""A mesh cut into parts (akb_model_create_part), all parts held by one
process on one GPU and stepped through akantu_b200.decompose.DistributedModel
(the interface forces summed on the device, as the all-reduce over
processes would), against the whole mesh in one model of the same mode
(B200): <= 1e-10 relative after 100 steps in AKB_MODE_FP64 and
AKB_MODE_FP32_BULK (each element's arithmetic is the same in both runs;
only the order of the interface sums differs)."""
import numpy as np
import pytest

from akantu_b200 import _abi, configs
from akantu_b200._lib import AkbError
from akantu_b200.decompose import DistributedModel

pytestmark = pytest.mark.gpu

STEPS = 100


def _workload():
    w = configs.cube_tet4(n=10)
    rng = np.random.default_rng(11)
    v0 = w["v0"] + rng.normal(0.0, 0.1, w["v0"].shape)
    v0[w["blocked"].astype(bool)] = 0.0
    w["v0"] = v0
    return w


def _rel(x, ref):
    return np.abs(x - ref).max() / np.abs(ref).max()


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_FP32_BULK], ids=["fp64", "fp32bulk"])
@pytest.mark.parametrize("nparts", [2, 3])
def test_parts_match_whole_mesh(mode, nparts):
    from akantu_b200.model import SolidMechanicsModel, material_from_dict
    w = _workload()
    whole = SolidMechanicsModel(w["mesh"], [material_from_dict(m) for m in w["materials"]],
                                precision=mode)
    whole.initFull()

    class F:
        set = whole.setField
        set_blocked = whole.setBlockedDOFs
        stable_time_step = whole.getStableTimeStep
        set_time_step = whole.setTimeStep
    dt = configs.setup_model(F, w)
    whole.solveSteps(STEPS)

    dm = DistributedModel(w["mesh"], w["materials"], nparts, precision=mode)
    dm.set_blocked(w["blocked"])
    dm.set_field(_abi.FIELD_DISPLACEMENT, w["u0"])
    dm.set_field(_abi.FIELD_VELOCITY, w["v0"])
    # a minimum over elements: the parts' minimum is the whole mesh's (before stepping)
    assert w["dt_factor"] * dm.stable_time_step() == dt
    dm.set_time_step(dt)
    dm.solve_steps(STEPS)
    for f in (_abi.FIELD_DISPLACEMENT, _abi.FIELD_VELOCITY, _abi.FIELD_ACCELERATION):
        e = _rel(dm.get_field(f), np.array(whole.getField(f)))
        assert e <= 1e-10, (f, e)
    # the lumped mass of the interface nodes is the whole mesh's
    assert _rel(dm.get_field(_abi.FIELD_MASS), np.array(whole.getField(_abi.FIELD_MASS))) <= 1e-14
    dm.close()
    whole.close()


def test_part_refuses_the_unsplit_step():
    w = _workload()
    dm = DistributedModel(w["mesh"], w["materials"], 2, precision=_abi.MODE_FP64)
    dm.set_time_step(1e-7)
    with pytest.raises(AkbError):
        dm.backends[0].m.solveSteps(1)
    dm.close()
