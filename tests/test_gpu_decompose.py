"""A mesh cut into parts (akb_model_create_part), all parts held by one
process on one GPU and stepped through akantu_b200.decompose.DistributedModel
with the neighbour exchange (akb_part_pack_forces, the blocks copied between
the parts as the NCCL send/recv between processes would carry them,
akb_part_step_end_exchange), against the whole mesh in one model of the same
mode (B200): <= 1e-10 relative after 100 steps in AKB_MODE_FP64 and
AKB_MODE_FP32_BULK (each element's arithmetic is the same in both runs;
only the order of the interface sums differs), and every part's copy of an
interface node equal to the others' bit for bit."""
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
        g = dm.get_field(f)
        e = _rel(g, np.array(whole.getField(f)))
        assert e <= 1e-10, (f, e)
        for p, b in zip(dm.parts, dm.backends):
            assert np.array_equal(b.get_field(f), g[p.nodes]), f  # copies equal the owner's
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


@pytest.mark.parametrize("nslabs", [2, 3])
def test_bar_slabs_match_whole_bar(nslabs):
    """The bench's weak-scaled layout: the bar built slab by slab
    (configs.bar_tet4_slabs), against the whole bar in one FP64 model."""
    from akantu_b200.model import SolidMechanicsModel, material_from_dict
    n = 8
    w = configs.bar_tet4(n, nslabs)
    whole = SolidMechanicsModel(w["mesh"], [material_from_dict(m) for m in w["materials"]],
                                precision=_abi.MODE_FP64)
    whole.initFull()

    class F:
        set = whole.setField
        set_blocked = whole.setBlockedDOFs
        stable_time_step = whole.getStableTimeStep
        set_time_step = whole.setTimeStep
    dt = configs.setup_model(F, w)
    whole.solveSteps(STEPS)
    s = configs.bar_tet4_slabs(n, nslabs, range(nslabs))
    dm = DistributedModel(None, s["materials"], nslabs, precision=_abi.MODE_FP64,
                          parts=s["parts"], nb_nodes=s["nb_nodes"])
    dm.set_blocked(s["blocked"])
    dm.set_field(_abi.FIELD_VELOCITY, s["v0"])
    assert s["dt_factor"] * dm.stable_time_step() == dt
    dm.set_time_step(dt)
    dm.solve_steps(STEPS)
    for f in (_abi.FIELD_DISPLACEMENT, _abi.FIELD_VELOCITY):
        e = _rel(dm.get_field(f), np.array(whole.getField(f)))
        assert e <= 1e-10, (f, e)
    dm.close()
    whole.close()


def test_exchange_plan_is_checked():
    import ctypes as C
    from akantu_b200._lib import lib
    w = _workload()
    dm = DistributedModel(w["mesh"], w["materials"], 2, precision=_abi.MODE_FP64)
    b, x = dm.backends[0], dm.plans[0]
    L = lib()
    i64 = C.POINTER(C.c_int64)

    def call(rows, n_recv, ptr, src):
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        ptr = np.ascontiguousarray(ptr, dtype=np.int64)
        src = np.ascontiguousarray(src, dtype=np.int64)
        return L.akb_part_set_exchange(b.m.handle, len(rows),
                                       rows.ctypes.data_as(C.POINTER(C.c_uint32)), n_recv,
                                       ptr.ctypes.data_as(i64), src.ctypes.data_as(i64))
    assert call(x.send_rows, x.n_recv, x.sum_ptr, x.sum_src) == _abi.AKB_OK
    bad_row = x.send_rows.copy()
    bad_row[0] = len(dm.parts[0].iface_local)  # one past the last interface row
    assert call(bad_row, x.n_recv, x.sum_ptr, x.sum_src) == _abi.AKB_ERR_INVALID_ARGUMENT
    no_own = x.sum_src.copy()
    no_own[no_own == -1] = 0  # no row sums its own value
    assert call(x.send_rows, x.n_recv, x.sum_ptr, no_own) == _abi.AKB_ERR_INVALID_ARGUMENT
    far = x.sum_src.copy()
    far[far >= 0] = x.n_recv  # a received row past the buffer
    assert call(x.send_rows, x.n_recv, x.sum_ptr, far) == _abi.AKB_ERR_INVALID_ARGUMENT
    dm.close()
