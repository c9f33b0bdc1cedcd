"""Edge cases of the explicit path against the oracle: a node that belongs
to no element (lumped mass 0: the reference's r / M is not finite,
solid_mechanics_model_mass.cc:79-95), a mesh without elements, and a blocked
node with zero mass (untouched, like every blocked DOF)."""
import numpy as np
import pytest

from akantu_b200 import _abi, configs
from akantu_b200.mesh import Mesh
from tests.golden_cases import GpuAdapter, OracleAdapter

pytestmark = pytest.mark.gpu


def plate_with_orphan():
    w = configs.plate_tri3(nx=10, ny=3, lx=1.0, ly=0.3)
    m = w["mesh"]
    nodes = np.vstack([m.nodes, [[2.0, 2.0]]])
    mesh = Mesh(2, m.element_type, nodes, m.connectivity)
    w["mesh"] = mesh
    for k in ("blocked", "u0", "v0"):
        w[k] = np.vstack([w[k], np.zeros((1, 2), dtype=w[k].dtype)])
    w["v0"][-1] = [0.1, -0.2]
    return w


@pytest.mark.parametrize("mode", [_abi.MODE_FP64_REFERENCE, _abi.MODE_FP64, _abi.MODE_FP32_BULK])
def test_orphan_node_follows_the_reference(mode):
    w = plate_with_orphan()
    cpu = OracleAdapter(w["mesh"], w["materials"])
    dt = configs.setup_model(cpu, w)
    cpu.solve_steps(20)
    dev = GpuAdapter(w["mesh"], w["materials"], precision=mode)
    configs.setup_model(dev, w)
    dev.set_time_step(dt)
    dev.solve_steps(20)
    for f in (_abi.FIELD_DISPLACEMENT, _abi.FIELD_VELOCITY, _abi.FIELD_ACCELERATION):
        a, b = dev.get(f), cpu.get(f)
        # the orphan node: not finite in both
        assert not np.isfinite(b[-1]).all()
        assert np.array_equal(np.isfinite(a), np.isfinite(b))
        tol = {0: 0.0, 1: 1e-10, 2: 2e-4}[mode]
        ok = np.isfinite(b)
        assert np.abs(a[ok] - b[ok]).max() <= tol * np.abs(b[ok]).max() + 1e-300


def test_blocked_orphan_node_is_untouched():
    w = plate_with_orphan()
    w["blocked"][-1] = 1
    dev = GpuAdapter(w["mesh"], w["materials"], precision=_abi.MODE_FP64)
    configs.setup_model(dev, w)
    dev.solve_steps(10)
    assert np.array_equal(dev.get(_abi.FIELD_VELOCITY)[-1], w["v0"][-1])
    assert np.isfinite(dev.get(_abi.FIELD_DISPLACEMENT)).all()


def test_mesh_without_elements():
    from akantu_b200.model import MaterialElastic, SolidMechanicsModel
    mesh = Mesh(3, _abi.TETRAHEDRON_4, np.zeros((4, 3)), np.zeros((0, 4), np.uint32))
    m = SolidMechanicsModel(mesh, [MaterialElastic(rho=1.0, E=1.0, nu=0.2)],
                            precision=_abi.MODE_FP64)
    m.initFull()
    assert m.getInfo().nb_elements == 0
    assert np.abs(m.getMass()).max() == 0.0
    m.setTimeStep(1e-3)
    m.solveSteps(3)
    m.close()


def test_dirichlet_arrays_reusable_on_return():
    """akb_apply_dirichlet queues its update without waiting for it: the
    caller's arrays are copied before the call returns, so overwriting them
    at once changes nothing; more calls than staging slots, of growing sizes,
    in a row."""
    import ctypes as C

    from akantu_b200._lib import check, lib
    from akantu_b200.model import SolidMechanicsModel, material_from_dict
    w = configs.plate_tri3(nx=40, ny=8, lx=1.0, ly=0.2)
    m = SolidMechanicsModel(w["mesh"], [material_from_dict(mm) for mm in w["materials"]],
                            precision=_abi.MODE_FP64)
    m.initFull()
    nn = w["mesh"].nodes.shape[0]
    rng = np.random.default_rng(3)
    expect_u = np.zeros((nn, 2))
    expect_b = np.zeros((nn, 2), dtype=np.uint8)
    for call in range(11):
        nodes = rng.choice(nn, size=5 + 20 * call, replace=False).astype(np.uint32)
        vals = rng.normal(size=nodes.size)
        comp = call % 2
        expect_u[nodes, comp] = vals
        expect_b[nodes, comp] = 1
        check(lib().akb_apply_dirichlet(m.handle, nodes.ctypes.data_as(C.POINTER(C.c_uint32)),
                                        nodes.size, comp,
                                        vals.ctypes.data_as(C.POINTER(C.c_double))))
        nodes[:] = 0            # the caller reuses its arrays right away
        vals[:] = np.nan
    u = np.array(m.getDisplacement())
    b = np.array(m.getBlockedDOFs(), dtype=np.uint8).reshape(-1, 2)
    assert np.array_equal(b, expect_b)
    assert np.array_equal(u[expect_b.astype(bool)], expect_u[expect_b.astype(bool)])
    m.close()


def test_dirichlet_all_components_and_async_energy():
    """akb_apply_dirichlet with AKB_ALL_COMPONENTS equals one call per
    component; akb_get_energy_async gives akb_get_energy's value once the
    stream is synchronised, for every step of a loop queued without
    waiting."""
    import torch

    from akantu_b200.model import SolidMechanicsModel, material_from_dict
    w = configs.cube_tet4(8)
    fixed = np.nonzero(w["blocked"][:, 0])[0]
    vals = np.random.default_rng(5).normal(scale=1e-6, size=(fixed.size, 3))
    runs = []
    for all_at_once in (True, False):
        m = SolidMechanicsModel(w["mesh"], [material_from_dict(mm) for mm in w["materials"]],
                                precision=_abi.MODE_FP64)
        m.initFull()
        m.setField(_abi.FIELD_VELOCITY, w["v0"])
        m.setTimeStep(0.8 * m.getStableTimeStep())
        slots = torch.zeros(20, dtype=torch.float64).pin_memory()
        sync_e = []
        for s in range(20):
            if all_at_once:
                m.applyDirichlet(fixed, _abi.ALL_COMPONENTS, vals * (s + 1))
            else:
                for c in range(3):
                    m.applyDirichlet(fixed, c, vals[:, c] * (s + 1))
            m.solveStep()
            if all_at_once:
                m.getEnergyAsync("kinetic", slots[s:s + 1].data_ptr())
            else:
                sync_e.append(m.getEnergy("kinetic"))
        m.synchronize()
        runs.append((np.array(m.getDisplacement()), slots.numpy().copy(), sync_e))
        m.close()
    (u1, e_async, _), (u2, _, e_sync) = runs
    assert np.array_equal(u1, u2)
    assert np.array_equal(e_async, np.array(e_sync))
