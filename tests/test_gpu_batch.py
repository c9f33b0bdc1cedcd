"""Batches of independent plates (akb_batch_create) against one model per
plate and against the oracle."""
import numpy as np
import pytest

from akantu_b200 import _abi, configs
from akantu_b200.batch import BatchModel
from akantu_b200.model import SolidMechanicsModel, material_from_dict
from tests.golden_cases import OracleAdapter

pytestmark = pytest.mark.gpu

STATE = (_abi.FIELD_DISPLACEMENT, _abi.FIELD_VELOCITY, _abi.FIELD_ACCELERATION)


def small_batch(n=12):
    return configs.plates_batch(n_instances=n, seed=7, min_elems=100, max_elems=3000)


def single_model(w, k, mode, opts):
    m = SolidMechanicsModel(w["meshes"][k], [material_from_dict(w["materials"][k])],
                            precision=mode, **opts)
    m.initFull()
    m.setBlockedDOFs(w["blocked"][k])
    m.setField(_abi.FIELD_DISPLACEMENT, w["u0"][k])
    return m


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_FP32_BULK])
@pytest.mark.parametrize("grid", [0, 7])
def test_batch_equals_one_model_per_plate(mode, grid):
    w = small_batch()
    opts = dict(patch_elements=512, patch_nodes=320)
    b = BatchModel(w["meshes"], w["materials"], precision=mode, patch_grid=grid, **opts)
    b.initFull()
    dts = configs.setup_batch(b, w)
    b.solveSteps(150)
    got = {f: b.getField(f) for f in STATE}
    for k in range(len(w["meshes"])):
        m = single_model(w, k, mode, opts)
        dt = m.getStableTimeStep()
        assert dt * w["dt_factor"] == dts[k]
        m.setTimeStep(dts[k])
        m.solveSteps(150)
        rows = b.instance_rows(k)
        for f in STATE:
            assert np.array_equal(got[f][rows], m.getField(f)), (k, f)
        m.close()


def test_batch_matches_oracle_and_energies():
    w = small_batch(6)
    b = BatchModel(w["meshes"], w["materials"], precision=_abi.MODE_FP64)
    b.initFull()
    dts = configs.setup_batch(b, w)
    b.solveSteps(200)
    u = b.getField(_abi.FIELD_DISPLACEMENT)
    ek = b.getEnergies("kinetic")
    ep = b.getEnergies("potential")
    for k in range(len(w["meshes"])):
        cpu = OracleAdapter(w["meshes"][k], w["materials"][k])
        cpu.set_blocked(w["blocked"][k])
        cpu.set(_abi.FIELD_DISPLACEMENT, w["u0"][k])
        assert w["dt_factor"] * cpu.stable_time_step() == dts[k]
        cpu.set_time_step(dts[k])
        cpu.solve_steps(200)
        ref = cpu.get(_abi.FIELD_DISPLACEMENT)
        rows = b.instance_rows(k)
        assert np.abs(u[rows] - ref).max() <= 1e-10 * np.abs(ref).max()
        assert ek[k] == pytest.approx(cpu.energy(_abi.ENERGY_KINETIC), rel=1e-10)
        assert ep[k] == pytest.approx(cpu.energy(_abi.ENERGY_POTENTIAL), rel=1e-10)


def test_models_with_different_patch_sizes_coexist():
    """The kernel's shared-memory limit is process-wide: a model built after
    another with smaller patches must not break the first one's launches."""
    w = small_batch(8)
    sizes = [m.getNbElement() for m in w["meshes"]]
    big, small = int(np.argmax(sizes)), int(np.argmin(sizes))
    opts = dict(patch_elements=2048, patch_nodes=1100)
    a = single_model(w, big, _abi.MODE_FP64, opts)
    a.setTimeStep(w["dt_factor"] * a.getStableTimeStep())
    b = single_model(w, small, _abi.MODE_FP64, dict(patch_elements=128, patch_nodes=100))
    b.setTimeStep(w["dt_factor"] * b.getStableTimeStep())
    a.solveSteps(40)
    b.solveSteps(40)
    ref = single_model(w, big, _abi.MODE_FP64, opts)
    ref.setTimeStep(w["dt_factor"] * ref.getStableTimeStep())
    ref.solveSteps(40)
    assert np.array_equal(a.getDisplacement(), ref.getDisplacement())
    for m in (a, b, ref):
        m.close()


def test_batch_rejects_reference_mode_and_mixed_types():
    from akantu_b200._lib import AkbError
    w = small_batch(2)
    b = BatchModel(w["meshes"], w["materials"], precision=_abi.MODE_FP64_REFERENCE)
    with pytest.raises(AkbError):
        b.initFull()
