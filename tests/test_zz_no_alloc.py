"""akb_kinetic_energy_static: the kinetic energy of a model's device arrays
computed without allocating device memory (for callers that cannot call
cudaMalloc mid-run: inside CUDA stream capture, or under a device-memory
budget owned by another allocator). Checked against akb_get_energy on two
consecutive calls. Collected last so that a failure here leaves every other
test already run."""
import ctypes as C

import numpy as np
import pytest

from akantu_b200 import _abi, configs
from tests.golden_cases import GpuAdapter

pytestmark = pytest.mark.gpu


def static_kinetic(model, out_tensor):
    from akantu_b200._lib import check, lib
    L = lib()
    dim = model.m.dim
    nn = model.m.mesh.getNbNodes()
    mass = model.m.devicePointer(_abi.FIELD_MASS)
    vel = model.m.devicePointer(_abi.FIELD_VELOCITY)
    model.m.synchronize()
    check(L.akb_kinetic_energy_static(C.c_void_p(mass), C.c_void_p(vel), nn, dim,
                                      C.c_void_p(out_tensor.data_ptr()), None))
    import torch
    torch.cuda.synchronize()
    return float(out_tensor.item())


def test_static_kinetic_energy_matches_model_on_two_calls():
    import torch
    w = configs.cube_tet4(n=10)
    model = GpuAdapter(w["mesh"], w["materials"], precision=_abi.MODE_FP64)
    configs.setup_model(model, w)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    results = []
    for steps in (7, 13):
        model.solve_steps(steps)
        ref = model.energy(_abi.ENERGY_KINETIC)
        got = static_kinetic(model, out)
        assert ref > 0
        assert abs(got - ref) <= 1e-12 * ref, (got, ref)
        results.append(got)
    assert results[0] != results[1]  # the second call saw the new state


def test_static_kinetic_energy_rejects_oversize():
    from akantu_b200._lib import lib
    L = lib()
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = L.akb_kinetic_energy_static(dummy, dummy, 8388609, 3, dummy, None)
    assert st == _abi.AKB_ERR_INVALID_ARGUMENT
    assert b"8388608" in L.akb_last_error()
