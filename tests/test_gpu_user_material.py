"""User materials (AKB_MATERIAL_USER): the step split around
Material::computeStress, with stresses written by the caller on the device,
against the built-in laws and against homogeneous RVEs."""
import numpy as np
import pytest

from akantu_b200 import _abi, configs
from akantu_b200._lib import AkbError, lib
from akantu_b200.mesh import block_hexahedron8
from akantu_b200.model import (MaterialElastic, MaterialNeohookean, MaterialUser,
                               SolidMechanicsModel)
from tests.fe2_cases import lame

pytestmark = pytest.mark.gpu


class TorchNeohookean(MaterialUser):
    def __init__(self, rho, E, nu):
        super().__init__(rho=rho, E=E, nu=nu, finite_deformation=True)
        self.lam, self.mu = lame(dict(E=E, nu=nu))

    def computeStress(self, grad_u, stress):
        import torch
        eye = torch.eye(3, dtype=grad_u.dtype, device=grad_u.device)
        F = eye + grad_u
        Cm = F.transpose(1, 2) @ F
        Ci = torch.linalg.inv(Cm)
        J = torch.linalg.det(F)
        S = self.mu * (eye - Ci) + (self.lam * torch.log(J))[:, None, None] * Ci
        stress.copy_(F @ S)


class TorchElastic(MaterialUser):
    def __init__(self, rho, E, nu):
        super().__init__(rho=rho, E=E, nu=nu, finite_deformation=False)
        self.lam, self.mu = lame(dict(E=E, nu=nu))

    def computeStress(self, grad_u, stress):
        import torch
        eye = torch.eye(3, dtype=grad_u.dtype, device=grad_u.device)
        tr = grad_u.diagonal(dim1=1, dim2=2).sum(-1)
        stress.copy_(self.mu * (grad_u + grad_u.transpose(1, 2)) + self.lam * tr[:, None, None] * eye)


class RveMaterial(MaterialUser):
    """Stresses from homogeneous periodic RVEs (the FE^2 coupling with a
    trivial microstructure)."""

    def __init__(self, rho, E, nu):
        super().__init__(rho=rho, E=E, nu=nu, finite_deformation=True)
        from akantu_b200.rve import SolidMechanicsModelRVE
        mat = dict(kind=_abi.MATERIAL_NEOHOOKEAN, rho=rho, E=E, nu=nu)
        self.rve = SolidMechanicsModelRVE(2, np.zeros(8, np.uint8), [mat],
                                          precision=_abi.MODE_FP64)

    def computeStress(self, grad_u, stress):
        out = self.rve.solve(grad_u)
        assert int(out["iterations"].max()) == 0
        stress.copy_(out["stress"])


def run_pair(mesh, builtin, user, blocked, v0, steps):
    res = []
    for mat in (builtin, user):
        m = SolidMechanicsModel(mesh, [mat], precision=_abi.MODE_FP64)
        m.initFull()
        m.setBlockedDOFs(blocked)
        m.setField(_abi.FIELD_VELOCITY, v0)
        dt = 0.5 * m.getStableTimeStep()
        m.setTimeStep(dt)
        m.solveSteps(steps)
        res.append((m.getDisplacement().copy(), m.getVelocity().copy(),
                    m.getInternalForce().copy()))
        m.close()
    return res


def test_user_neohookean_equals_builtin():
    w = configs.block_hex8(4, 0.04)
    mesh = w["mesh"]
    p = w["materials"][0]
    (u0, v0_, f0), (u1, v1, f1) = run_pair(
        mesh, MaterialNeohookean(rho=p["rho"], E=p["E"], nu=p["nu"]),
        TorchNeohookean(p["rho"], p["E"], p["nu"]), w["blocked"], w["v0"], 60)
    assert np.abs(u1 - u0).max() <= 1e-11 * np.abs(u0).max()
    assert np.abs(v1 - v0_).max() <= 1e-10 * np.abs(v0_).max()
    assert np.abs(f1 - f0).max() <= 1e-9 * np.abs(f0).max()


def test_user_small_strain_equals_builtin():
    w = configs.cube_tet4(4)
    p = w["materials"][0]
    (u0, _, _), (u1, _, _) = run_pair(
        w["mesh"], MaterialElastic(rho=p["rho"], E=p["E"], nu=p["nu"]),
        TorchElastic(p["rho"], p["E"], p["nu"]), w["blocked"], w["v0"], 60)
    assert np.abs(u1 - u0).max() <= 1e-11 * np.abs(u0).max()


def test_homogeneous_rve_material_equals_builtin():
    w = configs.block_hex8(3, 0.03)
    p = w["materials"][0]
    (u0, _, _), (u1, _, _) = run_pair(
        w["mesh"], MaterialNeohookean(rho=p["rho"], E=p["E"], nu=p["nu"]),
        RveMaterial(p["rho"], p["E"], p["nu"]), w["blocked"], w["v0"], 30)
    assert np.abs(u1 - u0).max() <= 1e-10 * np.abs(u0).max()


def test_user_model_errors():
    mesh = block_hexahedron8(2, 1.0)
    mat = TorchNeohookean(1000.0, 1e6, 0.3)
    m = SolidMechanicsModel(mesh, [mat], precision=_abi.MODE_FP64)
    m.initFull()
    m.setTimeStep(1e-6)
    L = lib()
    assert L.akb_solve_steps(m.handle, 2) == _abi.AKB_ERR_STATE
    assert L.akb_step_end(m.handle) == _abi.AKB_ERR_STATE
    assert L.akb_step_begin(m.handle) == _abi.AKB_OK
    assert L.akb_step_begin(m.handle) == _abi.AKB_ERR_STATE
    assert L.akb_step_end(m.handle) == _abi.AKB_OK
    m.close()
    for precision in (_abi.MODE_FP32_BULK, _abi.MODE_FP64_REFERENCE):
        with pytest.raises(AkbError):
            SolidMechanicsModel(mesh, [mat], precision=precision).initFull()
    with pytest.raises(AkbError):  # user and built-in materials mixed
        SolidMechanicsModel(mesh, [mat, MaterialElastic(rho=1.0, E=1.0)],
                            element_material=np.zeros(8, np.uint32),
                            precision=_abi.MODE_FP64).initFull()
