"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline leg. The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from akantu_b200 import _abi
from akantu_b200.mesh import element_properties

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(fast=False):
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(_HERE, "_build", name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.oracle_create.restype = P
    lib.oracle_create.argtypes = [C.POINTER(_abi.MeshDesc), C.c_int32,
                                  C.POINTER(_abi.MaterialDesc), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_int32)]
    lib.oracle_destroy.argtypes = [P]
    lib.oracle_field.restype = C.POINTER(C.c_double)
    lib.oracle_field.argtypes = [P, C.c_int32]
    lib.oracle_field_size.restype = C.c_int64
    lib.oracle_field_size.argtypes = [P, C.c_int32]
    lib.oracle_blocked.restype = C.POINTER(C.c_uint8)
    lib.oracle_blocked.argtypes = [P]
    for fn in ("oracle_assemble_mass_lumped", "oracle_solve_step",
               "oracle_assemble_internal_forces", "oracle_compute_stresses"):
        getattr(lib, fn).argtypes = [P]
    lib.oracle_stable_time_step.restype = C.c_double
    lib.oracle_stable_time_step.argtypes = [P]
    lib.oracle_set_time_step.argtypes = [P, C.c_double]
    lib.oracle_set_threads.argtypes = [P, C.c_int32]
    lib.oracle_solve_steps.argtypes = [P, C.c_int64]
    lib.oracle_energy.restype = C.c_double
    lib.oracle_energy.argtypes = [P, C.c_int32]
    lib.oracle_time_steps.restype = C.c_double
    lib.oracle_time_steps.argtypes = [P, C.c_int64]
    _LIBS[name] = lib
    return lib


def material_desc(kind=_abi.MATERIAL_ELASTIC, rho=1.0, E=1.0, nu=0.0,
                  plane_stress=False, finite_deformation=False):
    return _abi.MaterialDesc(kind, int(plane_stress), int(finite_deformation), 0,
                             float(rho), float(E), float(nu))


class OracleModel:
    """FP64 CPU restatement of SolidMechanicsModel on the explicit path."""

    def __init__(self, mesh, materials, element_material=None, fast=False):
        self.lib = _lib(fast)
        self.mesh = mesh
        self.dim, self.nnpe, self.nqp = element_properties(mesh.element_type)
        self._nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64)
        self._conn = np.ascontiguousarray(mesh.connectivity, dtype=np.uint32)
        desc = _abi.MeshDesc(mesh.spatial_dimension, mesh.element_type,
                             self._nodes.shape[0], self._conn.shape[0],
                             self._nodes.ctypes.data_as(C.POINTER(C.c_double)),
                             self._conn.ctypes.data_as(C.POINTER(C.c_uint32)))
        if isinstance(materials, _abi.MaterialDesc):
            materials = [materials]
        mats = (_abi.MaterialDesc * len(materials))(*materials)
        em = None
        if element_material is not None:
            self._em = np.ascontiguousarray(element_material, dtype=np.uint32)
            em = self._em.ctypes.data_as(C.POINTER(C.c_uint32))
        status = C.c_int32(0)
        self.h = self.lib.oracle_create(C.byref(desc), len(materials), mats, em,
                                        C.byref(status))
        if not self.h:
            raise RuntimeError("oracle_create failed: %s" % _abi.STATUS_NAMES[status.value])

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
            self.h = None

    def field(self, field):
        """numpy view on the model-owned array (writable)."""
        n = self.lib.oracle_field_size(self.h, field)
        p = self.lib.oracle_field(self.h, field)
        arr = np.ctypeslib.as_array(p, shape=(n,))
        if field in (_abi.FIELD_GRAD_U, _abi.FIELD_STRESS):
            return arr.reshape(-1, self.dim * self.dim)
        return arr.reshape(-1, self.dim)

    @property
    def displacement(self):
        return self.field(_abi.FIELD_DISPLACEMENT)

    @property
    def velocity(self):
        return self.field(_abi.FIELD_VELOCITY)

    @property
    def acceleration(self):
        return self.field(_abi.FIELD_ACCELERATION)

    @property
    def internal_force(self):
        return self.field(_abi.FIELD_INTERNAL_FORCE)

    @property
    def external_force(self):
        return self.field(_abi.FIELD_EXTERNAL_FORCE)

    @property
    def mass(self):
        return self.field(_abi.FIELD_MASS)

    @property
    def blocked(self):
        n = self._nodes.shape[0] * self.dim
        return np.ctypeslib.as_array(self.lib.oracle_blocked(self.h),
                                     shape=(n,)).reshape(-1, self.dim)

    def assemble_mass_lumped(self):
        self.lib.oracle_assemble_mass_lumped(self.h)

    def stable_time_step(self):
        return self.lib.oracle_stable_time_step(self.h)

    def set_time_step(self, dt):
        self.lib.oracle_set_time_step(self.h, dt)

    def set_threads(self, n):
        self.lib.oracle_set_threads(self.h, n)

    def solve_step(self):
        self.lib.oracle_solve_step(self.h)

    def solve_steps(self, n):
        self.lib.oracle_solve_steps(self.h, n)

    def assemble_internal_forces(self):
        self.lib.oracle_assemble_internal_forces(self.h)

    def compute_stresses(self):
        self.lib.oracle_compute_stresses(self.h)

    def energy(self, kind):
        return self.lib.oracle_energy(self.h, kind)

    def time_steps(self, n):
        return self.lib.oracle_time_steps(self.h, n)


# ---------------------------------------------------------------- FE^2 (RVE)
def _fe2_lib():
    lib = _lib()
    if getattr(lib, "_fe2_ready", False):
        return lib
    D, I32 = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    U8 = C.POINTER(C.c_uint8)
    lib.oracle_rve_solve.restype = C.c_int32
    lib.oracle_rve_solve.argtypes = [C.c_int32, C.c_double, U8, C.c_int32, D, D, I32, D, D,
                                     C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                     D, D]
    lib.oracle_rve_parameters.argtypes = [C.c_int32, C.c_double, C.c_int32, D, D, I32, D,
                                          C.c_double, C.c_double, D, D]
    lib.oracle_rve_stress.argtypes = [C.c_int32, C.c_double, U8, D, D, I32, D, D, D, D]
    lib._fe2_ready = True
    return lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class OracleRVE:
    """FP64 periodic voxel RVE (oracle/akb_fe2_oracle.cc)."""

    def __init__(self, cells, length, voxel_material, lambdas, mus, kinds):
        self.n = int(cells)
        self.L = float(length)
        self.vm = np.ascontiguousarray(voxel_material, dtype=np.uint8).ravel()
        assert self.vm.size == self.n ** 3
        self.lam = np.ascontiguousarray(lambdas, dtype=np.float64)
        self.mu = np.ascontiguousarray(mus, dtype=np.float64)
        self.kind = np.ascontiguousarray(kinds, dtype=np.int32)
        self.lib = _fe2_lib()

    def _H(self, grad_u):
        return np.ascontiguousarray(np.asarray(grad_u, dtype=np.float64).reshape(3, 3).T.ravel())

    def parameters(self, grad_u, time_step_factor=0.5, damping_factor=1.0):
        dt, cd = C.c_double(), C.c_double()
        H = self._H(grad_u)
        self.lib.oracle_rve_parameters(self.n, self.L, len(self.lam), _p(self.lam, C.c_double),
                                       _p(self.mu, C.c_double), _p(self.kind, C.c_int32),
                                       _p(H, C.c_double), time_step_factor, damping_factor,
                                       C.byref(dt), C.byref(cd))
        return dt.value, cd.value

    def solve(self, grad_u, fluct=None, max_iterations=2000, check_interval=10, tolerance=1e-4,
              time_step_factor=0.5, damping_factor=1.0):
        """grad_u: 3x3 (row i, column j = du_i/dX_j). Returns (P 3x3, fluct,
        iterations, residual)."""
        H = self._H(grad_u)
        w = np.zeros((self.n ** 3, 3)) if fluct is None else np.array(fluct, dtype=np.float64)
        w = np.ascontiguousarray(w)
        P = np.zeros(9)
        r = C.c_double()
        it = self.lib.oracle_rve_solve(self.n, self.L, _p(self.vm, C.c_uint8), len(self.lam),
                                       _p(self.lam, C.c_double), _p(self.mu, C.c_double),
                                       _p(self.kind, C.c_int32), _p(H, C.c_double),
                                       _p(w, C.c_double), max_iterations, check_interval,
                                       tolerance, time_step_factor, damping_factor,
                                       _p(P, C.c_double), C.byref(r))
        return P.reshape(3, 3).T.copy(), w, it, r.value

    def stress(self, grad_u, fluct):
        H = self._H(grad_u)
        w = np.ascontiguousarray(fluct, dtype=np.float64)
        P = np.zeros(9)
        f = np.zeros((self.n ** 3, 3))
        self.lib.oracle_rve_stress(self.n, self.L, _p(self.vm, C.c_uint8), _p(self.lam, C.c_double),
                                   _p(self.mu, C.c_double), _p(self.kind, C.c_int32),
                                   _p(H, C.c_double), _p(w, C.c_double), _p(P, C.c_double),
                                   _p(f, C.c_double))
        return P.reshape(3, 3).T.copy(), f


# ----------------------------------------------------------------- FE^2 (MLP)
def _mlp_lib():
    lib = _fe2_lib()
    if getattr(lib, "_mlp_ready", False):
        return lib
    D, F = C.POINTER(C.c_double), C.POINTER(C.c_float)
    lib.oracle_mlp_forward.argtypes = [C.c_int32] * 4 + [F, F, C.c_int64, D, D, C.c_int32]
    lib.oracle_mlp_gradients.restype = C.c_double
    lib.oracle_mlp_gradients.argtypes = [C.c_int32] * 4 + [F, F, C.c_int64, D, D, D, C.c_int32]
    lib._mlp_ready = True
    return lib


class OracleMLP:
    """FP64 twin of the tensor-core MLP (oracle/akb_fe2_oracle.cc)."""

    def __init__(self, nin, nout, width, nhidden, params, in_shift=None, in_scale=None,
                 out_shift=None, out_scale=None):
        self.shape = (nin, nout, width, nhidden)
        self.params = np.ascontiguousarray(params, dtype=np.float32)
        z = lambda n, v: np.full(n, v, np.float32)
        self.scaling = np.ascontiguousarray(np.concatenate([
            z(nin, 0) if in_shift is None else np.asarray(in_shift, np.float32),
            z(nin, 1) if in_scale is None else np.asarray(in_scale, np.float32),
            z(nout, 0) if out_shift is None else np.asarray(out_shift, np.float32),
            z(nout, 1) if out_scale is None else np.asarray(out_scale, np.float32)]))
        self.lib = _mlp_lib()

    def forward(self, x, emulate_bf16=True):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros((x.shape[0], self.shape[1]))
        self.lib.oracle_mlp_forward(*self.shape, _p(self.params, C.c_float),
                                    _p(self.scaling, C.c_float), x.shape[0], _p(x, C.c_double),
                                    _p(y, C.c_double), int(emulate_bf16))
        return y

    def gradients(self, x, target, emulate_bf16=True):
        x = np.ascontiguousarray(x, dtype=np.float64)
        t = np.ascontiguousarray(target, dtype=np.float64)
        g = np.zeros(self.params.size)
        loss = self.lib.oracle_mlp_gradients(*self.shape, _p(self.params, C.c_float),
                                             _p(self.scaling, C.c_float), x.shape[0],
                                             _p(x, C.c_double), _p(t, C.c_double),
                                             _p(g, C.c_double), int(emulate_bf16))
        return loss, g
