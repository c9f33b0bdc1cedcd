"""Loads libakb.so (built in-tree by akantu_b200/csrc/Makefile) and declares
the C signatures of include/akb.h. There is no fallback: if the library is
missing or fails to load, every model call raises."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libakb.so")
_lib = None

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
DBL = C.c_double
PD = C.POINTER(C.c_double)
PU8 = C.POINTER(C.c_uint8)
PU32 = C.POINTER(C.c_uint32)

# name -> (restype, argtypes); the exported surface of include/akb.h
SIGNATURES = {
    "akb_abi_version": (I32, []),
    "akb_last_error": (C.c_char_p, []),
    "akb_model_create": (I32, [C.POINTER(_abi.MeshDesc), I32, C.POINTER(_abi.MaterialDesc),
                               PU32, C.POINTER(_abi.ModelOptions), C.POINTER(P)]),
    "akb_model_destroy": (I32, [P]),
    "akb_model_get_info": (I32, [P, C.POINTER(_abi.ModelInfo)]),
    "akb_set_field": (I32, [P, I32, PD, I64]),
    "akb_get_field": (I32, [P, I32, PD, I64]),
    "akb_field_device_pointer": (I32, [P, I32, C.POINTER(P)]),
    "akb_get_node_numbering": (I32, [P, PU32, I64]),
    "akb_set_blocked_dofs": (I32, [P, PU8, I64]),
    "akb_get_blocked_dofs": (I32, [P, PU8, I64]),
    "akb_assemble_mass_lumped": (I32, [P]),
    "akb_get_stable_time_step": (I32, [P, PD]),
    "akb_set_time_step": (I32, [P, DBL]),
    "akb_get_time_step": (I32, [P, PD]),
    "akb_solve_step": (I32, [P]),
    "akb_solve_steps": (I32, [P, I64]),
    "akb_time_solve_steps": (I32, [P, I64, PD]),
    "akb_assemble_internal_forces": (I32, [P]),
    "akb_compute_stresses": (I32, [P]),
    "akb_get_energy": (I32, [P, I32, PD]),
    "akb_get_energy_async": (I32, [P, I32, P]),
    "akb_apply_dirichlet": (I32, [P, PU32, I64, I32, PD]),
    "akb_time_kernels": (I32, [P, I64, PD, I32]),
    "akb_kernel_name": (C.c_char_p, [P, I32]),
    "akb_batch_create": (I32, [C.POINTER(_abi.BatchDesc), C.POINTER(_abi.ModelOptions),
                               C.POINTER(P)]),
    "akb_batch_get_layout": (I32, [P, C.POINTER(I32), C.POINTER(I64), C.POINTER(I64)]),
    "akb_batch_set_time_steps": (I32, [P, PD]),
    "akb_batch_get_stable_time_steps": (I32, [P, PD]),
    "akb_batch_get_energies": (I32, [P, I32, PD]),
    "akb_kinetic_energy_static": (I32, [P, P, I64, I32, P, P]),
    "akb_synchronize": (I32, [P]),
    "akb_model_create_part": (I32, [C.POINTER(_abi.MeshDesc), I32, C.POINTER(_abi.MaterialDesc),
                                    PU32, C.POINTER(_abi.ModelOptions), PU32, I64,
                                    C.POINTER(P)]),
    "akb_part_step_begin": (I32, [P]),
    "akb_part_export_forces": (I32, [P, P]),
    "akb_part_step_end": (I32, [P, P]),
    "akb_part_export_mass": (I32, [P, P]),
    "akb_part_import_mass": (I32, [P, P]),
    "akb_part_set_exchange": (I32, [P, I64, PU32, I64, C.POINTER(I64), C.POINTER(I64)]),
    "akb_part_pack_forces": (I32, [P, P]),
    "akb_part_step_end_exchange": (I32, [P, P]),
    "akb_part_pack_mass": (I32, [P, P]),
    "akb_part_import_mass_exchange": (I32, [P, P]),
    # include/akb_mesh.h
    "akb_msh_read": (I32, [C.c_char_p, I32, C.POINTER(P)]),
    "akb_msh_parse": (I32, [C.c_char_p, I64, I32, C.POINTER(P)]),
    "akb_msh_destroy": (I32, [P]),
    "akb_msh_get_mesh": (I32, [P, C.POINTER(_abi.MeshDesc)]),
    "akb_msh_get_nb_groups": (I32, [P, C.POINTER(I32)]),
    "akb_msh_get_group": (I32, [P, I32, C.POINTER(C.c_char_p), C.POINTER(I64), C.POINTER(PU32),
                                C.POINTER(I64), C.POINTER(PU32)]),
    "akb_msh_get_group_facets": (I32, [P, I32, C.POINTER(I64), C.POINTER(I32), C.POINTER(PU32)]),
    "akb_neumann_forces": (I32, [I32, I64, C.POINTER(C.c_double), I64, I32, C.POINTER(C.c_uint32),
                                 I32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "akb_facet_points": (I32, [I32]),
    "akb_facet_quadrature": (I32, [I32, I64, C.POINTER(C.c_double), I64, I32,
                                   C.POINTER(C.c_uint32), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    # include/akb_fe2.h
    "akb_step_begin": (I32, [P]),
    "akb_step_end": (I32, [P]),
    "akb_model_get_stream": (I32, [P, C.POINTER(P)]),
    "akb_rve_create": (I32, [C.POINTER(_abi.RveDesc), C.POINTER(_abi.RveOptions), C.POINTER(P)]),
    "akb_rve_destroy": (I32, [P]),
    "akb_rve_get_info": (I32, [P, C.POINTER(_abi.RveInfo)]),
    "akb_rve_solve": (I32, [P, I64, P, P, P, P, P, P]),
    "akb_rve_solve_indexed": (I32, [P, I64, P, P, P, P, P, P, P, P]),
    "akb_rve_stress": (I32, [P, I64, P, P, P, P, P]),
    "akb_mlp_create": (I32, [I32, I32, I32, I32, I32, P, C.POINTER(P)]),
    "akb_mlp_destroy": (I32, [P]),
    "akb_mlp_get_parameter_count": (I32, [P, C.POINTER(I64)]),
    "akb_mlp_set_parameters": (I32, [P, C.POINTER(C.c_float), I64]),
    "akb_mlp_get_parameters": (I32, [P, C.POINTER(C.c_float), I64]),
    "akb_mlp_set_scaling": (I32, [P] + [C.POINTER(C.c_float)] * 4),
    "akb_mlp_forward": (I32, [P, I64, P, P, P]),
    "akb_mlp_stress": (I32, [P, I64, P, P, C.c_double, C.c_double, P, P, P]),
    "akb_mlp_gradients": (I32, [P, I64, P, P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "akb_mlp_train_step": (I32, [P, I64, P, P, C.c_float, C.POINTER(C.c_float)]),
    "akb_mlp_compute_gradients": (I32, [P, I64, P, P, C.POINTER(C.c_float)]),
    "akb_mlp_gradient_device_pointer": (I32, [P, C.POINTER(P)]),
    "akb_mlp_apply_gradients": (I32, [P, C.c_float]),
}


class AkbError(RuntimeError):
    def __init__(self, status, message):
        self.status = status
        super().__init__("%s (%s)" % (message, _abi.STATUS_NAMES.get(status, status)))


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "csrc")], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libakb.so is not built: run `make -C akantu_b200/csrc` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.akb_abi_version() != _abi.ABI_VERSION:
        raise ImportError("libakb.so ABI version mismatch")
    _lib = L
    return L


def check(status):
    if status != _abi.AKB_OK:
        msg = lib().akb_last_error().decode(errors="replace")
        raise AkbError(status, msg)
