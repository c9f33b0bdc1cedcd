"""B200-native explicit central-difference dynamics with lumped mass.

A drop-in for Akantu's SolidMechanicsModel explicit path
(initFull(_analysis_method=_explicit_lumped_mass) / solveStep /
Material::computeStress) on one GPU. The compute runs in libakb.so
(hand-written CUDA for sm_100a) behind the C ABI of include/akb.h.
"""
from . import _abi
from ._abi import (MODE_FP32_BULK, MODE_FP64, MODE_FP64_REFERENCE, HEXAHEDRON_8,
                   SEGMENT_2, TETRAHEDRON_4, TRIANGLE_3)
from .mesh import Mesh
from .model import (MaterialElastic, MaterialNeohookean, MaterialUser, SolidMechanicsModel,
                    _explicit_lumped_mass)

_segment_2 = SEGMENT_2
_triangle_3 = TRIANGLE_3
_tetrahedron_4 = TETRAHEDRON_4
_hexahedron_8 = HEXAHEDRON_8

__all__ = ["Mesh", "SolidMechanicsModel", "MaterialElastic", "MaterialNeohookean", "MaterialUser",
           "_explicit_lumped_mass", "MODE_FP64_REFERENCE", "MODE_FP64", "MODE_FP32_BULK"]
