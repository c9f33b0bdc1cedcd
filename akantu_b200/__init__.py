"""B200-native explicit central-difference dynamics with lumped mass.

A drop-in for Akantu's SolidMechanicsModel explicit path
(initFull(_analysis_method=_explicit_lumped_mass) / solveStep /
Material::computeStress) on one GPU. The compute runs in libakb.so
(hand-written CUDA for sm_100a) behind the C ABI of include/akb.h.
"""
from . import _abi
from ._abi import (MODE_FP32_BULK, MODE_FP64, MODE_FP64_REFERENCE, HEXAHEDRON_8,
                   SEGMENT_2, TETRAHEDRON_4, TRIANGLE_3)
from .material_plugin import (Material, MaterialFactory, MeshDataMaterialSelectorString, _ghost,
                              _not_ghost, _pat_internal, _pat_modifiable, _pat_parsable,
                              _pat_parsmod, _pat_readable, _pat_writable, parseInput)
from .mesh import Mesh
from .model import (DirichletFunctor, FixedValue, FreeBoundary, FromHigherDim, FromSameDim,
                    FromStress, FromTraction, Increment, IncrementValue, MaterialElastic,
                    MaterialNeohookean, MaterialUser, NeumannFunctor, SolidMechanicsModel,
                    _explicit_lumped_mass, _x, _y, _z)



def initialize(*args, **kwargs):
    """Kept for scripts written against older interfaces: as in the
    reference's Python package, there is nothing to initialise; an input
    file is read with parseInput."""
    raise RuntimeError("initialize is not needed: read an input file with parseInput")


def finalize(*args, **kwargs):
    raise RuntimeError("finalize is not needed")


_segment_2 = SEGMENT_2
_triangle_3 = TRIANGLE_3
_tetrahedron_4 = TETRAHEDRON_4
_hexahedron_8 = HEXAHEDRON_8

__all__ = ["Mesh", "SolidMechanicsModel", "MaterialElastic", "MaterialNeohookean", "MaterialUser",
           "Material", "MaterialFactory", "MeshDataMaterialSelectorString", "parseInput",
           "FixedValue", "FreeBoundary", "FromTraction", "FromStress", "IncrementValue",
           "Increment", "DirichletFunctor", "NeumannFunctor",
           "_explicit_lumped_mass", "_x", "_y", "_z", "_not_ghost", "_ghost",
           "MODE_FP64_REFERENCE", "MODE_FP64", "MODE_FP32_BULK"]
