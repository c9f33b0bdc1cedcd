"""ctypes mirror of the structs and constants declared in include/akb.h."""
import ctypes as C

ABI_VERSION = 1

# status codes
AKB_OK = 0
AKB_ERR_INVALID_ARGUMENT = 1
AKB_ERR_BAD_MESH = 2
AKB_ERR_NEGATIVE_JACOBIAN = 3
AKB_ERR_NON_FINITE = 4
AKB_ERR_CUDA = 5
AKB_ERR_TIMEOUT = 6
AKB_ERR_STATE = 7
AKB_ERR_UNSUPPORTED = 8
AKB_ERR_OUT_OF_MEMORY = 9

STATUS_NAMES = {
    0: "ok", 1: "invalid argument", 2: "bad mesh", 3: "negative jacobian",
    4: "non-finite value", 5: "CUDA error", 6: "timeout", 7: "invalid state",
    8: "unsupported", 9: "out of memory",
}

# element types
SEGMENT_2 = 1
TRIANGLE_3 = 2
TETRAHEDRON_4 = 3
HEXAHEDRON_8 = 4

# materials
MATERIAL_ELASTIC = 0
MATERIAL_NEOHOOKEAN = 1
MATERIAL_USER = 2

# precision modes
MODE_FP64_REFERENCE = 0
MODE_FP64 = 1
MODE_FP32_BULK = 2

# fields
FIELD_DISPLACEMENT = 0
FIELD_VELOCITY = 1
FIELD_ACCELERATION = 2
FIELD_EXTERNAL_FORCE = 3
FIELD_INTERNAL_FORCE = 4
FIELD_MASS = 5
FIELD_NODES = 6
FIELD_GRAD_U = 7
FIELD_STRESS = 8

# energies
ENERGY_KINETIC = 0
ENERGY_POTENTIAL = 1
ENERGY_EXTERNAL_WORK = 2

ALL_COMPONENTS = -1  # akb_apply_dirichlet: every component, values row per node


class MeshDesc(C.Structure):
    _fields_ = [
        ("spatial_dimension", C.c_int32),
        ("element_type", C.c_int32),
        ("nb_nodes", C.c_int64),
        ("nb_elements", C.c_int64),
        ("nodes", C.POINTER(C.c_double)),
        ("connectivity", C.POINTER(C.c_uint32)),
    ]


class MaterialDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("plane_stress", C.c_int32),
        ("finite_deformation", C.c_int32),
        ("reserved", C.c_int32),
        ("rho", C.c_double),
        ("E", C.c_double),
        ("nu", C.c_double),
    ]


class ModelOptions(C.Structure):
    _fields_ = [
        ("precision_mode", C.c_int32),
        ("device", C.c_int32),
        ("stream", C.c_void_p),
        ("patch_elements", C.c_int32),
        ("patch_nodes", C.c_int32),
        ("patch_grid", C.c_int32),
    ]


class BatchDesc(C.Structure):
    _fields_ = [
        ("nb_instances", C.c_int32),
        ("meshes", C.POINTER(MeshDesc)),
        ("materials", C.POINTER(MaterialDesc)),
    ]


class ModelInfo(C.Structure):
    _fields_ = [
        ("spatial_dimension", C.c_int32),
        ("element_type", C.c_int32),
        ("nodes_per_element", C.c_int32),
        ("quadrature_points_per_element", C.c_int32),
        ("nb_nodes", C.c_int64),
        ("nb_elements", C.c_int64),
        ("precision_mode", C.c_int32),
        ("nb_materials", C.c_int32),
        ("device_bytes", C.c_int64),
    ]


# ---- include/akb_fe2.h
class RveDesc(C.Structure):
    _fields_ = [("cells", C.c_int32), ("nb_materials", C.c_int32), ("length", C.c_double),
                ("voxel_material", C.POINTER(C.c_uint8)),
                ("materials", C.POINTER(MaterialDesc))]


class RveOptions(C.Structure):
    _fields_ = [("precision_mode", C.c_int32), ("device", C.c_int32), ("stream", C.c_void_p),
                ("max_iterations", C.c_int32), ("check_interval", C.c_int32),
                ("tolerance", C.c_double), ("time_step_factor", C.c_double),
                ("damping_factor", C.c_double)]


class RveInfo(C.Structure):
    _fields_ = [("cells", C.c_int32), ("precision_mode", C.c_int32), ("nb_nodes", C.c_int64),
                ("volume_fraction", C.c_double * 8), ("shared_bytes", C.c_int64)]

# Neumann condition kinds (akb_neumann_kind)
NEUMANN_TRACTION = 0
NEUMANN_STRESS = 1
