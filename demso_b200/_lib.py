"""ctypes binding of ``libdemso_b200.so`` (C ABI in include/demso_b200.h).

Loading fails loudly when the library has not been built: there is no
Python or CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdemso_b200.so")

DEM_MAX_MATERIALS = 10
STATUS = {0: "DEM_OK", 1: "DEM_ERR_INVALID_ARG", 2: "DEM_ERR_CUDA", 3: "DEM_ERR_OOB",
          4: "DEM_ERR_TIMEOUT", 5: "DEM_ERR_NO_MEMORY", 6: "DEM_ERR_CAPACITY"}
CTX_PRESSURE = 1
CTX_ACCEL = 2
CTX_DIRECT = 4
CTX_AUTOTUNE = 8
CTX_CALLER_STATE = 16
CTX_RESIDENT = 32
STATE_PAD = 8  # DEM_STATE_PAD
STEP_VARIANTS = 4  # DEM_STEP_VARIANTS
NUM_STAGES = 3  # DEM_NUM_STAGES: sort, reorder, collide + integrate
ADJ_NUM_COEF = 7  # DEM_ADJ_NUM_COEF


class DemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "?"), code, msg))
        self.code = code


class DemMaterial(C.Structure):
    _fields_ = [("normalStiffness", C.c_float), ("shearStiffness", C.c_float),
                ("normalDamping", C.c_float), ("boundaryDamping", C.c_float),
                ("frictionCoefficient", C.c_float), ("attractCoefficient", C.c_float)]


class DemSystem(C.Structure):
    _fields_ = [("numParticles", C.c_uint32), ("cubeDimension", C.c_float * 2),
                ("gridSize", C.c_uint32 * 2), ("timeStep", C.c_float),
                ("gravity", C.c_float * 2), ("boundaryNormalStiffness", C.c_float),
                ("boundaryShearStiffness", C.c_float), ("numMaterials", C.c_uint32),
                ("materials", DemMaterial * DEM_MAX_MATERIALS)]


class DemDsmlInfo(C.Structure):
    _fields_ = [("numParticles", C.c_uint32), ("numTypes", C.c_uint32),
                ("numFollowed", C.c_uint32), ("imageHeight", C.c_uint32),
                ("numRectangles", C.c_uint32), ("numTriangles", C.c_uint32),
                ("numSingles", C.c_uint32), ("controlledType", C.c_int32),
                ("timeStep", C.c_float), ("simDuration", C.c_float)]


class DemDsmlType(C.Structure):
    _fields_ = [("id", C.c_char * 64), ("name", C.c_char * 128), ("mass", C.c_float),
                ("radius", C.c_float), ("color", C.c_float * 3)]


DSML_NO_JITTER = 1  # DEM_DSML_NO_JITTER


class DemControl(C.Structure):
    _fields_ = [("pos", C.c_float * 2), ("vel", C.c_float * 2), ("theta", C.c_float),
                ("omega", C.c_float), ("radius", C.c_float), ("material", C.c_uint32),
                ("drift", C.c_double * 2), ("wrapYBelow", C.c_double), ("wrapYTo", C.c_double),
                ("wrapXAbove", C.c_double), ("wrapXTo", C.c_double)]


class DemStepVariant(C.Structure):
    _fields_ = [("variant", C.c_int32), ("threads", C.c_uint32), ("blocksPerSm", C.c_uint32),
                ("tuned", C.c_int32), ("medianMs", C.c_float * STEP_VARIANTS)]


class DemRenderParams(C.Structure):
    _fields_ = [("imageDIMx", C.c_uint32), ("imageDIMy", C.c_uint32), ("bgColor", C.c_uint32),
                ("viewRotations", C.c_uint32), ("colorByPressure", C.c_uint32),
                ("maxPressure", C.c_float), ("color", (C.c_float * 3) * DEM_MAX_MATERIALS)]

class DemStateSet(C.Structure):
    _fields_ = [("pos", C.c_void_p), ("vel", C.c_void_p), ("theta", C.c_void_p),
                ("omega", C.c_void_p), ("radius", C.c_void_p), ("mass", C.c_void_p),
                ("id", C.c_void_p), ("type", C.c_void_p)]

# (name, restype, argtypes)
_P = C.c_void_p
_U = C.c_uint32
_SYS = C.POINTER(DemSystem)
SIGNATURES = [
    ("dem_abi_version", C.c_int, []),
    ("dem_last_error_string", C.c_char_p, []),
    ("dem_validate_system", C.c_int, [_SYS]),
    ("dem_calc_hash", C.c_int, [_SYS, _P, _P, _P, _U, _P]),
    ("dem_sort_scratch_bytes", C.c_size_t, [_U, _U]),
    ("dem_sort_particles", C.c_int, [_P, _P, _U, _U, _P, C.c_size_t, _P]),
    ("dem_sort_particles_static", C.c_int, [_P, _P, _U, _U, _P]),
    ("dem_reorder_data_and_find_cell_start", C.c_int,
     [_SYS, _P, _P] + [_P] * 9 + [_P, _P] + [_P] * 8 + [_U, _U, _P]),
    ("dem_collide", C.c_int, [_SYS, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U, _U, _P, _P]),
    ("dem_integrate_system", C.c_int, [_SYS, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _U, _P]),
    ("dem_create", C.c_int, [_SYS, _U, _U, C.POINTER(_P)]),
    ("dem_create_rows", C.c_int, [_SYS, _U, _U, _U, _U, C.POINTER(_P)]),
    ("dem_batch_create", C.c_int, [_SYS, _U, _U, C.POINTER(_P)]),
    ("dem_batch_specimen", C.c_int, [_P, _U, C.POINTER(_U), C.POINTER(_U)]),
    ("dem_batch_set_systems", C.c_int, [_P, _P, _U, _P]),
    ("dem_destroy", C.c_int, [_P]),
    ("dem_set_system", C.c_int, [_P, _SYS]),
    ("dem_set_state", C.c_int, [_P, _U] + [_P] * 8 + [C.c_int, _P]),
    ("dem_get_state", C.c_int, [_P] + [_P] * 12 + [C.c_int, _P]),
    ("dem_adopt_state", C.c_int, [_P, _U, C.POINTER(DemStateSet), C.POINTER(DemStateSet), _P]),
    ("dem_state_view", C.c_int, [_P, C.POINTER(DemStateSet), C.POINTER(C.c_int)]),
    ("dem_row_slots", C.c_int, [_P, _U, _U, C.POINTER(_U), C.POINTER(_U), _P]),
    ("dem_step", C.c_int, [_P, _U, _P]),
    ("dem_get_cells", C.c_int, [_P, _P, _P, _P]),
    ("dem_check", C.c_int, [_P, _P]),
    ("dem_debug_fail_allocation", C.c_int, [C.c_int]),
    ("dem_debug_live_allocations", C.c_longlong, []),
    ("dem_debug_sort_hold", C.c_int, [_P, _U, _U]),
    ("dem_kernels_per_step", C.c_int, [_P]),
    ("dem_set_step_variant", C.c_int, [_P, C.c_int32]),
    ("dem_get_step_variant", C.c_int, [_P, C.POINTER(DemStepVariant)]),
    ("dem_get_followed", C.c_int, [_P, _P, _U, _P, _P]),
    ("dem_get_followed_async", C.c_int, [_P, _P, _U, _P, _P]),
    ("dem_step_followed", C.c_int, [_P, _U, _P, _U, _P, _P]),
    ("dem_profile_begin", C.c_int, [_P, _U]),
    ("dem_profile_end", C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(_U)]),
    ("dem_adj_forward", C.c_int, [_P, _U, _U, _P]),
    ("dem_adj_backward", C.c_int, [_P, _P, _P, _P, C.POINTER(C.c_double), _P]),
    ("dem_scene_rsa", C.c_int, [_U, _P, C.c_float, C.c_float, C.c_uint64, _U, _U, _P,
                                C.POINTER(_U)]),
    ("dem_set_control", C.c_int, [_P, C.POINTER(DemControl), _P]),
    ("dem_get_control", C.c_int, [_P, C.POINTER(DemControl), C.POINTER(C.c_float), _P]),
    ("dem_render_particles", C.c_int, [_SYS, _P, _P, _P, _P, _P, _U,
                                       C.POINTER(DemRenderParams), _P, _P, _P]),
    ("dem_render", C.c_int, [_P, C.POINTER(DemRenderParams), _P, _P]),
    ("dem_dsml_load", C.c_int, [C.c_char_p, C.c_uint64, _U, C.POINTER(_P)]),
    ("dem_dsml_parse", C.c_int, [C.c_char_p, C.c_size_t, C.c_uint64, _U, C.POINTER(_P)]),
    ("dem_dsml_free", None, [_P]),
    ("dem_dsml_info", C.c_int, [_P, C.POINTER(DemDsmlInfo)]),
    ("dem_dsml_system", C.c_int, [_P, _SYS]),
    ("dem_dsml_state", C.c_int, [_P] + [_P] * 8),
    ("dem_dsml_followed", C.c_int, [_P, _P]),
    ("dem_dsml_type", C.c_int, [_P, _U, C.POINTER(DemDsmlType)]),
]

_lib = None


def load():
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(LIB_PATH):
        raise RuntimeError("demso_b200 native library missing (%s); build it with "
                           "`python -m demso_b200.build`" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        msg = load().dem_last_error_string()
        raise DemError(rc, msg.decode() if msg else "")
