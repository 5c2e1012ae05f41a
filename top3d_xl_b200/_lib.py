"""ctypes binding of libtopx.so (include/topx.h).

The library is loaded from this package directory.  There is no fallback: if
libtopx.so is missing or cannot be loaded, importing the engine raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtopx.so")

TOPX_OK, TOPX_STOP = 0, 1
ERRORS = {-1: "TOPX_ERR_ARG", -2: "TOPX_ERR_STATE", -3: "TOPX_ERR_CUDA", -4: "TOPX_ERR_MODEL",
          -5: "TOPX_ERR_NUMERIC", -6: "TOPX_ERR_INTERNAL", -7: "TOPX_ERR_TIMEOUT"}

ARR = dict(ENODMAT=0, ELEMAPBACK=1, NODMAPBACK=2, NODESONBOUNDARY=3, ELEMENTSONBOUNDARY=4,
           ELEMENTUPWARDMAP=5, TRANSFERMAT=6, SOLIDNODEMAP=7, FIXEDDOFS=8, MAPUNIQUEKES=9,
           ISTHISELE2NDLEVEL=10, PASSIVEELEMENTS=11)


class Params(C.Structure):
    _fields_ = [("modulus", C.c_double), ("poissonRatio", C.c_double), ("modulusMin", C.c_double),
                ("SIMPpenalty", C.c_double), ("cellSize", C.c_double), ("tol", C.c_double),
                ("maxIT", C.c_int), ("weightFactorJacobi", C.c_double),
                ("coarsestResolutionControl", C.c_int64), ("precision", C.c_int), ("device", C.c_int),
                ("coarse_coop", C.c_int), ("typeVcycle", C.c_int), ("specifyPassiveRegions", C.c_int * 3)]


class Info(C.Structure):
    _fields_ = [("numLevels", C.c_int), ("nelx", C.c_int), ("nely", C.c_int), ("nelz", C.c_int),
                ("numElements", C.c_int64), ("numNodes", C.c_int64), ("numDOFs", C.c_int64),
                ("resX", C.c_int * 8), ("resY", C.c_int * 8), ("resZ", C.c_int * 8),
                ("levelElements", C.c_int64 * 8), ("levelNodes", C.c_int64 * 8),
                ("numLoadCases", C.c_int), ("numFixedDOFs", C.c_int64), ("numPassive", C.c_int64)]


class Iter(C.Structure):
    _fields_ = [("loop", C.c_int), ("c", C.c_double), ("vol", C.c_double), ("sharp", C.c_double),
                ("cons", C.c_double), ("change", C.c_double), ("its", C.c_int * 8), ("filter_its", C.c_int),
                ("t_assemble", C.c_double), ("t_cg", C.c_double), ("t_opt", C.c_double),
                ("t_filter", C.c_double), ("t_total", C.c_double)]


NSECTIONS = 14


class Profile(C.Structure):
    _fields_ = [("ku_ms", C.c_double), ("ku_launches", C.c_int64), ("pcg_iterations", C.c_int64),
                ("section_ms", C.c_double * NSECTIONS), ("section_count", C.c_int64 * NSECTIONS)]


class ServerParams(C.Structure):
    _fields_ = [("slots", C.c_int), ("hbm_budget_bytes", C.c_double), ("precision", C.c_int), ("device", C.c_int)]


class Job(C.Structure):
    _fields_ = [("nely", C.c_int), ("nelx", C.c_int), ("nelz", C.c_int), ("voxels", C.POINTER(C.c_uint8)),
                ("consType", C.c_int), ("V0", C.c_double), ("nLoop", C.c_int), ("rMin", C.c_double),
                ("rHat", C.c_double), ("keep_density", C.c_int)]


class JobResult(C.Structure):
    _fields_ = [("status", C.c_int), ("loops", C.c_int), ("cSolid", C.c_double), ("c_last", C.c_double),
                ("pcg_its", C.c_int64), ("numElements", C.c_int64), ("footprint_estimate", C.c_int64),
                ("footprint_bytes", C.c_int64), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_end", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("done", C.c_int64), ("failed", C.c_int64), ("running", C.c_int64),
                ("queued", C.c_int64), ("max_running", C.c_int), ("budget_bytes", C.c_double),
                ("peak_bytes", C.c_double)]


# exported symbols and their argument types (checked by tests/test_abi.py)
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_SZ = C.c_size_t
SIGNATURES = {
    "topx_default_params": [C.POINTER(Params)],
    "topx_create": [C.POINTER(_P), C.POINTER(Params)],
    "topx_destroy": [_P],
    "topx_last_error": [_P],
    "topx_version": [],
    "topx_load_voxels": [_P, C.POINTER(C.c_uint8), C.c_int, C.c_int, C.c_int],
    "topx_load_topvoxel": [_P, C.c_char_p],
    "topx_set_bc": [_P, _D, C.c_int64, _D, C.c_int64],
    "topx_get_info": [_P, C.POINTER(Info)],
    "topx_get_ke": [_P, _D],
    "topx_get_index_array": [_P, C.c_int, C.c_int, _I32, _SZ, C.POINTER(_SZ)],
    "topx_get_transfer_coeffi": [_P, C.c_int, _D, _SZ, C.POINTER(_SZ)],
    "topx_get_load": [_P, C.c_int, _D, _SZ],
    "topx_set_moduli": [_P, _D, _SZ],
    "topx_ku": [_P, _D, _D, _SZ],
    "topx_ku_noalloc": [_P, C.c_void_p, C.c_void_p, _SZ],
    "topx_assemble": [_P],
    "topx_selftest_wait": [_P, C.c_int],
    "topx_vcycle": [_P, _D, _D, _SZ],
    "topx_write_design_nii": [_D, C.c_int, C.c_int, C.c_int, C.c_char_p],
    "topx_write_design_stl": [_D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_char_p, C.POINTER(C.c_int64)],
    "topx_get_diag": [_P, C.c_int, _D, _SZ],
    "topx_pcg": [_P, C.c_int, _D, _SZ, C.POINTER(C.c_int)],
    "topx_filter": [_P, C.c_double, _D, _D, _SZ, C.POINTER(C.c_int)],
    "topx_unit_compliance": [_P, _D, _D, _SZ],
    "topx_begin": [_P, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, _D],
    "topx_step": [_P, C.POINTER(Iter)],
    "topx_run": [_P, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, C.POINTER(Iter),
                 C.POINTER(C.c_int), _D],
    "topx_get_density": [_P, _D, _SZ],
    "topx_set_density": [_P, _D, _SZ],
    "topx_get_displacement": [_P, C.c_int, _D, _SZ],
    "topx_timer_start": [_P],
    "topx_timer_stop": [_P, _D],
    "topx_set_profiling": [_P, C.c_int],
    "topx_get_profile": [_P, C.POINTER(Profile)],
    "topx_profile_section_name": [C.c_int],
    "topx_launch_count": [],
    "topx_server_default_params": [C.POINTER(ServerParams)],
    "topx_server_create": [C.POINTER(_P), C.POINTER(ServerParams)],
    "topx_server_destroy": [_P],
    "topx_server_submit": [_P, C.POINTER(Job), C.POINTER(C.c_int64)],
    "topx_server_poll": [_P, C.c_int64, C.POINTER(JobResult)],
    "topx_server_wait": [_P, C.c_int64, C.POINTER(JobResult)],
    "topx_server_get_history": [_P, C.c_int64, C.POINTER(Iter), C.c_int, C.POINTER(C.c_int)],
    "topx_server_get_density": [_P, C.c_int64, _D, _SZ],
    "topx_server_get_stats": [_P, C.POINTER(ServerStats)],
    "topx_server_last_error": [_P],
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libtopx.so and declare its prototypes; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libtopx.so not built at {path}; run `python -m top3d_xl_b200.build`")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_char_p if name in ("topx_last_error", "topx_version", "topx_profile_section_name",
                                            "topx_server_last_error") \
            else C.c_int64 if name == "topx_launch_count" else C.c_int
    _lib = lib
    return lib
