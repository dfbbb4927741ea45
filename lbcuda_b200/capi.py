"""ctypes binding of include/lbx.h (the C ABI of liblbx.so)."""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblbx.so")

MODEL = {"bgk": 0, "cg": 1, "cg-diffdens": 2, "cg-d3q27": 3, "cg-diffdens-d3q27": 4}
STORAGE = {"f32": 0, "f16": 1, "bf16": 2, "f64": 3, "f16sd": 4, "bf16sd": 5, "f16sdp": 6, "bf16sdp": 7}
WETTING = {"janus": 0, "neutral": 1}

FLUID_WALL, FLUID_FLUID, FLUID_SPHERELIST, FLUID_SPHEREDEAD, FLUID_PARTICLECM = 0, 1, 2, 4, 5


class LbxParams(C.Structure):
    """Mirror of ``lbx_params`` (include/lbx.h)."""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("model", C.c_int32), ("storage", C.c_int32), ("wetting", C.c_int32),
        ("lrotate", C.c_int32), ("max_particles", C.c_int32),
        ("tau", C.c_float), ("tauR", C.c_float), ("tauB", C.c_float),
        ("sigma", C.c_float), ("beta", C.c_float),
        ("rho0R", C.c_float), ("rho0B", C.c_float),
        ("radius", C.c_float), ("rmass", C.c_float), ("max_vel", C.c_float),
        ("ext_force", C.c_float * 3), ("ext_torque", C.c_float * 3),
        ("hz_k", C.c_float), ("hz_rmin", C.c_float), ("hz_rcap", C.c_float),
        ("lubrication", C.c_int32),
        ("lubric_k", C.c_float), ("lubric_rmin", C.c_float), ("lubric_rcap", C.c_float),
        ("kinematic", C.c_int32), ("closure", C.c_int32),
        ("closure_gap_min", C.c_float), ("closure_gap_max", C.c_float), ("closure_vmax", C.c_float),
        ("exact_tiles", C.c_int32), ("densR", C.c_float), ("densB", C.c_float),
    ]


class LBXError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        msg = _lib.lbx_error_string(code).decode() if _lib is not None else str(code)
        super().__init__(f"{where}: lbx status {code} ({msg})" if where else f"lbx status {code} ({msg})")


_lib = None

_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_I8 = C.POINTER(C.c_int8)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes)
SIGNATURES = {
    "lbx_default_params": (None, [C.POINTER(LbxParams), C.c_int32, C.c_int32, C.c_int32]),
    "lbx_create": (C.c_int, [C.POINTER(LbxParams), _PP]),
    "lbx_destroy": (C.c_int, [_P]),
    "lbx_set_fields": (C.c_int, [_P, _F, _F, C.c_float, C.c_float, C.c_float]),
    "lbx_set_pops": (C.c_int, [_P, _F, _F]),
    "lbx_step": (C.c_int, [_P, C.c_int32]),
    "lbx_init_rho": (C.c_int, [_P]),
    "lbx_make_list_atoms": (C.c_int, [C.c_void_p]),
    "lbx_init_isfluid": (C.c_int, [C.c_void_p]),
    "lbx_del_fluid": (C.c_int, [C.c_void_p]),
    "lbx_make_fluid": (C.c_int, [C.c_void_p]),
    "lbx_virtual_rho": (C.c_int, [C.c_void_p]),
    "lbx_partbb": (C.c_int, [C.c_void_p]),
    "lbx_partbb_p2n": (C.c_int, [C.c_void_p]),
    "lbx_partbb_p2n2": (C.c_int, [C.c_void_p]),
    "lbx_inter_force_particles": (C.c_int, [C.c_void_p]),
    "lbx_time_step_force_particles": (C.c_int, [C.c_void_p]),
    "lbx_time_step_cg": (C.c_int, [_P]),
    "lbx_time_step_bgk": (C.c_int, [_P]),
    "lbx_get_fields": (C.c_int, [_P, _F, _F, _F, _F]),
    "lbx_get_fields_f64": (C.c_int, [_P, _D, _D, _D, _D]),
    "lbx_get_pops": (C.c_int, [_P, _F, _F]),
    "lbx_get_flags": (C.c_int, [_P, _I8]),
    "lbx_get_sums": (C.c_int, [_P, _D, _D]),
    "lbx_get_links": (C.c_int, [_P, _I32, _I8, _I32, C.c_int64, _I64]),
    "lbx_set_particles": (C.c_int, [_P, C.c_int32, _D, _D, _D, _D]),
    "lbx_get_particles": (C.c_int, [_P, _D, _D, _D, _D, _D, _D]),
    "lbx_closure_init": (C.c_int, [_F, C.c_int32]),
    "lbx_closure_train": (C.c_int, [_F, _F, _F, C.c_int32, C.c_int32, C.c_float, C.c_int32, _F]),
    "lbx_closure_grad": (C.c_int, [_F, _F, _F, C.c_int32, _F]),
    "lbx_closure_infer": (C.c_int, [_F, _F, C.c_int32, _F]),
    "lbx_closure_infer_noalloc": (C.c_int, [_F, _F, C.c_int32, _F]),
    "lbx_closure_set": (C.c_int, [_P, _F]),
    "lbx_ensemble_create": (C.c_int, [C.c_int32, C.POINTER(LbxParams), _PP]),
    "lbx_ensemble_destroy": (C.c_int, [_P]),
    "lbx_ensemble_box": (C.c_int, [_P, C.c_int32, _PP]),
    "lbx_ensemble_step": (C.c_int, [_P, C.c_int32]),
    "lbx_ensemble_time": (C.c_int, [_P, C.c_int32, _D]),
    "lbx_ensemble_tune": (C.c_int, [_P, C.c_int32, _I32, _D]),
    "lbx_sync": (C.c_int, [_P]),
    "lbx_status": (C.c_int, [_P, _I32, _I32, _I64]),
    "lbx_error_string": (C.c_char_p, [C.c_int]),
    "lbx_get_step": (C.c_int, [_P, _I64]),
    "lbx_set_schedule": (C.c_int, [_P, C.c_int32]),
    "lbx_set_lean_shape": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "lbx_set_lean_copies": (C.c_int, [_P, C.c_int32]),
    "lbx_set_zrange": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "lbx_plane_bytes": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int64)]),
    "lbx_pack_planes": (C.c_int, [_P, C.c_int32, C.c_int32, _P]),
    "lbx_unpack_planes": (C.c_int, [_P, C.c_int32, C.c_int32, _P]),
    "lbx_get_stream": (C.c_int, [_P, _PP]),
    "lbx_time_steps": (C.c_int, [_P, C.c_int32, _D, _D, _I64]),
}


def header_symbols():
    """Function names declared in include/lbx.h (parsed from the header)."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "lbx.h")
    text = open(hdr).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbx_[a-z0-9_]+)\s*\(", text)))


def lib_path():
    return _LIB_PATH


def lib():
    """Load liblbx.so (raises if it is missing: the CUDA path has no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"liblbx.so not built at {_LIB_PATH}; run `python -m lbcuda_b200.build`")
    L = C.CDLL(_LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc, where=""):
    if rc != 0:
        raise LBXError(rc, where)
    return rc
