"""ctypes binding of libb3dgpu.so (include/b3dgpu.h).  The library is required: importing the kernels
without it, or calling them without a CUDA device, raises instead of falling back to anything else."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("B3DGPU_LIB", os.path.join(HERE, "libb3dgpu.so"))

_P = ctypes.c_void_p
_I = ctypes.c_int
_Q = ctypes.c_int64

# name -> argument types (every entry point returns int)
SIGNATURES = {
    "b3d_version": [],
    "b3d_supported_limbs": [_I],
    "b3d_align": [_I, _P, _P, _Q, _Q, _Q, _Q, _Q, _Q, _Q, _P, _P, _P, _Q, _I, _P],
    "b3d_gemm_aligned": [_I, _P, _P, _Q, _P, _P, _Q, _Q, _Q, _Q, _Q, _P, _P, _Q, _P],
    "b3d_mul": [_I, _P, _P, _Q, _P, _P, _P, _Q, _P, _Q, _P, _P, _Q, _P],
    "b3d_add": [_I, _P, _P, _Q, _P, _P, _P, _Q, _P, _Q, _P, _P, _Q, _P],
    "b3d_cauchy_level": [_I, _P, _P, _Q, _P, _P, _Q, _P, _P, _P, _Q, _P],
    "b3d_pole_level": [_I, _P, _P, _Q, _P, _P, _Q, _P, _P, _Q, _P, _P, _P, _P, _Q, _Q, _I, _P, _P, _Q, _P, _P, _Q, _P],
    "b3d_pole_level_mma": [_I, _P, _P, _Q, _P, _P, _Q, _P, _P, _Q, _P, _P, _P, _P, _Q, _Q, _I, _P, _P, _Q, _P, _P, _Q,
                           _P, _P],
    "b3d_moments_level": [_I, _P, _P, _Q, _P, _P, _Q, _P, _P, _P, _Q, _Q, _I, _P, _P, _Q, _P],
    "b3d_moments_stage": [_I, _P, _P, _Q, _P, _P, _Q, _P, _P, _P, _Q, _Q, _Q, _Q, _P, _P, _Q, _P],
    "b3d_moments_flush": [_I, _P, _P, _Q, _P, _Q, _I, _Q, _Q, _I, _P, _P, _I, _I, _I, _I, _P, _P, _Q, _P],
    "b3d_resize": [_I, _P, _P, _Q, _Q, _I, _P, _P, _Q, _P],
    "b3d_cauchy_align": [_I, _P, _P, _Q, _P, _P, _P, _Q, _P],
    "b3d_cauchy_level2": [_I, _P, _P, _Q, _P, _P, _Q, _P, _P, _P, _Q, _P],
    "b3d_cauchy_level3": [_I, _P, _P, _Q, _P, _P, _Q, _P, _Q, _P, _P, _Q, _P],
    "b3d_cauchy_align_sm": [_I, _P, _P, _Q, _P, _P, _P, _Q, _P],
    "b3d_cauchy_level4": [_I, _P, _P, _Q, _P, _P, _Q, _P, _Q, _P, _P, _Q, _P],
    "b3d_cauchy_digits": [_P, _P, _Q, _I, _Q, _Q, _I, _Q, _P, _P],
    "b3d_cauchy_add_hinf": [_I, _P, _P, _Q, _P, _P, _Q, _P, _P, _P, _Q, _P],
    "b3d_pole_level_noalloc": [_I, _P, _P, _Q, _P, _P, _Q, _P, _P, _Q, _P, _P, _P, _P, _Q, _Q, _I, _P, _P, _Q, _P],
    "b3d_format_decimal": [_I, _P, _P, _Q, _Q, _P, _P, _P, _P, _P],
    "b3d_poly_sizes": [_I, _P, _P, _Q, _P, _Q, _I, _I, _P, _P, _P, _P],
    "b3d_emit_text": [_P, _I, _P, _P, _P, _P, _P, _P, _Q, _P, _P],
    "b3d_plan_build": [_Q, _Q, _Q, _Q, _P, _I, _P],
    "b3d_plan_scalars": [_P, _P],
    "b3d_plan_keys": [_P, _P, _P, _P],
    "b3d_plan_layout": [_P, _P, _P, _P],
    "b3d_plan_level_dims": [_P, _Q, _P],
    "b3d_plan_level": [_P, _Q, _P],
    "b3d_setup_numbers": [_P, _Q, _I, _I, _P, _Q, _P],
}
VOID = {"b3d_plan_destroy": [_P]}             # entry points without a status


class LevelTables(ctypes.Structure):
    """struct b3d_level_tables"""
    _fields_ = [("m", _Q), ("nb", _Q), ("Mr", _Q), ("Kc", _Q), ("N", _Q), ("hlevels", _Q), ("Jh", _Q),
                ("gsrc", _P), ("gj", _P), ("rowd", _P), ("nrow", _P), ("cold", _P), ("ncol", _P), ("col", _P)]


class DecimalTables(ctypes.Structure):
    """struct b3d_decimal_tables"""
    _fields_ = [("pow5", _P), ("pow5_limbs", _P), ("bounds", _P), ("kmax", _I), ("fw", _I), ("p", _I),
                ("stride", _I)]


SIGNATURES["b3d_format_decimal"][5] = ctypes.POINTER(DecimalTables)
SIGNATURES["b3d_cauchy_level"][7] = ctypes.POINTER(LevelTables)
SIGNATURES["b3d_cauchy_align"][4] = ctypes.POINTER(LevelTables)
SIGNATURES["b3d_cauchy_digits"][0] = ctypes.POINTER(LevelTables)
SIGNATURES["b3d_cauchy_level2"][7] = ctypes.POINTER(LevelTables)
SIGNATURES["b3d_cauchy_level3"][7] = ctypes.POINTER(LevelTables)
SIGNATURES["b3d_cauchy_align_sm"][4] = ctypes.POINTER(LevelTables)
SIGNATURES["b3d_cauchy_level4"][7] = ctypes.POINTER(LevelTables)
SIGNATURES["b3d_cauchy_add_hinf"][7] = ctypes.POINTER(LevelTables)
ctypes_byref = ctypes.byref


class B3DError(RuntimeError):
    pass


_lib = None


def lib():
    """the loaded library (raises B3DError if it is missing: build it with python -m blocksvibe_b200.build)"""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise B3DError(f"{LIB_PATH} not found: build it with `python -m blocksvibe_b200.build`")
        h = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(h, name)
            f.argtypes, f.restype = args, _I
        for name, args in VOID.items():
            f = getattr(h, name)
            f.argtypes, f.restype = args, None
        h.b3d_last_error.argtypes, h.b3d_last_error.restype = [], ctypes.c_char_p
        _lib = h
    return _lib


def call(name, *args):
    """call an entry point; a nonzero status raises B3DError with the library's message"""
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise B3DError(f"{name} failed ({rc}): {lib().b3d_last_error().decode()}")
    return rc


def exported_symbols():
    return ["b3d_last_error"] + list(SIGNATURES) + list(VOID)
