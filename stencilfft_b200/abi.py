"""ctypes bindings of the C ABI in include/zmodel_b200.h."""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
HEADER = ROOT / "include" / "zmodel_b200.h"

ZM_OK = 0
ZM_ERR_INVALID_ARG = 1
ZM_ERR_CONSTRAINT = 2
ZM_ERR_MISALIGNED = 3
ZM_ERR_NO_MEMORY = 4
ZM_ERR_CUDA = 5
ZM_ERR_TIMEOUT = 6
ZM_ERR_UNSUPPORTED = 7
ZM_ERR_WORKSPACE = 8

ZM_C128 = 0
ZM_C64 = 1
ZM_FLAG_PERMUTE_ONLY = 0x1
ZM_FLAG_HOST_ONLY = 0x2
ZM_FLAG_OWN_WORKSPACE = 0x4

ZM_SPECTRAL_GAUSSIAN = 0
ZM_SPECTRAL_POISSON = 1
ZM_SPECTRAL_SCALE = 2
ZM_FIELD_UNIFORM = 0
ZM_FIELD_GAUSSIAN = 1

_i64 = ctypes.c_int64
_P = ctypes.c_void_p
_D = ctypes.c_double
_PI64 = ctypes.POINTER(_i64)


class zm_plan_info(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("dtype", ctypes.c_int), ("n", _i64), ("b", _i64),
                ("p", _i64), ("local_dim", _i64), ("vec", _i64), ("vec_split", _i64), ("m", _i64),
                ("ranks", _i64), ("rank_elems", _i64), ("total_elems", _i64),
                ("elem_bytes", ctypes.c_size_t), ("field_bytes", ctypes.c_size_t),
                ("workspace_bytes", ctypes.c_size_t)]


class zm_batch_field(ctypes.Structure):
    _fields_ = [("n", _i64), ("b", _i64), ("p", _i64), ("offset", _i64), ("elems", _i64)]


class ZmError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str):
        super().__init__(f"{what} failed with status {status}: {detail}")
        self.status = status


# name -> argtypes (restype int unless listed in _RESTYPES)
SIGNATURES = {
    "zm_plan_create": [ctypes.POINTER(_P), ctypes.c_int, _i64, _i64, _i64, ctypes.c_int, ctypes.c_uint],
    "zm_plan_destroy": [_P],
    "zm_plan_get_info": [_P, ctypes.POINTER(zm_plan_info)],
    "zm_plan_workspace_size": [_P, ctypes.POINTER(ctypes.c_size_t)],
    "zm_plan_device_status": [_P, ctypes.POINTER(ctypes.c_int)],
    "zm_plan_kernel_variants": [_P, ctypes.POINTER(ctypes.c_int)],
    "zm_plan_set_kernel_variant": [_P, ctypes.c_int],
    "zm_autotune_b": [ctypes.c_int, _i64, _i64, ctypes.c_int, ctypes.c_int, _PI64, ctypes.POINTER(ctypes.c_int),
                      ctypes.POINTER(ctypes.c_float)],
    "zm_plan_autotune": [_P, _P, _P, _P, ctypes.c_int, _P, ctypes.POINTER(ctypes.c_int),
                         ctypes.POINTER(ctypes.c_float)],
    "zm_fft_forward": [_P, _P, _P, _P, _P],
    "zm_fft_inverse": [_P, _P, _P, _P, _D, _D, _P],
    "zm_fft_inverse_static": [_P, _P, _P, _D, _D, _P],
    "zm_laplace": [_P, _P, _P, _D, _P],
    "zm_laplace_dx_dy": [_P, _P, _P, _P, _P, _D, _D, _P],
    "zm_dx": [_P, _P, _P, _D, _P],
    "zm_dy": [_P, _P, _P, _D, _P],
    "zm_dx_real": [_P, _P, _P, _D, _P],
    "zm_dy_real": [_P, _P, _P, _D, _P],
    "zm_fft_forward_vjp": [_P, _P, _P, _P, _P],
    "zm_fft_inverse_vjp": [_P, _P, _P, _P, _D, _D, _P],
    "zm_laplace_vjp": [_P, _P, _P, _D, _P],
    "zm_dx_vjp": [_P, _P, _P, _D, _P],
    "zm_dy_vjp": [_P, _P, _P, _D, _P],
    "zm_natural_to_real": [_P, _P, _P, _P],
    "zm_real_to_natural": [_P, _P, _P, _P],
    "zm_natural_to_reciprocal": [_P, _P, _P, _P],
    "zm_reciprocal_to_natural": [_P, _P, _P, _P],
    "zm_spectral_apply": [_P, _P, ctypes.c_int, _D, _P],
    "zm_spectral_apply_vjp": [_P, _P, ctypes.c_int, _D, _P],
    "zm_fill_field": [_P, _P, ctypes.c_int, ctypes.c_uint64, _P],
    "zm_fill_modes": [_P, _P, ctypes.c_int, _PI64, ctypes.POINTER(_D), _D, ctypes.c_uint64, _P],
    "zm_real_to_global": [_P, _i64, _i64, _i64, _i64, _i64, _i64, _PI64, _PI64, _PI64],
    "zm_global_to_real": [_P, _i64, _i64, _i64, _PI64, _PI64, _PI64, _PI64, _PI64, _PI64],
    "zm_reciprocal_to_global": [_P, _i64, _i64, _i64, _i64, _i64, _i64, _PI64, _PI64, _PI64],
    "zm_global_to_reciprocal": [_P, _i64, _i64, _i64, _PI64, _PI64, _PI64, _PI64, _PI64, _PI64],
    "zm_batch_create": [ctypes.POINTER(_P), ctypes.c_int, _PI64, _PI64, _PI64, ctypes.c_int],
    "zm_batch_destroy": [_P],
    "zm_batch_get_field": [_P, ctypes.c_int, ctypes.POINTER(zm_batch_field)],
    "zm_batch_total_elems": [_P, _PI64],
    "zm_batch_fill": [_P, _P, ctypes.c_int, ctypes.c_uint64, _P],
    "zm_batch_forward": [_P, _P, _P, _P],
    "zm_batch_inverse": [_P, _P, _P, _P, ctypes.c_int, _P],
    "zm_batch_poisson": [_P, _P, _P, _P, _P, _D, _P],
    "zm_batch_status": [_P, ctypes.POINTER(ctypes.c_int)],
    "zm_batch_barrier_probe": [_P, ctypes.c_int, _P],
    "zm_batch_autotune_b": [_i64, _i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _PI64,
                            ctypes.POINTER(ctypes.c_float)],
    "zm_last_error_string": [],
    "zm_status_string": [ctypes.c_int],
    "zm_launch_count": [],
    "zm_version": [],
}
_RESTYPES = {"zm_last_error_string": ctypes.c_char_p, "zm_status_string": ctypes.c_char_p,
             "zm_launch_count": ctypes.c_uint64, "zm_version": ctypes.c_char_p}

_lib = None


def library_path() -> Path:
    env = os.environ.get("ZMODEL_B200_LIB")
    return Path(env) if env else PKG / "lib" / "libzmodel_b200.so"


def lib():
    """Load libzmodel_b200.so (raises if it has not been built -- there is no fallback)."""
    global _lib
    if _lib is None:
        path = library_path()
        if not path.exists():
            raise RuntimeError(f"{path} is missing: build it with `python -m stencilfft_b200._build` "
                               "(the CUDA library is the only implementation)")
        L = ctypes.CDLL(str(path))
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = L
    return _lib


def check(status: int, what: str) -> None:
    if status != ZM_OK:
        detail = lib().zm_last_error_string().decode(errors="replace")
        raise ZmError(status, what, detail)


def launch_count() -> int:
    return int(lib().zm_launch_count())


def declared_symbols() -> list[str]:
    """Every function the public header declares (parsed from include/zmodel_b200.h)."""
    import re
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s+\*?\s*(zm_[a-z_0-9]+)\s*\(", text,
                                 flags=re.M)))
