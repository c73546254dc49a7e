"""ctypes front end of the CPU oracle (test infrastructure only).

Arrays are numpy: complex fields are ``complex128`` in the interleaved whole-grid
layout (all virtual ranks, rank-major, each rank in the reference's rank-local
layout); natural-layout fields are ``(N, N)`` / ``(N, N, N)`` arrays.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

_i64 = ctypes.c_int64
_P = ctypes.c_void_p
_lib = None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (gcc, OpenMP)."""
    subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        sig = {
            "zo_check_config": [ctypes.c_int, _i64, _i64, _i64],
            "zo_real_layout_map": [ctypes.c_int, _i64, _i64, _i64, _P],
            "zo_reciprocal_layout_map": [ctypes.c_int, _i64, _i64, _i64, _P],
            "zo_real_layout_inverse_map": [ctypes.c_int, _i64, _i64, _i64, _P],
            "zo_reciprocal_layout_inverse_map": [ctypes.c_int, _i64, _i64, _i64, _P],
            "zo_init_ramp": [ctypes.c_int, _i64, _i64, _i64, _P],
            "zo_vector_pack": [ctypes.c_int, _i64, _i64, _i64, _P, _P, _i64],
            "zo_vector_unpack": [ctypes.c_int, _i64, _i64, _i64, _P, _P, _i64],
            "zo_fill_uniform": [ctypes.c_uint64, _i64, _i64, _P],
            "zo_fill_gaussian": [ctypes.c_uint64, _i64, _i64, _P],
            "zo_forward_fft": [ctypes.c_int, _i64, _i64, _i64, _P, _P, ctypes.c_int],
            "zo_forward_first_pass": [ctypes.c_int, _i64, _i64, _i64, _P, _P, ctypes.c_int],
            "zo_inverse_fft": [ctypes.c_int, _i64, _i64, _i64, _P, _P, ctypes.c_double,
                               ctypes.c_double, ctypes.c_int],
            "zo_laplace_2d": [_i64, _i64, _i64, _P, _P],
            "zo_laplace_3d": [_i64, _i64, _i64, _P, _P],
            "zo_dx": [_i64, _i64, _i64, _P, _P, ctypes.c_double, ctypes.c_int],
            "zo_dy": [_i64, _i64, _i64, _P, _P, ctypes.c_double, ctypes.c_int],
            "zo_max_threads": [],
            "zo_set_threads": [ctypes.c_int],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int if name != "zo_set_threads" else None
        for name in ("zo_lp", "zo_ct", "zo_lp_inv", "zo_ct_inv"):
            f = getattr(L, name)
            f.argtypes = [_i64, _i64, _i64, _i64, ctypes.POINTER(_i64)]
            f.restype = ctypes.c_int
        for name in ("zo_real_to_global", "zo_reciprocal_to_global"):
            f = getattr(L, name)
            f.argtypes = [_i64] * 7 + [ctypes.POINTER(_i64)] * 2
            f.restype = ctypes.c_int
        for name in ("zo_global_to_real", "zo_global_to_reciprocal"):
            f = getattr(L, name)
            f.argtypes = [_i64] * 5 + [ctypes.POINTER(_i64)] * 4
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _chk(rc: int, what: str):
    if rc != 0:
        raise ValueError(f"oracle {what} rejected the configuration (rc={rc})")


def derived(dim: int, n: int, b: int, p: int) -> dict:
    """L, VEC, VP, M and rank counts of a layout (zmodel/utils.h:45-71)."""
    _chk(lib().zo_check_config(dim, n, b, p), "check_config")
    L = n // p
    vec = L // b
    return {"L": L, "VEC": vec, "VP": vec // p, "M": b * p,
            "ranks": p ** dim, "rank_elems": L ** dim, "total": n ** dim}


def grid_elems(dim: int, n: int) -> int:
    return n ** dim


# ------------------------------------------------------------------ layouts

def real_layout_map(dim, n, b, p) -> np.ndarray:
    out = np.empty(n ** dim, dtype=np.int64)
    _chk(lib().zo_real_layout_map(dim, n, b, p, _ptr(out)), "real_layout_map")
    return out


def reciprocal_layout_map(dim, n, b, p) -> np.ndarray:
    out = np.empty(n ** dim, dtype=np.int64)
    _chk(lib().zo_reciprocal_layout_map(dim, n, b, p, _ptr(out)), "reciprocal_layout_map")
    return out


def real_layout_inverse_map(dim, n, b, p) -> np.ndarray:
    out = np.empty(n ** dim, dtype=np.int64)
    _chk(lib().zo_real_layout_inverse_map(dim, n, b, p, _ptr(out)), "real_layout_inverse_map")
    return out


def reciprocal_layout_inverse_map(dim, n, b, p) -> np.ndarray:
    out = np.empty(n ** dim, dtype=np.int64)
    _chk(lib().zo_reciprocal_layout_inverse_map(dim, n, b, p, _ptr(out)),
         "reciprocal_layout_inverse_map")
    return out


def natural_to_real_layout(x: np.ndarray, b: int, p: int) -> np.ndarray:
    """Natural (N,N[,N]) field -> interleaved real layout (flat)."""
    dim, n = x.ndim, x.shape[0]
    return np.ascontiguousarray(x.reshape(-1)[real_layout_map(dim, n, b, p)])


def real_layout_to_natural(buf: np.ndarray, dim: int, n: int, b: int, p: int) -> np.ndarray:
    return buf[real_layout_inverse_map(dim, n, b, p)].reshape((n,) * dim)


def natural_to_reciprocal_layout(X: np.ndarray, b: int, p: int) -> np.ndarray:
    dim, n = X.ndim, X.shape[0]
    return np.ascontiguousarray(X.reshape(-1)[reciprocal_layout_map(dim, n, b, p)])


def reciprocal_layout_to_natural(buf: np.ndarray, dim: int, n: int, b: int, p: int) -> np.ndarray:
    return buf[reciprocal_layout_inverse_map(dim, n, b, p)].reshape((n,) * dim)


def index_map(name: str, n: int, b: int, p: int, *args: int):
    """Scalar utils.h index maps: lp, ct, lp_inv, ct_inv, real_to_global,
    global_to_real, reciprocal_to_global, global_to_reciprocal (2D)."""
    L = lib()
    f = getattr(L, "zo_" + name)
    nout = {"lp": 1, "ct": 1, "lp_inv": 1, "ct_inv": 1, "real_to_global": 2,
            "reciprocal_to_global": 2, "global_to_real": 4, "global_to_reciprocal": 4}[name]
    outs = [_i64() for _ in range(nout)]
    _chk(f(n, b, p, *args, *[ctypes.byref(o) for o in outs]), name)
    vals = [o.value for o in outs]
    return vals[0] if nout == 1 else tuple(vals)


# ----------------------------------------------------------------- fixtures

def init_ramp(dim, n, b, p) -> np.ndarray:
    out = np.empty(n ** dim, dtype=np.complex128)
    _chk(lib().zo_init_ramp(dim, n, b, p, _ptr(out)), "init_ramp")
    return out


def uniform_field(seed: int, count: int, first: int = 0) -> np.ndarray:
    """Counter-based U[-1,1) complex field in natural order (shared with the device generator)."""
    out = np.empty(count, dtype=np.complex128)
    lib().zo_fill_uniform(seed, first, count, _ptr(out))
    return out


def gaussian_field(seed: int, count: int, first: int = 0) -> np.ndarray:
    out = np.empty(count, dtype=np.complex128)
    lib().zo_fill_gaussian(seed, first, count, _ptr(out))
    return out


# --------------------------------------------------------------- transforms

def forward_fft(buf: np.ndarray, dim, n, b, p, do_compute: bool = True) -> np.ndarray:
    buf = np.ascontiguousarray(buf, dtype=np.complex128)
    out = np.empty_like(buf)
    _chk(lib().zo_forward_fft(dim, n, b, p, _ptr(buf), _ptr(out), int(do_compute)), "forward_fft")
    return out


def forward_first_pass(buf: np.ndarray, dim, n, b, p, do_compute: bool = True) -> np.ndarray:
    buf = np.ascontiguousarray(buf, dtype=np.complex128)
    out = np.empty_like(buf)
    _chk(lib().zo_forward_first_pass(dim, n, b, p, _ptr(buf), _ptr(out), int(do_compute)),
         "forward_first_pass")
    return out


def inverse_fft(buf: np.ndarray, dim, n, b, p, scale: complex = 1.0,
                do_compute: bool = True) -> np.ndarray:
    buf = np.ascontiguousarray(buf, dtype=np.complex128)
    out = np.empty_like(buf)
    scale = complex(scale)
    _chk(lib().zo_inverse_fft(dim, n, b, p, _ptr(buf), _ptr(out), scale.real, scale.imag,
                              int(do_compute)), "inverse_fft")
    return out


# ----------------------------------------------------------------- stencils

def laplace(buf: np.ndarray, dim, n, b, p) -> np.ndarray:
    buf = np.ascontiguousarray(buf, dtype=np.complex128)
    out = np.empty_like(buf)
    f = lib().zo_laplace_2d if dim == 2 else lib().zo_laplace_3d
    _chk(f(n, b, p, _ptr(buf), _ptr(out)), "laplace")
    return out


def _deriv(fn, buf, n, b, p, delta):
    buf = np.ascontiguousarray(buf)
    if buf.dtype == np.complex128:
        ncomp = 2
    elif buf.dtype == np.float64:
        ncomp = 1
    else:
        raise TypeError("dx/dy oracle takes float64 or complex128")
    out = np.empty_like(buf)
    _chk(fn(n, b, p, _ptr(buf), _ptr(out), float(delta), ncomp), "dx/dy")
    return out


def dx(buf, n, b, p, delta=1.0):
    return _deriv(lib().zo_dx, buf, n, b, p, delta)


def dy(buf, n, b, p, delta=1.0):
    return _deriv(lib().zo_dy, buf, n, b, p, delta)


def max_threads() -> int:
    return lib().zo_max_threads()


def set_threads(n: int) -> None:
    lib().zo_set_threads(int(n))


# ------------------------------------------------------- reference host code

def ref_host_lib(n: int, b: int, p: int):
    """The reference's own utils.h/utils.cu compiled for (N_DIM, B_DIM, P_DIM), or None."""
    path = REF_DIR / f"libzref_host_N{n}_B{b}_P{p}.so"
    if not path.exists():
        return None
    L = ctypes.CDLL(str(path))
    ip = ctypes.POINTER(ctypes.c_int)
    for name in ("zr_packed_to_block_cyclic", "zr_block_cyclic_to_packed", "zr_lp", "zr_ct",
                 "zr_lp_inv", "zr_ct_inv"):
        getattr(L, name).argtypes = [ctypes.c_int]
        getattr(L, name).restype = ctypes.c_int
    L.zr_real_layout_map.argtypes = [ctypes.c_int, _P]
    L.zr_reciprocal_layout_map.argtypes = [ctypes.c_int, _P]
    L.zr_init_host.argtypes = [ctypes.c_int, ctypes.c_int, _P]
    L.zr_init_host_3d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]
    L.zr_init_host_scalar.argtypes = [ctypes.c_int, ctypes.c_int, _P]
    L.zr_global_to_real.argtypes = [ctypes.c_int, ctypes.c_int] + [ip] * 4
    L.zr_global_to_reciprocal.argtypes = [ctypes.c_int, ctypes.c_int] + [ip] * 4
    L.zr_global_to_real_3d.argtypes = [ctypes.c_int] * 3 + [ip] * 6
    L.zr_global_to_reciprocal_3d.argtypes = [ctypes.c_int] * 3 + [ip] * 6
    return L


def ref_available() -> bool:
    return REF_DIR.exists() and any(REF_DIR.glob("libzref_host_*.so"))


os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")
