"""ctypes front end of the reference's own GPU pipeline (TEST INFRASTRUCTURE ONLY).

`oracle/_ref/libzref_gpu_N<n>_B<b>_P<p>[_aware].so` is the reference's unmodified zmodel
CUDA code (utils.cu, transforms/fft.cu, fft3d.cu, stencils/laplace.cu, laplace3d.cu, dx.cu,
dy.cu) with cuFFT, built by `make -C oracle ref-gpu REF_ROOT=...` together with the
thread-per-rank MPI stand-in of `oracle/refgpu/`.  One call runs every virtual rank of
the reference as a host thread on the current GPU and returns the whole grid.  Arrays
use the same whole-grid layout as the library and the C oracle: rank-major, each rank in
the reference's rank-local layout.  Only tests call this module.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_LOG = 1 << 16
_P = ctypes.c_void_p


def lib_path(n: int, b: int, p: int, gpu_aware: bool = False) -> Path:
    return REF_DIR / f"libzref_gpu_N{n}_B{b}_P{p}{'_aware' if gpu_aware else ''}.so"


def available(n: int, b: int, p: int, gpu_aware: bool = False) -> bool:
    return lib_path(n, b, p, gpu_aware).exists()


def stage_times(log: str) -> dict:
    """The reference's own TIME_MPI_MAX_NS prints ("FFT0 123 ns", fft.cu:8-18) -> {tag: [ns]}."""
    out: dict = {}
    for tag, ns in re.findall(r"^([A-Z_0-9]+) (\d+) ns$", log, flags=re.M):
        out.setdefault(tag, []).append(int(ns))
    return out


class RefPipeline:
    """The reference pipeline compiled for one (N_DIM, B_DIM, P_DIM)."""

    def __init__(self, n: int, b: int, p: int, gpu_aware: bool = False):
        path = lib_path(n, b, p, gpu_aware)
        if not path.exists():
            raise FileNotFoundError(f"{path.name} not built (make -C oracle ref-gpu REF_ROOT=...)")
        L = ctypes.CDLL(str(path))
        i = ctypes.c_int
        L.zr_config.argtypes = [ctypes.POINTER(i)] * 4
        L.zr_fft.argtypes = [i, _P, _P, i, i, ctypes.c_double, ctypes.c_double, i,
                             ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, i]
        L.zr_laplace.argtypes = [i, _P, _P, i, ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, i]
        L.zr_dxdy.argtypes = [i, _P, _P, ctypes.c_double]
        for f in (L.zr_config, L.zr_fft, L.zr_laplace, L.zr_dxdy):
            f.restype = i
        vals = [i() for _ in range(4)]
        L.zr_config(*[ctypes.byref(v) for v in vals])
        self.n, self.b, self.p, aware = (v.value for v in vals)
        assert (self.n, self.b, self.p) == (n, b, p), path
        self.gpu_aware = bool(aware)
        self._lib = L

    @staticmethod
    def _arr(x, dtype):
        a = np.ascontiguousarray(x, dtype=dtype)
        return a, a.ctypes.data_as(_P)

    def _check(self, x, dim):
        if x.size != self.n ** dim:
            raise ValueError(f"expected {self.n ** dim} elements, got {x.size}")

    def fft(self, x, dim: int, inverse: bool = False, do_compute: bool = True,
            scale: complex = 1.0, reps: int = 0):
        """forward_fft / inverse_fft (or the _3d forms); returns (out, mean ms, log)."""
        self._check(x, dim)
        a, pa = self._arr(x, np.complex128)
        out = np.empty_like(a)
        ms = ctypes.c_double()
        log = ctypes.create_string_buffer(_LOG)
        s = complex(scale)
        rc = self._lib.zr_fft(dim, pa, out.ctypes.data_as(_P), int(inverse), int(do_compute),
                              s.real, s.imag, int(reps), ctypes.byref(ms), log, _LOG)
        if rc != 0:
            raise RuntimeError(f"reference fft failed (rc={rc})")
        return out, ms.value, log.value.decode(errors="replace")

    def laplace(self, x, dim: int, reps: int = 0):
        """pack_laplace + communicate_laplace + laplace (or the 3D chain); (out, ms, log)."""
        self._check(x, dim)
        a, pa = self._arr(x, np.complex128)
        out = np.empty_like(a)
        ms = ctypes.c_double()
        log = ctypes.create_string_buffer(_LOG)
        rc = self._lib.zr_laplace(dim, pa, out.ctypes.data_as(_P), int(reps), ctypes.byref(ms), log, _LOG)
        if rc != 0:
            raise RuntimeError(f"reference laplace failed (rc={rc})")
        return out, ms.value, log.value.decode(errors="replace")

    def _deriv(self, axis, x, delta):
        self._check(x, 2)
        a, pa = self._arr(x, np.float64)
        out = np.empty_like(a)
        rc = self._lib.zr_dxdy(axis, pa, out.ctypes.data_as(_P), float(delta))
        if rc != 0:
            raise RuntimeError(f"reference dx/dy failed (rc={rc}; needs B >= 2)")
        return out

    def dx(self, x, delta: float = 1.0):
        """The reference's real (Scalar) dx kernel over every rank."""
        return self._deriv(0, x, delta)

    def dy(self, x, delta: float = 1.0):
        return self._deriv(1, x, delta)
