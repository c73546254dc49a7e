"""Batch: many independent 2D fields of uneven N, each on its own (N, B, P) layout,
processed by one persistent launch per call (the zm_batch_* entry points).

Batch buffers are flat device tensors of ``total`` elements; field i occupies
``[offset_i, offset_i + N_i^2)`` in the reference layout of its own plan.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

from . import abi
from .abi import check, lib
from .plan import _DT, _ptr, _stream_ptr


class Batch:
    def __init__(self, ns: Sequence[int], bs: Sequence[int], ps: Sequence[int], dtype="c64"):
        if not (len(ns) == len(bs) == len(ps)) or len(ns) == 0:
            raise ValueError("ns, bs and ps must be non-empty and of equal length")
        self.dtype = _DT[dtype]
        arr = ctypes.c_int64 * len(ns)
        h = ctypes.c_void_p()
        check(lib().zm_batch_create(ctypes.byref(h), len(ns), arr(*ns), arr(*bs), arr(*ps), self.dtype),
              "zm_batch_create")
        self._h = h
        tot = ctypes.c_int64()
        check(lib().zm_batch_total_elems(self._h, ctypes.byref(tot)), "zm_batch_total_elems")
        self.total = tot.value
        self.fields = []
        for i in range(len(ns)):
            f = abi.zm_batch_field()
            check(lib().zm_batch_get_field(self._h, i, ctypes.byref(f)), "zm_batch_get_field")
            self.fields.append({"n": f.n, "b": f.b, "p": f.p, "offset": f.offset, "elems": f.elems})

    @property
    def torch_dtype(self):
        import torch
        return torch.complex128 if self.dtype == abi.ZM_C128 else torch.complex64

    def empty(self, device="cuda"):
        import torch
        return torch.empty(self.total, dtype=self.torch_dtype, device=device)

    def field(self, buf, i: int):
        """View of field i (its N^2 elements in its plan's layout) inside a batch buffer."""
        f = self.fields[i]
        return buf[f["offset"]:f["offset"] + f["elems"]]

    def _check(self, t, name):
        if t is None:
            raise ValueError(f"{name} is required")
        if t.dtype != self.torch_dtype or t.numel() < self.total or not t.is_cuda or not t.is_contiguous():
            raise ValueError(f"{name}: expected a contiguous CUDA {self.torch_dtype} tensor of >= "
                             f"{self.total} elements")

    def fill(self, out, kind: int = abi.ZM_FIELD_GAUSSIAN, first_seed: int = 0, stream=None):
        self._check(out, "out")
        check(lib().zm_batch_fill(self._h, _ptr(out), int(kind), int(first_seed), _stream_ptr(stream)),
              "zm_batch_fill")
        return out

    def forward_fft(self, inp, out, stream=None):
        self._check(inp, "in"), self._check(out, "out")
        check(lib().zm_batch_forward(self._h, _ptr(inp), _ptr(out), _stream_ptr(stream)), "zm_batch_forward")
        return out

    def inverse_fft(self, inp, out, work=None, normalise: bool = True, stream=None):
        self._check(inp, "in"), self._check(out, "out")
        check(lib().zm_batch_inverse(self._h, _ptr(inp), _ptr(out), _ptr(work), int(bool(normalise)),
                                     _stream_ptr(stream)), "zm_batch_inverse")
        return out

    def poisson(self, rhs, phi, residual, work, length: float = 1.0, stream=None):
        """phi = IFFT(FFT(rhs) / -(2 pi |k| / length)^2), k = 0 -> 0; residual = Lap_h(phi) - rhs."""
        self._check(rhs, "rhs"), self._check(phi, "phi"), self._check(work, "work")
        if residual is not None:
            self._check(residual, "residual")
        check(lib().zm_batch_poisson(self._h, _ptr(rhs), _ptr(phi), _ptr(residual), _ptr(work),
                                     float(length), _stream_ptr(stream)), "zm_batch_poisson")
        return phi

    def status(self) -> int:
        """Synchronise; 1 if a grid barrier timed out since the last call (flag cleared)."""
        v = ctypes.c_int()
        check(lib().zm_batch_status(self._h, ctypes.byref(v)), "zm_batch_status")
        return v.value

    def barrier_probe(self, missing: int, stream=None) -> None:
        """Launch the grid-barrier probe (missing = 1: the barrier times out by design)."""
        check(lib().zm_batch_barrier_probe(self._h, int(missing), _stream_ptr(stream)), "zm_batch_barrier_probe")

    @staticmethod
    def autotune_b(n: int, p: int, dtype="c64", count: int = 4, reps: int = 3) -> tuple[int, float]:
        b, ms = ctypes.c_int64(), ctypes.c_float()
        check(lib().zm_batch_autotune_b(int(n), int(p), _DT[dtype], int(count), int(reps), ctypes.byref(b),
                                        ctypes.byref(ms)), "zm_batch_autotune_b")
        return b.value, ms.value

    def close(self):
        if getattr(self, "_h", None):
            lib().zm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
