"""Plan: the host-side mirror of the zmodel entry points over one whole virtual-rank grid.

The reference exposes, per MPI rank, ``forward_fft<do_compute>(FftBuffers&, row_comm,
col_comm, id, plans, ctx)`` and friends (zmodel/transforms/fft.h:28-64,
zmodel/stencils/laplace.h:28-38, dx.cu:10, dy.cu:10).  Here one call processes every
virtual rank: the communicators and rank id are folded into the plan, and the
buffers are whole-grid device tensors (rank-major, each rank in the reference's
rank-local layout).  Like the reference, ``forward_fft(buf0, buf1)`` reads buf0 and
writes buf1, and transforms may use buf0 as scratch unless a workspace is given.
"""
from __future__ import annotations

import ctypes
from typing import Optional

from . import abi
from .abi import check, lib

_DT = {"c128": abi.ZM_C128, "c64": abi.ZM_C64, abi.ZM_C128: abi.ZM_C128, abi.ZM_C64: abi.ZM_C64}


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _ptr(t) -> int:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


class Plan:
    """Immutable description of an N^dim field on a P^dim virtual-rank grid with B x B blocks."""

    def __init__(self, dim: int, n: int, b: int, p: int, dtype="c128", permute_only: bool = False,
                 host_only: bool = False, own_workspace: bool = False):
        """host_only: no device resources (ZM_FLAG_HOST_ONLY) -- sizes and index maps only.
        own_workspace: the plan holds one field of workspace (ZM_FLAG_OWN_WORKSPACE), used by
        transforms called without `work`; such calls must not overlap on two streams."""
        self._h = ctypes.c_void_p()
        flags = ((abi.ZM_FLAG_PERMUTE_ONLY if permute_only else 0) | (abi.ZM_FLAG_HOST_ONLY if host_only else 0)
                 | (abi.ZM_FLAG_OWN_WORKSPACE if own_workspace else 0))
        if dtype not in _DT:
            raise ValueError(f"dtype must be 'c128' or 'c64', got {dtype!r}")
        check(lib().zm_plan_create(ctypes.byref(self._h), int(dim), int(n), int(b), int(p),
                                   _DT[dtype], flags), "zm_plan_create")
        info = abi.zm_plan_info()
        check(lib().zm_plan_get_info(self._h, ctypes.byref(info)), "zm_plan_get_info")
        self.info = info
        self.dim, self.n, self.b, self.p = dim, n, b, p
        self.dtype = "c128" if _DT[dtype] == abi.ZM_C128 else "c64"
        self.permute_only = permute_only

    # ------------------------------------------------------------ properties
    @property
    def handle(self):
        return self._h

    @property
    def total(self) -> int:
        return int(self.info.total_elems)

    @property
    def field_bytes(self) -> int:
        return int(self.info.field_bytes)

    @property
    def torch_dtype(self):
        import torch
        return torch.complex128 if self.dtype == "c128" else torch.complex64

    def derived(self) -> dict:
        i = self.info
        return {"L": i.local_dim, "VEC": i.vec, "VP": i.vec_split, "M": i.m, "ranks": i.ranks,
                "rank_elems": i.rank_elems}

    def empty(self, device="cuda", real: bool = False):
        import torch
        if real:
            dt = torch.float64 if self.dtype == "c128" else torch.float32
        else:
            dt = self.torch_dtype
        return torch.empty(self.total, dtype=dt, device=device)

    def _check(self, t, name, real=False):
        import torch
        if t is None:
            raise ValueError(f"{name} is None")
        if not t.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor")
        exp = (torch.float64 if self.dtype == "c128" else torch.float32) if real else self.torch_dtype
        if t.dtype != exp:
            raise TypeError(f"{name} has dtype {t.dtype}, plan expects {exp}")
        if t.numel() != self.total or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous tensor of {self.total} elements")

    # ------------------------------------------------------------ tuning
    @property
    def kernel_variants(self) -> int:
        n = ctypes.c_int()
        check(lib().zm_plan_kernel_variants(self._h, ctypes.byref(n)), "zm_plan_kernel_variants")
        return n.value

    def set_kernel_variant(self, variant: int) -> None:
        check(lib().zm_plan_set_kernel_variant(self._h, int(variant)), "zm_plan_set_kernel_variant")

    def device_status(self) -> int:
        """Synchronise; 1 if a bounded wait in one of this plan's kernels gave up (cleared)."""
        v = ctypes.c_int()
        check(lib().zm_plan_device_status(self._h, ctypes.byref(v)), "zm_plan_device_status")
        return v.value

    def autotune(self, a, b, work=None, reps: int = 3, stream=None) -> tuple[int, float]:
        """Time a forward + inverse round trip per kernel variant and keep the fastest.

        `a`, `b`, `work` are overwritten; returns (variant, ms per round trip)."""
        self._check(a, "a"), self._check(b, "b")
        v, ms = ctypes.c_int(), ctypes.c_float()
        check(lib().zm_plan_autotune(self._h, _ptr(a), _ptr(b), _ptr(work), int(reps), _stream_ptr(stream),
                                     ctypes.byref(v), ctypes.byref(ms)), "zm_plan_autotune")
        return v.value, ms.value

    # ------------------------------------------------------------ transforms
    def forward_fft(self, buf0, buf1, work=None, stream=None):
        """forward_fft / forward_fft_3d: real layout buf0 -> reciprocal layout buf1."""
        self._check(buf0, "buf0"), self._check(buf1, "buf1")
        check(lib().zm_fft_forward(self._h, _ptr(buf0), _ptr(buf1), _ptr(work), _stream_ptr(stream)),
              "zm_fft_forward")
        return buf1

    def inverse_fft(self, buf0, buf1, scale: complex = 1.0, work=None, stream=None):
        """inverse_fft / inverse_fft_3d: reciprocal layout buf0 -> real layout buf1, times scale."""
        self._check(buf0, "buf0"), self._check(buf1, "buf1")
        s = complex(scale)
        check(lib().zm_fft_inverse(self._h, _ptr(buf0), _ptr(buf1), _ptr(work), s.real, s.imag,
                                   _stream_ptr(stream)), "zm_fft_inverse")
        return buf1

    forward_fft_3d = forward_fft
    inverse_fft_3d = inverse_fft

    # -------------------------------------------------------------- stencils
    def laplace(self, inp, out, inv_h2: float = 1.0, stream=None):
        self._check(inp, "in"), self._check(out, "out")
        check(lib().zm_laplace(self._h, _ptr(inp), _ptr(out), float(inv_h2), _stream_ptr(stream)),
              "zm_laplace")
        return out

    laplace_3d = laplace

    def laplace_dx_dy(self, inp, lap, gx, gy, inv_h2: float = 1.0, delta: float = 1.0, stream=None):
        """Laplacian, dx and dy of a 2D complex field in one launch (each bit-identical to
        laplace / dx / dy)."""
        for t, nm in ((inp, "in"), (lap, "lap"), (gx, "dx"), (gy, "dy")):
            self._check(t, nm)
        check(lib().zm_laplace_dx_dy(self._h, _ptr(inp), _ptr(lap), _ptr(gx), _ptr(gy), float(inv_h2),
                                     float(delta), _stream_ptr(stream)), "zm_laplace_dx_dy")
        return lap, gx, gy

    def dx(self, inp, out, delta: float = 1.0, stream=None):
        real = not inp.is_complex()
        self._check(inp, "in", real), self._check(out, "out", real)
        f = lib().zm_dx_real if real else lib().zm_dx
        check(f(self._h, _ptr(inp), _ptr(out), float(delta), _stream_ptr(stream)), "zm_dx")
        return out

    def dy(self, inp, out, delta: float = 1.0, stream=None):
        real = not inp.is_complex()
        self._check(inp, "in", real), self._check(out, "out", real)
        f = lib().zm_dy_real if real else lib().zm_dy
        check(f(self._h, _ptr(inp), _ptr(out), float(delta), _stream_ptr(stream)), "zm_dy")
        return out

    # ------------------------------------------------------------------ VJPs
    def forward_fft_vjp(self, grad_out, grad_in, work=None, stream=None):
        self._check(grad_out, "grad_out"), self._check(grad_in, "grad_in")
        check(lib().zm_fft_forward_vjp(self._h, _ptr(grad_out), _ptr(grad_in), _ptr(work),
                                       _stream_ptr(stream)), "zm_fft_forward_vjp")
        return grad_in

    def inverse_fft_vjp(self, grad_out, grad_in, scale: complex = 1.0, work=None, stream=None):
        self._check(grad_out, "grad_out"), self._check(grad_in, "grad_in")
        s = complex(scale)
        check(lib().zm_fft_inverse_vjp(self._h, _ptr(grad_out), _ptr(grad_in), _ptr(work), s.real,
                                       s.imag, _stream_ptr(stream)), "zm_fft_inverse_vjp")
        return grad_in

    def laplace_vjp(self, grad_out, grad_in, inv_h2: float = 1.0, stream=None):
        self._check(grad_out, "grad_out"), self._check(grad_in, "grad_in")
        check(lib().zm_laplace_vjp(self._h, _ptr(grad_out), _ptr(grad_in), float(inv_h2),
                                   _stream_ptr(stream)), "zm_laplace_vjp")
        return grad_in

    def dx_vjp(self, grad_out, grad_in, delta: float = 1.0, stream=None):
        self._check(grad_out, "grad_out"), self._check(grad_in, "grad_in")
        check(lib().zm_dx_vjp(self._h, _ptr(grad_out), _ptr(grad_in), float(delta),
                              _stream_ptr(stream)), "zm_dx_vjp")
        return grad_in

    def dy_vjp(self, grad_out, grad_in, delta: float = 1.0, stream=None):
        self._check(grad_out, "grad_out"), self._check(grad_in, "grad_in")
        check(lib().zm_dy_vjp(self._h, _ptr(grad_out), _ptr(grad_in), float(delta),
                              _stream_ptr(stream)), "zm_dy_vjp")
        return grad_in

    # ---------------------------------------------------- layouts / operators
    def natural_to_real(self, natural, out, stream=None):
        check(lib().zm_natural_to_real(self._h, _ptr(natural), _ptr(out), _stream_ptr(stream)),
              "zm_natural_to_real")
        return out

    def real_to_natural(self, buf, out, stream=None):
        check(lib().zm_real_to_natural(self._h, _ptr(buf), _ptr(out), _stream_ptr(stream)),
              "zm_real_to_natural")
        return out

    def natural_to_reciprocal(self, natural, out, stream=None):
        check(lib().zm_natural_to_reciprocal(self._h, _ptr(natural), _ptr(out), _stream_ptr(stream)),
              "zm_natural_to_reciprocal")
        return out

    def reciprocal_to_natural(self, buf, out, stream=None):
        check(lib().zm_reciprocal_to_natural(self._h, _ptr(buf), _ptr(out), _stream_ptr(stream)),
              "zm_reciprocal_to_natural")
        return out

    def spectral_apply(self, data, op: int, a: float, stream=None):
        self._check(data, "data")
        check(lib().zm_spectral_apply(self._h, _ptr(data), int(op), float(a), _stream_ptr(stream)),
              "zm_spectral_apply")
        return data

    def spectral_apply_vjp(self, grad, op: int, a: float, stream=None):
        """VJP of spectral_apply (in place; the real diagonal multipliers are self-adjoint)."""
        self._check(grad, "grad")
        check(lib().zm_spectral_apply_vjp(self._h, _ptr(grad), int(op), float(a), _stream_ptr(stream)),
              "zm_spectral_apply_vjp")
        return grad

    def fill(self, out, kind: int, seed: int, stream=None):
        self._check(out, "out")
        check(lib().zm_fill_field(self._h, _ptr(out), int(kind), int(seed), _stream_ptr(stream)),
              "zm_fill_field")
        return out

    def fill_modes(self, out, modes, amps, noise: float, seed: int, stream=None):
        import numpy as np
        self._check(out, "out")
        m = np.ascontiguousarray(np.asarray(modes, dtype=np.int64).reshape(-1))
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.float64).reshape(-1))
        n = len(m) // 2
        check(lib().zm_fill_modes(self._h, _ptr(out), n, m.ctypes.data_as(abi._PI64),
                                  a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), float(noise),
                                  int(seed), _stream_ptr(stream)), "zm_fill_modes")
        return out

    # ----------------------------------------------------------- index maps
    def real_to_global(self, rid, cid, lr, lc, did=0, ld=0):
        o = [ctypes.c_int64() for _ in range(3)]
        check(lib().zm_real_to_global(self._h, rid, cid, did, ld, lr, lc, *map(ctypes.byref, o)),
              "zm_real_to_global")
        gd, gr, gc = (v.value for v in o)
        return (gr, gc) if self.dim == 2 else (gd, gr, gc)

    def global_to_real(self, *g):
        gd, gr, gc = (0, *g) if self.dim == 2 else g
        o = [ctypes.c_int64() for _ in range(6)]
        check(lib().zm_global_to_real(self._h, gd, gr, gc, *map(ctypes.byref, o)), "zm_global_to_real")
        rid, cid, did, ld, lr, lc = (v.value for v in o)
        return (rid, cid, lr, lc) if self.dim == 2 else (rid, cid, did, ld, lr, lc)

    def reciprocal_to_global(self, rid, cid, lr, lc, did=0, ld=0):
        o = [ctypes.c_int64() for _ in range(3)]
        check(lib().zm_reciprocal_to_global(self._h, rid, cid, did, ld, lr, lc, *map(ctypes.byref, o)),
              "zm_reciprocal_to_global")
        kd, kr, kc = (v.value for v in o)
        return (kr, kc) if self.dim == 2 else (kd, kr, kc)

    def global_to_reciprocal(self, *k):
        kd, kr, kc = (0, *k) if self.dim == 2 else k
        o = [ctypes.c_int64() for _ in range(6)]
        check(lib().zm_global_to_reciprocal(self._h, kd, kr, kc, *map(ctypes.byref, o)),
              "zm_global_to_reciprocal")
        rid, cid, did, ld, lr, lc = (v.value for v in o)
        return (rid, cid, lr, lc) if self.dim == 2 else (rid, cid, did, ld, lr, lc)

    # ------------------------------------------------------------ lifetime
    def close(self):
        if self._h and self._h.value:
            lib().zm_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def autotune_b(dim: int, n: int, p: int, dtype="c64", reps: int = 2) -> tuple[int, int, float]:
    """Fastest (B, kernel variant, ms per forward + inverse round trip) for an N^dim field
    on a P^dim grid (zm_autotune_b)."""
    b, v, ms = ctypes.c_int64(), ctypes.c_int(), ctypes.c_float()
    check(lib().zm_autotune_b(int(dim), int(n), int(p), _DT[dtype], int(reps), ctypes.byref(b), ctypes.byref(v),
                              ctypes.byref(ms)), "zm_autotune_b")
    return b.value, v.value, ms.value
