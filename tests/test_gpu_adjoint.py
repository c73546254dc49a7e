"""Adjoint of a spectral-solve pipeline through the VJP entry points (2D complex64,
N = 4096, P = 4, B = 32; u, t ~ N(0,1) from the counter generator, seeds 3 and 4):

    L(u) = || Lap(IFFT(G * FFT(u))) - t ||^2,   G(k) = exp(-|k|^2 / (2 (N/16)^2))

with k the signed frequency, IFFT normalised by 1/N^2 and Lap the reference's periodic
5-point Laplacian (no 1/h^2).  Gradient convention: dL/du = dL/dRe(u) + i dL/dIm(u)
= 2 A^H (A u - t) for the linear map A.  Checked by the adjoint dot-product test, by
central finite differences along 16 random directions recomputed in FP64 (the complex128
plan), and against an FP64 numpy gradient."""
import numpy as np
import pytest

import oracle as O
from helpers import to_host

pytestmark = pytest.mark.gpu

N, B, P = 4096, 32, 4
SIGMA = N / 16


def _plans():
    from stencilfft_b200 import Plan
    return Plan(2, N, B, P, dtype="c64"), Plan(2, N, B, P, dtype="c128")


class _Pipeline:
    """A and A^H of the loss on one plan, with preallocated temporaries."""

    def __init__(self, pl):
        from stencilfft_b200 import abi
        self.pl, self.op = pl, abi.ZM_SPECTRAL_GAUSSIAN
        self.spec, self.tmp, self.work = pl.empty(), pl.empty(), pl.empty()

    def forward(self, u, out):
        pl = self.pl
        pl.forward_fft(u, self.spec, work=self.work)
        pl.spectral_apply(self.spec, self.op, SIGMA)
        pl.inverse_fft(self.spec, self.tmp, scale=1.0 / N ** 2, work=self.work)
        pl.laplace(self.tmp, out)
        return out

    def adjoint(self, r, out):
        pl = self.pl
        pl.laplace_vjp(r, self.tmp)
        pl.inverse_fft_vjp(self.tmp, self.spec, scale=1.0 / N ** 2, work=self.work)
        pl.spectral_apply_vjp(self.spec, self.op, SIGMA)
        pl.forward_fft_vjp(self.spec, out, work=self.work)
        return out


def _cdot(a, b):
    """<a, b> = sum conj(a) b in FP64 on the device."""
    import torch
    return complex(torch.vdot(a.to(torch.complex128), b.to(torch.complex128)))


def _norm(a):
    import torch
    return float(torch.linalg.vector_norm(a.to(torch.complex128)))


def _inputs(pl):
    from stencilfft_b200 import abi
    u, t = pl.empty(), pl.empty()
    pl.fill(u, abi.ZM_FIELD_GAUSSIAN, 3)
    pl.fill(t, abi.ZM_FIELD_GAUSSIAN, 4)
    return u, t


def _gradient(pipe, u, t):
    r = pipe.forward(u, pipe.pl.empty())
    r.sub_(t)
    g = pipe.adjoint(r, pipe.pl.empty())
    g.mul_(2.0)
    return g


def test_pipeline_dot_product():
    """<A x, y> = <x, A^H y> for the composite map, rel <= 1e-5 in complex64."""
    from stencilfft_b200 import abi
    pl, _ = _plans()
    pipe = _Pipeline(pl)
    x, y = pl.empty(), pl.empty()
    pl.fill(x, abi.ZM_FIELD_GAUSSIAN, 11)
    pl.fill(y, abi.ZM_FIELD_GAUSSIAN, 12)
    ax = pipe.forward(x, pl.empty())
    ahy = pipe.adjoint(y, pl.empty())
    lhs, rhs = _cdot(ax, y), _cdot(x, ahy)
    rel = abs(lhs - rhs) / abs(lhs)
    print(f"\nadjoint dot-product (pipeline, c64 N={N}): rel {rel:.3e}")
    assert rel <= 1e-5, (lhs, rhs)


def test_gradient_central_differences_fp64():
    """Re<dL/du, d> against (L(u + eps d) - L(u - eps d)) / (2 eps), eps = 1e-3, with L
    recomputed in FP64 (complex128 plan) at the complex64 inputs; 16 directions."""
    import torch
    from stencilfft_b200 import abi
    pl64, pl128 = _plans()
    u, t = _inputs(pl64)
    g = _gradient(_Pipeline(pl64), u, t)
    pipe128 = _Pipeline(pl128)
    u128, t128 = u.to(torch.complex128), t.to(torch.complex128)
    tmp, d = pl128.empty(), pl128.empty()
    eps = 1e-3

    def loss(v):
        pipe128.forward(v, tmp)
        tmp.sub_(t128)
        return _norm(tmp) ** 2

    gnorm = _norm(g)
    worst = 0.0
    for i in range(16):
        pl128.fill(d, abi.ZM_FIELD_GAUSSIAN, 1000 + i)
        fd = (loss(u128 + eps * d) - loss(u128 - eps * d)) / (2 * eps)
        an = _cdot(g, d).real
        err = abs(fd - an) / (gnorm * _norm(d))
        worst = max(worst, err)
    print(f"\ncentral differences (16 directions, eps={eps}, FP64 recompute): worst "
          f"|FD - Re<g,d>| / (|g| |d|) = {worst:.3e}")
    # the c64 gradient carries ~1e-7 relative rounding; a direction can pick up at most
    # that fraction of |g| |d|
    assert worst <= 2e-6, worst


def test_gradient_against_fp64_reference():
    """The complex64 adjoint gradient against dL/du computed with numpy in FP64:
    2 ifft2(G fft2(Lap(Lap(ifft2(G fft2 u)) - t))), rel-L2 <= 1e-5."""
    pl64, _ = _plans()
    u, t = _inputs(pl64)
    g = _gradient(_Pipeline(pl64), u, t)
    un = O.real_layout_to_natural(to_host(u), 2, N, B, P)
    tn = O.real_layout_to_natural(to_host(t), 2, N, B, P)
    k = np.fft.fftfreq(N, 1.0 / N)
    G = np.exp(-(k[:, None] ** 2 + k[None, :] ** 2) / (2 * SIGMA ** 2))

    def lap(x):
        return (np.roll(x, 1, 0) + np.roll(x, -1, 0) + np.roll(x, 1, 1) + np.roll(x, -1, 1) - 4 * x)

    r = lap(np.fft.ifft2(G * np.fft.fft2(un))) - tn
    g_ref = 2 * np.fft.ifft2(G * np.fft.fft2(lap(r)))
    gn = O.real_layout_to_natural(to_host(g), 2, N, B, P)
    err = np.linalg.norm(gn - g_ref) / np.linalg.norm(g_ref)
    print(f"\nc64 adjoint gradient vs FP64 numpy gradient: rel-L2 {err:.3e}")
    assert err <= 1e-5, err


def test_adjoint_cost_close_to_forward():
    """The VJP chain runs the same kernels as the forward chain (conjugate-direction
    passes, the transposed stencil): its device time stays within 1.2x of the forward."""
    import torch
    pl, _ = _plans()
    pipe = _Pipeline(pl)
    u, t = _inputs(pl)
    out = pl.empty()

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    tf = timed(lambda: pipe.forward(u, out))
    ta = timed(lambda: pipe.adjoint(t, out))
    print(f"\nforward chain {tf:.3f} ms, VJP chain {ta:.3f} ms, ratio {ta / tf:.3f}")
    assert ta <= 1.2 * tf, (ta, tf)
