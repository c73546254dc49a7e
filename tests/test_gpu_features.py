"""GPU tests of the features around the transforms: adjoints (VJPs), layout
converters, reciprocal-space operators, seeded generators and error paths."""
import ctypes

import numpy as np
import pytest

import oracle as O
from helpers import TOL, rand_field, relerr, to_dev, to_host

pytestmark = pytest.mark.gpu


def _plan(dim, n, b, p, dt, **kw):
    from stencilfft_b200 import Plan
    return Plan(dim, n, b, p, dtype=dt, **kw)


def _vdot(a, b):
    return np.vdot(a.ravel(), b.ravel())


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("dim,n,b,p", [(2, 64, 4, 2), (2, 256, 16, 4), (3, 32, 2, 4)])
def test_adjoint_dot_products(dim, n, b, p, dt):
    """<A x, y> = <x, A^H y> for the forward/inverse transforms and the stencils."""
    import torch
    pl = _plan(dim, n, b, p, dt)
    x = O.natural_to_real_layout(rand_field(dim, n, 1), b, p)
    y = O.natural_to_real_layout(rand_field(dim, n, 2), b, p)
    dx_, dy_ = to_dev(x, dt), to_dev(y, dt)
    t1, t2, w = torch.empty_like(dx_), torch.empty_like(dx_), torch.empty_like(dx_)
    tol = 1e-12 if dt == "c128" else 1e-5
    # forward FFT
    pl.forward_fft(dx_, t1, work=w)
    pl.forward_fft_vjp(dy_, t2, work=w)
    lhs, rhs = _vdot(to_host(t1), y), _vdot(x, to_host(t2))
    assert abs(lhs - rhs) / abs(lhs) < tol
    # inverse FFT with a complex scale
    s = complex(0.3, -0.7) / n ** dim
    pl.inverse_fft(dx_, t1, scale=s, work=w)
    pl.inverse_fft_vjp(dy_, t2, scale=s, work=w)
    lhs, rhs = _vdot(to_host(t1), y), _vdot(x, to_host(t2))
    assert abs(lhs - rhs) / abs(lhs) < tol
    # Laplacian (self-adjoint)
    pl.laplace(dx_, t1, inv_h2=2.0)
    pl.laplace_vjp(dy_, t2, inv_h2=2.0)
    lhs, rhs = _vdot(to_host(t1), y), _vdot(x, to_host(t2))
    assert abs(lhs - rhs) / abs(lhs) < tol
    if dim == 2:
        for f, fv in ((pl.dx, pl.dx_vjp), (pl.dy, pl.dy_vjp)):
            f(dx_, t1, delta=0.5)
            fv(dy_, t2, delta=0.5)
            lhs, rhs = _vdot(to_host(t1), y), _vdot(x, to_host(t2))
            assert abs(lhs - rhs) / abs(lhs) < tol


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("dim,n,b,p", [(2, 64, 4, 2), (2, 128, 8, 4), (3, 16, 2, 2), (3, 32, 2, 4),
                                       # the tiled reciprocal converter: runs of 4, 8, 16, 32
                                       (2, 4096, 64, 4), (2, 1024, 32, 2), (2, 2048, 32, 2),
                                       (2, 2048, 16, 2), (3, 256, 8, 2)])
def test_layout_converters(dim, n, b, p, dt):
    import torch
    pl = _plan(dim, n, b, p, dt)
    x = rand_field(dim, n, 4)
    nat = to_dev(x.reshape(-1), dt)
    inter = torch.empty_like(nat)
    pl.natural_to_real(nat, inter)
    exp = O.natural_to_real_layout(x, b, p)
    assert np.array_equal(to_host(inter), exp.astype(np.complex64 if dt == "c64" else np.complex128))
    back = torch.empty_like(nat)
    pl.real_to_natural(inter, back)
    assert torch.equal(back, nat)
    pl.natural_to_reciprocal(nat, inter)
    exp = O.natural_to_reciprocal_layout(x, b, p)
    assert np.array_equal(to_host(inter), exp.astype(np.complex64 if dt == "c64" else np.complex128))
    pl.reciprocal_to_natural(inter, back)
    assert torch.equal(back, nat)


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_spectral_poisson_roundtrip(dt):
    """forward -> divide by -|k|^2 -> inverse solves the periodic Poisson equation
    (the C5 pipeline's pointwise step); checked against numpy in natural layout."""
    import torch
    from stencilfft_b200 import abi
    dim, n, b, p = 2, 128, 8, 2
    pl = _plan(dim, n, b, p, dt)
    x = rand_field(dim, n, 6)
    buf = O.natural_to_real_layout(x, b, p)
    d0 = to_dev(buf, dt)
    d1, w = torch.empty_like(d0), torch.empty_like(d0)
    pl.forward_fft(d0, d1, work=w)
    a = 2 * np.pi          # h = 1/N: physical wavenumber = 2 pi k
    pl.spectral_apply(d1, abi.ZM_SPECTRAL_POISSON, a)
    pl.inverse_fft(d1, d0, scale=1.0 / n ** 2, work=w)
    got = O.real_layout_to_natural(to_host(d0), dim, n, b, p)
    k = np.fft.fftfreq(n, 1.0 / n)
    K2 = (k[:, None] ** 2 + k[None, :] ** 2) * a * a
    F = np.fft.fft2(x)
    with np.errstate(divide="ignore", invalid="ignore"):
        F = np.where(K2 == 0, 0, F / -K2)
    assert relerr(got, np.fft.ifft2(F)) < TOL[dt] * 10
    # Gaussian filter
    d0.copy_(to_dev(buf, dt))
    pl.forward_fft(d0, d1, work=w)
    pl.spectral_apply(d1, abi.ZM_SPECTRAL_GAUSSIAN, n / 16)
    pl.inverse_fft(d1, d0, scale=1.0 / n ** 2, work=w)
    got = O.real_layout_to_natural(to_host(d0), dim, n, b, p)
    G = np.exp(-(k[:, None] ** 2 + k[None, :] ** 2) / (2 * (n / 16) ** 2))
    assert relerr(got, np.fft.ifft2(G * np.fft.fft2(x))) < TOL[dt] * 10


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_generators_match_oracle_stream(dt):
    import torch
    from stencilfft_b200 import abi
    dim, n, b, p = 2, 256, 8, 4
    pl = _plan(dim, n, b, p, dt)
    d = pl.empty()
    pl.fill(d, abi.ZM_FIELD_UNIFORM, 11)
    exp = O.natural_to_real_layout(O.uniform_field(11, n * n).reshape(n, n), b, p)
    got = to_host(d)
    if dt == "c128":
        assert np.array_equal(got, exp)
    else:
        assert np.array_equal(got, exp.astype(np.complex64))
    pl.fill(d, abi.ZM_FIELD_GAUSSIAN, 2)
    exp = O.natural_to_real_layout(O.gaussian_field(2, n * n).reshape(n, n), b, p)
    assert relerr(to_host(d), exp) < (1e-13 if dt == "c128" else 1e-6)
    # plane waves: the FFT of one mode is a single spike
    pl.fill_modes(d, [[3, -5]], [[2.0, 1.0]], 0.0, 0)
    out, w = torch.empty_like(d), torch.empty_like(d)
    pl.forward_fft(d, out, work=w)
    X = O.reciprocal_layout_to_natural(to_host(out), 2, n, b, p)
    spike = np.zeros((n, n), complex)
    spike[(-5) % n, 3] = (2 + 1j) * n * n
    assert relerr(X, spike) < TOL[dt] * 10


def test_error_paths():
    import torch
    from stencilfft_b200 import abi
    pl = _plan(2, 64, 4, 2, "c128")
    L = abi.lib()
    a = torch.empty(64 * 64 + 2, dtype=torch.complex128, device="cuda")
    b_ = torch.empty(64 * 64, dtype=torch.complex128, device="cuda")
    mis = ctypes.c_void_p(a.data_ptr() + 8)
    assert L.zm_fft_forward(pl.handle, mis, b_.data_ptr(), None, None) == abi.ZM_ERR_MISALIGNED
    assert L.zm_fft_forward(pl.handle, b_.data_ptr(), b_.data_ptr(), None, None) == abi.ZM_ERR_INVALID_ARG
    assert L.zm_laplace(pl.handle, b_.data_ptr(), b_.data_ptr(), 1.0, None) == abi.ZM_ERR_INVALID_ARG
    assert L.zm_fft_forward(pl.handle, None, b_.data_ptr(), None, None) == abi.ZM_ERR_INVALID_ARG
    p3 = _plan(3, 16, 2, 2, "c128")
    c = torch.empty(16 ** 3, dtype=torch.complex128, device="cuda")
    e = torch.empty_like(c)
    assert L.zm_dx(p3.handle, c.data_ptr(), e.data_ptr(), 1.0, None) == abi.ZM_ERR_UNSUPPORTED
    # the context is still healthy
    torch.cuda.synchronize()


def test_launch_counter_advances():
    import torch
    from stencilfft_b200 import launch_count
    pl = _plan(2, 64, 4, 2, "c128")
    d = pl.empty()
    d.zero_()
    o = torch.empty_like(d)
    before = launch_count()
    pl.forward_fft(d, o)
    pl.laplace(d, o)
    assert launch_count() - before == 3


@pytest.mark.parametrize("dt", ["c64", "c128"])
def test_autotune_keeps_results(dt):
    """zm_plan_autotune: picks a listed variant, leaves a = IFFT(FFT(a)) / N^2, and the
    tuned plan still matches the oracle."""
    import torch
    n, b, p = 4096, 32, 4
    pl = _plan(2, n, b, p, dt)
    assert pl.kernel_variants >= 2
    x = O.natural_to_real_layout(rand_field(2, n, 7), b, p)
    a = to_dev(x, dt)
    bb, w = torch.empty_like(a), torch.empty_like(a)
    v, ms = pl.autotune(a, bb, work=w, reps=2)
    assert 0 <= v < pl.kernel_variants and ms > 0
    # a went through (reps + 1) round trips per variant: rounding accumulates in c64
    tol = 1e-12 if dt == "c128" else 5e-6
    assert relerr(to_host(a), x) < tol
    a = to_dev(x, dt)
    pl.forward_fft(a, bb, work=w)
    assert relerr(to_host(bb), O.forward_fft(x, 2, n, b, p)) < TOL[dt]


@pytest.mark.parametrize("dt", ["c64", "c128"])
def test_calls_capture_in_cuda_graph(dt):
    """No call allocates or synchronises: forward -> spectral op -> inverse -> Laplacian
    captured in a CUDA graph and replayed gives the eager results bit for bit."""
    import torch
    from stencilfft_b200 import abi, launch_count
    n, b, p = 1024, 32, 4
    pl = _plan(2, n, b, p, dt)
    u = pl.empty()
    pl.fill(u, abi.ZM_FIELD_GAUSSIAN, 21)
    spec, back, lap, work = pl.empty(), pl.empty(), pl.empty(), pl.empty()

    def chain():
        pl.forward_fft(u, spec, work=work)
        pl.spectral_apply(spec, abi.ZM_SPECTRAL_GAUSSIAN, n / 16)
        pl.inverse_fft(spec, back, scale=1.0 / n ** 2, work=work)
        pl.laplace(back, lap)

    chain()
    torch.cuda.synchronize()
    eager = lap.clone()
    lap.zero_()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        chain()
    l0 = launch_count()
    graph.replay()
    torch.cuda.synchronize()
    assert launch_count() == l0
    assert torch.equal(lap, eager)
    assert pl.device_status() == 0
    del graph


def test_autotune_b_picks_a_valid_layout():
    """zm_autotune_b: the chosen B satisfies the layout constraints and a plan with it
    transforms correctly."""
    from stencilfft_b200 import Plan, autotune_b
    n, p = 1024, 2
    b, v, ms = autotune_b(2, n, p, "c64", reps=1)
    L = n // p
    assert b >= 1 and L % b == 0 and (L // b) % p == 0 and ms > 0
    pl = Plan(2, n, b, p, dtype="c64")
    assert 0 <= v < max(1, pl.kernel_variants)
    x = O.natural_to_real_layout(rand_field(2, n, 8), b, p)
    out = pl.empty()
    pl.forward_fft(to_dev(x, "c64"), out, work=pl.empty())
    assert relerr(to_host(out), O.forward_fft(x, 2, n, b, p)) < TOL["c64"]


def test_error_paths_fused_stencils_and_workspace():
    """Argument checks of zm_laplace_dx_dy and of the workspace of the out-of-place
    forward configuration; the context stays usable."""
    import torch
    from stencilfft_b200 import ZmError, abi
    pl = _plan(2, 256, 16, 4, "c64")
    a, b_, c, d = pl.empty(), pl.empty(), pl.empty(), pl.empty()
    pl.fill(a, abi.ZM_FIELD_GAUSSIAN, 1)
    with pytest.raises(ZmError):
        pl.laplace_dx_dy(a, b_, b_, c)                 # outputs overlap
    with pytest.raises(ZmError):
        pl.laplace_dx_dy(a, a, c, d)                   # in overlaps an output
    with pytest.raises(ZmError):
        pl.laplace_dx_dy(a, b_, c, d, delta=0.0)
    p3 = _plan(3, 16, 2, 2, "c64")
    x = p3.empty()
    with pytest.raises(ZmError):
        p3.laplace_dx_dy(x, p3.empty(), p3.empty(), p3.empty())
    big = _plan(2, 16384, 64, 4, "c64")                # has the out-of-place forward configuration
    L = abi.lib()
    u = big.empty()
    o = big.empty()
    # a workspace that overlaps the output is rejected before any launch
    assert L.zm_fft_forward(big.handle, u.data_ptr(), o.data_ptr(), o.data_ptr(), None) == abi.ZM_ERR_INVALID_ARG
    del u, o
    torch.cuda.synchronize()


@pytest.mark.parametrize("dim,n,b,p,dt", [(2, 1024, 32, 2, "c128"), (2, 16384, 64, 4, "c64"),
                                          (3, 64, 4, 4, "c64")])
def test_own_workspace_plan(dim, n, b, p, dt):
    """ZM_FLAG_OWN_WORKSPACE (the compat header's default): work=None uses the plan's own
    workspace, so the input is preserved and the results are bit-identical to passing a
    workspace; at the headline size the call is as fast as with a caller workspace."""
    import torch
    from stencilfft_b200 import Plan, abi
    pl = Plan(dim, n, b, p, dtype=dt)
    po = Plan(dim, n, b, p, dtype=dt, own_workspace=True)
    u = pl.empty()
    pl.fill(u, abi.ZM_FIELD_GAUSSIAN, 4)
    keep = u.clone()
    s1, s2, w = pl.empty(), pl.empty(), pl.empty()
    pl.forward_fft(u, s1, work=w)
    po.forward_fft(u, s2)
    assert torch.equal(s1, s2) and torch.equal(u, keep)
    b1, b2 = pl.empty(), pl.empty()
    pl.inverse_fft(s1, b1, scale=1.0 / n ** dim, work=w)
    po.inverse_fft(s2, b2, scale=1.0 / n ** dim)
    assert torch.equal(b1, b2) and torch.equal(s1, s2)
    if n == 16384:
        def t(fn, reps=10):
            fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps
        ms_work = t(lambda: pl.forward_fft(u, s1, work=w))
        ms_own = t(lambda: po.forward_fft(u, s2))
        print(f"\nforward N=16384 c64: caller workspace {ms_work:.3f} ms, plan workspace {ms_own:.3f} ms")
        assert ms_own < 1.1 * ms_work
