"""GPU parity tests: the CUDA path through the C ABI against the oracle.

Bars (the reference's own contract): layout / permutation outputs bit-exact;
transforms and stencils within relative L2 1e-12 (complex128) / 1e-6 (complex64)
of the oracle; the FP64 2D Laplacian and dx / dy bit-exact (same accumulation order).
"""
import numpy as np
import pytest

import oracle as O
from helpers import TOL, ramp_spectrum, rand_field, relerr, to_dev, to_host

pytestmark = pytest.mark.gpu

# run.sh / run3d.sh sweep corners + small benchmark-shaped layouts
CFG_2D = [(2, 64, 1, 2), (2, 64, 2, 2), (2, 64, 4, 2), (2, 64, 16, 2), (2, 64, 1, 4), (2, 64, 4, 4),
          (2, 128, 8, 4), (2, 256, 8, 2), (2, 256, 16, 4), (2, 512, 16, 2), (2, 1024, 32, 2),
          (2, 1024, 64, 4), (2, 512, 32, 4), (2, 2048, 32, 2), (2, 4096, 64, 4), (2, 4096, 32, 4)]
CFG_3D = [(3, 16, 2, 2), (3, 16, 4, 2), (3, 32, 2, 4), (3, 32, 4, 2), (3, 64, 4, 4)]


def _plan(dim, n, b, p, dt, **kw):
    from stencilfft_b200 import Plan
    return Plan(dim, n, b, p, dtype=dt, **kw)


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("dim,n,b,p", CFG_2D + CFG_3D)
def test_forward_inverse_match_oracle(dim, n, b, p, dt):
    import torch
    x = rand_field(dim, n, seed=n * 7 + b + p)
    buf = O.natural_to_real_layout(x, b, p)
    ref = O.forward_fft(buf, dim, n, b, p)
    pl = _plan(dim, n, b, p, dt)
    d_in = to_dev(buf, dt)
    d_out = torch.empty_like(d_in)
    work = torch.empty_like(d_in)
    pl.forward_fft(d_in, d_out, work=work)
    got = to_host(d_out)
    assert relerr(got, ref) < TOL[dt], relerr(got, ref)
    # input preserved when a workspace is given
    assert np.array_equal(to_host(d_in), buf.astype(np.complex64 if dt == "c64" else np.complex128))
    back = torch.empty_like(d_in)
    pl.inverse_fft(d_out, back, scale=1.0 / n ** dim, work=work)
    ref_back = O.inverse_fft(ref, dim, n, b, p, scale=1.0 / n ** dim)
    assert relerr(to_host(back), ref_back) < TOL[dt]
    assert relerr(to_host(back), buf) < TOL[dt]


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("dim,n,b,p", [(2, 4096, 32, 4), (2, 4096, 64, 4), (2, 1024, 32, 2)])
def test_every_kernel_variant_matches_oracle(dim, n, b, p, dt):
    """Each tile shape of the fused pass (cluster size, lines per tile) gives the same transform."""
    import torch
    x = rand_field(dim, n, seed=17)
    buf = O.natural_to_real_layout(x, b, p)
    ref = O.forward_fft(buf, dim, n, b, p)
    pl = _plan(dim, n, b, p, dt)
    assert pl.kernel_variants >= 1
    d_in = to_dev(buf, dt)
    d_out, work, back = torch.empty_like(d_in), torch.empty_like(d_in), torch.empty_like(d_in)
    for v in range(pl.kernel_variants):
        pl.set_kernel_variant(v)
        pl.forward_fft(d_in, d_out, work=work)
        assert relerr(to_host(d_out), ref) < TOL[dt], v
        pl.inverse_fft(d_out, back, scale=1.0 / n ** dim, work=work)
        assert relerr(to_host(back), buf) < TOL[dt], v


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("dim,n,b,p", [(2, 64, 4, 2), (2, 128, 8, 4), (2, 1024, 32, 2), (2, 4096, 64, 4),
                                       (3, 16, 2, 2), (3, 32, 2, 4), (3, 64, 4, 4)])
def test_reference_ramp_fixture_known_answer(dim, n, b, p, dt):
    """The reference's init_host fixture (x = global linear index, zmodel/utils.cu), which
    the oracle reproduces bit-exactly, through the CUDA forward transform against its
    closed-form spectrum, and back through the inverse."""
    import torch
    buf = O.init_ramp(dim, n, b, p)
    want = O.natural_to_reciprocal_layout(ramp_spectrum(dim, n), b, p)
    pl = _plan(dim, n, b, p, dt)
    d_in = to_dev(buf, dt)
    d_out, work, back = torch.empty_like(d_in), torch.empty_like(d_in), torch.empty_like(d_in)
    pl.forward_fft(d_in, d_out, work=work)
    assert relerr(to_host(d_out), want) < TOL[dt], relerr(to_host(d_out), want)
    pl.inverse_fft(d_out, back, scale=1.0 / n ** dim, work=work)
    assert relerr(to_host(back), buf) < TOL[dt]


@pytest.mark.parametrize("dim,n,b,p", CFG_2D[:6] + CFG_3D[:3])
def test_reference_contract_buf0_clobbered(dim, n, b, p):
    """work=None: buf0 may be used as scratch (fft.cu:189-198); results unchanged."""
    import torch
    x = rand_field(dim, n, seed=3)
    buf = O.natural_to_real_layout(x, b, p)
    pl = _plan(dim, n, b, p, "c128")
    d0 = to_dev(buf, "c128")
    d1 = torch.empty_like(d0)
    pl.forward_fft(d0, d1)
    ref = O.forward_fft(buf, dim, n, b, p)
    assert relerr(to_host(d1), ref) < 1e-12
    d2 = torch.empty_like(d0)
    pl.inverse_fft(d1, d2, scale=complex(0.5, 0.25))
    assert relerr(to_host(d2), O.inverse_fft(ref, dim, n, b, p, scale=complex(0.5, 0.25))) < 1e-12


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("dim,n,b,p", CFG_2D + CFG_3D)
def test_permutation_only_bit_exact(dim, n, b, p, dt):
    """do_compute=false pipelines: pure data movement, bit-identical to the reference chain."""
    import torch
    ramp = (np.arange(n ** dim, dtype=np.float64) % 4093) + 1j * (np.arange(n ** dim) % 7)
    pl = _plan(dim, n, b, p, dt, permute_only=True)
    d0 = to_dev(ramp, dt)
    d1 = torch.empty_like(d0)
    work = torch.empty_like(d0)
    pl.forward_fft(d0, d1, work=work)
    ref = O.forward_fft(ramp, dim, n, b, p, do_compute=False)
    assert np.array_equal(to_host(d1), ref)
    d2 = torch.empty_like(d0)
    pl.inverse_fft(d1, d2, scale=0.5, work=work)
    assert np.array_equal(to_host(d2), ramp)


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("dim,n,b,p", CFG_2D + CFG_3D)
def test_laplace_matches_oracle(dim, n, b, p, dt):
    import torch
    x = rand_field(dim, n, seed=5)
    buf = O.natural_to_real_layout(x, b, p)
    ref = O.laplace(buf, dim, n, b, p)
    pl = _plan(dim, n, b, p, dt)
    d0 = to_dev(buf, dt)
    d1 = torch.empty_like(d0)
    pl.laplace(d0, d1, inv_h2=1.0)
    got = to_host(d1)
    if dt == "c128" and dim == 2:
        assert np.array_equal(got, ref)          # same accumulation order, exact 4*c
    else:
        assert relerr(got, ref) < TOL[dt]
    # h = 1/N scaling
    pl.laplace(d0, d1, inv_h2=float(n * n))
    assert relerr(to_host(d1), ref * n * n) < TOL[dt]


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("n,b,p", [(128, 8, 2), (256, 16, 2), (256, 4, 4), (256, 64, 2)])
def test_laplace3d_long_lines_match_oracle(n, b, p, dt):
    """Lines of 64 (complex64) / 128 (complex128) vectors take the several-vectors-per-
    thread 3D kernel: every block-boundary and wrap case of x, y and z at a local side of
    128 (N = 256, P = 2); the side-64 cases keep the one-vector kernel."""
    import torch
    x = rand_field(3, n, seed=11)
    buf = O.natural_to_real_layout(x, b, p)
    ref = O.laplace(buf, 3, n, b, p)
    pl = _plan(3, n, b, p, dt)
    d0 = to_dev(buf, dt)
    d1 = torch.empty_like(d0)
    pl.laplace(d0, d1, inv_h2=float(n * n))
    assert relerr(to_host(d1), ref * n * n) < TOL[dt]


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("dim,n,b,p", [c for c in CFG_2D if c[2] >= 2])
def test_dx_dy_match_oracle(dim, n, b, p, dt):
    import torch
    x = rand_field(2, n, seed=9)
    buf = O.natural_to_real_layout(x, b, p)
    pl = _plan(2, n, b, p, dt)
    d0 = to_dev(buf, dt)
    d1 = torch.empty_like(d0)
    h = 1.0 / n
    for fn, orf in ((pl.dx, O.dx), (pl.dy, O.dy)):
        fn(d0, d1, delta=h)
        ref = orf(buf, n, b, p, h)
        got = to_host(d1)
        if dt == "c128":
            assert np.array_equal(got, ref)
        else:
            assert relerr(got, ref) < TOL[dt]
    # real Scalar form (dx.cu / dy.cu operate on double)
    rreal = np.ascontiguousarray(buf.real)
    dr = torch.from_numpy(rreal.astype(np.float64 if dt == "c128" else np.float32)).cuda()
    do = torch.empty_like(dr)
    pl.dx(dr, do, delta=h)
    refr = O.dx(rreal, n, b, p, h)
    if dt == "c128":
        assert np.array_equal(do.cpu().numpy(), refr)
    else:
        assert relerr(do.cpu().numpy().astype(np.float64), refr) < TOL[dt]


def test_dx_dy_accept_b1_as_extension():
    """B = 1 is outside the reference's dx/dy (dx.cu:100); here it is the same global stencil."""
    import torch
    n, b, p = 64, 1, 2
    x = rand_field(2, n, seed=2)
    buf = O.natural_to_real_layout(x, b, p)
    pl = _plan(2, n, b, p, "c128")
    d0 = to_dev(buf, "c128")
    d1 = torch.empty_like(d0)
    pl.dx(d0, d1, delta=1.0)
    gx = O.real_layout_to_natural(to_host(d1), 2, n, b, p)
    rx = (np.roll(x, 2, 1) - 8 * np.roll(x, 1, 1) + 8 * np.roll(x, -1, 1) - np.roll(x, -2, 1)) / 12
    assert relerr(gx, rx) < 1e-14


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("n,b,p", [(64, 4, 2), (64, 1, 2), (256, 16, 4), (1024, 32, 2), (512, 8, 4)])
def test_laplace_dx_dy_fused_bit_identical(n, b, p, dt):
    """zm_laplace_dx_dy: each output bit-identical to its own stencil call."""
    import torch
    from stencilfft_b200 import abi
    pl = _plan(2, n, b, p, dt)
    u = pl.empty()
    pl.fill(u, abi.ZM_FIELD_GAUSSIAN, 5)
    lap, gx, gy = pl.empty(), pl.empty(), pl.empty()
    pl.laplace_dx_dy(u, lap, gx, gy, inv_h2=float(n * n), delta=1.0 / n)
    ref = pl.empty()
    pl.laplace(u, ref, inv_h2=float(n * n))
    assert torch.equal(lap, ref)
    pl.dx(u, ref, delta=1.0 / n)
    assert torch.equal(gx, ref)
    pl.dy(u, ref, delta=1.0 / n)
    assert torch.equal(gy, ref)
