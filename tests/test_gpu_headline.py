"""The headline layout (2D N=16384, P=4, B=64 -- the bench's workload) pinned to FP64 on
generic fields, for the complex64 compensated and the complex128 forms.

Reference values, computed on the device in FP64 from the natural-layout field (the
library's natural <-> interleaved converters are bit-exact permutations, tested against
the reference's own index maps elsewhere):
* the full spectrum of cuFFT's complex128 2D transform (`torch.fft.fft2`; the reference's
  own FFT arithmetic is cuFFT Z2Z);
* an exact DFT of 64 x 64 randomly chosen coefficients, as two dense FP64 sums (a row
  sum then a column sum) with twiddle angles reduced exactly in integers -- no FFT
  library involved.  Its error estimate of the full-spectrum relative L2 is
  sqrt(N^2 / S * sum |err|^2) / ||X||, with ||X||^2 = N^2 ||x||^2 (Parseval);
* the 5-point Laplacian and 4th-order dx / dy (h = 1/N) as `torch.roll` sums.
Fields: the bench's 32 seeded Fourier modes (|k| <= N/8) plus 1e-3 noise, and a
Gaussian N(0,1) field.  Bars: relative L2 1e-12 (complex128) and 1e-6 (complex64).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, B, P = 16384, 64, 4


def _norm(t):
    import torch
    return float(torch.linalg.vector_norm(t.to(torch.complex128)))


def _field(pl, kind):
    from stencilfft_b200 import abi
    import bench
    u = pl.empty()
    if kind == "modes":
        modes, amps = bench.modes_and_amps(N)
        pl.fill_modes(u, modes, amps, bench.NOISE, bench.NOISE_SEED)
    else:
        pl.fill(u, abi.ZM_FIELD_GAUSSIAN, 9)
    return u


def _exact_dft_sample(nat2d, k1, k2):
    """X[k1_i, k2_j] = sum_y sum_x u[y, x] w^(k1_i y + k2_j x), w = exp(-2 pi i / N), FP64."""
    import torch
    dev = nat2d.device
    n = torch.arange(N, dtype=torch.int64, device=dev)
    ang2 = ((n[:, None] * k2[None, :]) % N).to(torch.float64) * (-2.0 * np.pi / N)
    W2 = torch.polar(torch.ones_like(ang2), ang2)                   # (N, S2)
    Y = nat2d @ W2                                                  # sum over x
    ang1 = ((k1[:, None] * n[None, :]) % N).to(torch.float64) * (-2.0 * np.pi / N)
    W1 = torch.polar(torch.ones_like(ang1), ang1)                   # (S1, N)
    return W1 @ Y                                                   # sum over y


@pytest.mark.parametrize("kind", ["modes", "gauss"])
def test_headline_transforms_against_fp64(kind):
    import torch
    from stencilfft_b200 import Plan
    p128, p64 = Plan(2, N, B, P, dtype="c128"), Plan(2, N, B, P, dtype="c64")
    u = _field(p128, kind)
    nat = p128.empty()
    p128.real_to_natural(u, nat)
    X = torch.fft.fft2(nat.view(N, N)).reshape(-1)                  # FP64 cuFFT spectrum
    xnorm = _norm(u)
    Xnorm = N * xnorm                                              # Parseval

    # exact DFT of 64 x 64 random coefficients pins the cuFFT spectrum too
    rng = np.random.default_rng(2024)
    k1 = torch.from_numpy(rng.choice(N, 64, replace=False)).cuda()
    k2 = torch.from_numpy(rng.choice(N, 64, replace=False)).cuda()
    Z = _exact_dft_sample(nat.view(N, N), k1, k2)
    S = Z.numel()

    def sample_err(spec_nat):
        got = spec_nat.view(N, N)[k1][:, k2].to(torch.complex128)
        return float(np.sqrt(N * N / S) * _norm(got - Z)) / Xnorm

    assert sample_err(X) < 1e-12

    spec, work = p128.empty(), p128.empty()
    p128.forward_fft(u, spec, work=work)
    got = p128.empty()
    p128.reciprocal_to_natural(spec, got)
    e128 = _norm(got - X) / _norm(X)
    assert e128 < 1e-12, e128
    assert sample_err(got) < 1e-12
    del got

    # complex128 inverse of the FP64 spectrum returns the field (pins the inverse's
    # own permutation, not just its mirror image of the forward)
    Xr = p128.empty()
    p128.natural_to_reciprocal(X, Xr)
    back = p128.empty()
    p128.inverse_fft(Xr, back, scale=1.0 / (N * N), work=work)
    assert _norm(back - u) / xnorm < 1e-12
    del back, work

    # complex64 compensated form
    u64 = u.to(torch.complex64)
    s64, w64 = p64.empty(), p64.empty()
    p64.forward_fft(u64, s64, work=w64)
    e64_vs_c128 = _norm(s64.to(torch.complex128) - spec) / _norm(spec)
    assert e64_vs_c128 < 1e-6, e64_vs_c128
    g64 = p64.empty()
    p64.reciprocal_to_natural(s64, g64)
    e64 = _norm(g64.to(torch.complex128) - X) / _norm(X)
    assert e64 < 1e-6, e64
    assert sample_err(g64) < 1e-6
    del g64, spec
    b64 = p64.empty()
    p64.inverse_fft(Xr.to(torch.complex64), b64, scale=1.0 / (N * N), work=w64)
    assert _norm(b64.to(torch.complex128) - u) / xnorm < 1e-6
    print(f"\nN={N} {kind}: c128 fwd rel-L2 vs FP64 {e128:.2e}; c64 fwd {e64:.2e} (vs c128 {e64_vs_c128:.2e})")


def _roll_stencils(f, h):
    import torch
    r = torch.roll
    lap = (r(f, 1, 0) + r(f, -1, 0) + r(f, 1, 1) + r(f, -1, 1) - 4 * f) / (h * h)
    dx = (r(f, 2, 1) - 8 * r(f, 1, 1) + 8 * r(f, -1, 1) - r(f, -2, 1)) / (12 * h)
    dy = (r(f, 2, 0) - 8 * r(f, 1, 0) + 8 * r(f, -1, 0) - r(f, -2, 0)) / (12 * h)
    return lap, dx, dy


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_headline_stencils_against_roll(dt):
    """Laplacian, dx, dy (separately and in the fused launch) at N=16384 against FP64 rolls."""
    import torch
    from stencilfft_b200 import Plan
    p128 = Plan(2, N, B, P, dtype="c128")
    u128 = _field(p128, "gauss")
    nat = p128.empty()
    p128.real_to_natural(u128, nat)
    h = 1.0 / N
    want = _roll_stencils(nat.view(N, N), h)
    del nat
    pl = p128 if dt == "c128" else Plan(2, N, B, P, dtype="c64")
    u = u128 if dt == "c128" else u128.to(torch.complex64)
    del u128
    tol = 1e-12 if dt == "c128" else 1e-6
    out, natout = pl.empty(), pl.empty()
    for fn, w in ((lambda a, o: pl.laplace(a, o, inv_h2=1.0 / (h * h)), want[0]),
                  (lambda a, o: pl.dx(a, o, delta=h), want[1]),
                  (lambda a, o: pl.dy(a, o, delta=h), want[2])):
        fn(u, out)
        pl.real_to_natural(out, natout)
        err = _norm(natout.view(N, N) - w) / _norm(w)
        assert err < tol, err
    lap, gx, gy = pl.empty(), pl.empty(), pl.empty()
    pl.laplace_dx_dy(u, lap, gx, gy, inv_h2=1.0 / (h * h), delta=h)
    for o, w in ((lap, want[0]), (gx, want[1]), (gy, want[2])):
        pl.real_to_natural(o, natout)
        assert _norm(natout.view(N, N) - w) / _norm(w) < tol


def test_headline_c128_every_tile_variant():
    """Every complex128 tile shape of the 2^14-point lines (clusters of two / four, one or
    two lines per tile, and their persistent forms staging the next tile in tensor memory)
    gives the default configuration's spectrum, in place (no workspace), and returns the
    field."""
    import torch
    from stencilfft_b200 import Plan
    pl = Plan(2, N, B, P, dtype="c128")
    u = _field(pl, "gauss")
    a, want, got = pl.empty(), pl.empty(), pl.empty()
    work = pl.empty()
    pl.forward_fft(u, want, work=work)            # default: out of place
    del work
    for v in range(pl.kernel_variants):
        pl.set_kernel_variant(v)
        a.copy_(u)
        pl.forward_fft(a, got)                    # in place on the variant's tiles
        assert _norm(got - want) / _norm(want) < 1e-14, v
        a.copy_(got)
        pl.inverse_fft(a, got, scale=1.0 / (N * N))
        assert _norm(got - u) / _norm(u) < 1e-12, v
        assert pl.device_status() == 0
