"""The library against the reference's OWN GPU pipeline (cuFFT + its hand-written
pack / unpack / repack / stencil kernels, unmodified, one host thread per MPI rank through
the in-process MPI stand-in of oracle/refgpu/), on the same seeded inputs.

Bars: transforms and stencils within relative L2 1e-12 of the reference (complex128, the
reference's only precision) and 1e-6 for the complex64 form; the permutation-only chains
(the reference's do_compute=false, fft.cu:211-213) bit-exact; the 2D Laplacian and the real
dx / dy bit-exact (their products are by powers of two, so contraction cannot change a bit).
The C oracle is pinned to the same reference outputs here.

The runner libraries are built from the reference sources by `make -C oracle ref-gpu`;
where they were not built (no reference checkout at build time) these tests skip.
"""
import numpy as np
import pytest

import oracle as O
from oracle import refgpu as R
from helpers import TOL, rand_field, relerr, to_dev, to_host

pytestmark = pytest.mark.gpu

CFG_2D = [(64, 4, 2), (64, 2, 4), (128, 8, 2), (256, 8, 4), (512, 16, 2), (1024, 32, 2)]
CFG_3D = [(16, 2, 2), (32, 4, 2), (32, 2, 4), (64, 4, 4)]
CASES = [(2,) + c for c in CFG_2D] + [(3,) + c for c in CFG_3D]


def _ref(n, b, p, aware=False):
    if not R.available(n, b, p, aware):
        pytest.skip(f"reference GPU runner for N={n} B={b} P={p} not built")
    return R.RefPipeline(n, b, p, aware)


def _plan(dim, n, b, p, dt, **kw):
    from stencilfft_b200 import Plan
    return Plan(dim, n, b, p, dtype=dt, **kw)


@pytest.mark.parametrize("dim,n,b,p", CASES)
def test_forward_inverse_match_reference_pipeline(dim, n, b, p):
    import torch
    ref = _ref(n, b, p)
    buf = O.natural_to_real_layout(rand_field(dim, n, seed=41 + n + b + p), b, p)
    want, _, _ = ref.fft(buf, dim)
    # the C oracle follows the reference pipeline
    assert relerr(O.forward_fft(buf, dim, n, b, p), want) < 1e-12
    s = 1.0 / n ** dim
    want_back, _, _ = ref.fft(want, dim, inverse=True, scale=s)
    assert relerr(want_back, buf) < 1e-12
    for dt in ("c128", "c64"):
        pl = _plan(dim, n, b, p, dt)
        d_in = to_dev(buf, dt)
        d_out, work, back = torch.empty_like(d_in), torch.empty_like(d_in), torch.empty_like(d_in)
        pl.forward_fft(d_in, d_out, work=work)
        assert relerr(to_host(d_out), want) < TOL[dt], (dt, relerr(to_host(d_out), want))
        pl.inverse_fft(to_dev(want, dt), back, scale=s, work=work)
        assert relerr(to_host(back), want_back) < TOL[dt]


@pytest.mark.parametrize("dim,n,b,p", CASES)
def test_permutation_only_bit_exact_vs_reference_pipeline(dim, n, b, p):
    """do_compute=false: the reference's pure data movement (placeholder copies for the
    FFTs, unit twiddles); the library's permutation-only plans move the same bits."""
    import torch
    ref = _ref(n, b, p)
    ramp = (np.arange(n ** dim, dtype=np.float64) % 4093) + 1j * (np.arange(n ** dim) % 7)
    want, _, _ = ref.fft(ramp, dim, do_compute=False)
    assert np.array_equal(O.forward_fft(ramp, dim, n, b, p, do_compute=False), want)
    want_back, _, _ = ref.fft(want, dim, inverse=True, do_compute=False)
    assert np.array_equal(want_back, ramp)
    pl = _plan(dim, n, b, p, "c128", permute_only=True)
    d0 = to_dev(ramp, "c128")
    d1, work = torch.empty_like(d0), torch.empty_like(d0)
    pl.forward_fft(d0, d1, work=work)
    assert np.array_equal(to_host(d1), want)


@pytest.mark.parametrize("dim,n,b,p", CASES)
def test_laplace_matches_reference_pipeline(dim, n, b, p):
    import torch
    ref = _ref(n, b, p)
    buf = O.natural_to_real_layout(rand_field(dim, n, seed=7 * n + b), b, p)
    want, _, _ = ref.laplace(buf, dim)
    got_oracle = O.laplace(buf, dim, n, b, p)
    pl = _plan(dim, n, b, p, "c128")
    d0 = to_dev(buf, "c128")
    d1 = torch.empty_like(d0)
    pl.laplace(d0, d1, inv_h2=1.0)
    got = to_host(d1)
    if dim == 2:
        assert np.array_equal(got_oracle, want)
        assert np.array_equal(got, want)
    else:
        # -6 * centre is not exact: the reference (nvcc, contraction on) and the oracle
        # (contraction off) may differ in the last bit
        assert relerr(got_oracle, want) < 1e-15
        assert relerr(got, want) < 1e-15
    pl64 = _plan(dim, n, b, p, "c64")
    d0 = to_dev(buf, "c64")
    d1 = torch.empty_like(d0)
    pl64.laplace(d0, d1, inv_h2=1.0)
    assert relerr(to_host(d1), want) < TOL["c64"]


@pytest.mark.parametrize("n,b,p", [c for c in CFG_2D if c[1] >= 2])
def test_dx_dy_bit_exact_vs_reference_pipeline(n, b, p):
    """The reference's real dx / dy kernels (dx.cu:10-82, dy.cu:10-103) with every rank's
    halos packed by its own host pack functions from the neighbours' data."""
    import torch
    ref = _ref(n, b, p)
    rng = np.random.default_rng(n + b + p)
    x = O.natural_to_real_layout(rng.standard_normal((n, n)), b, p).real.copy()
    pl = _plan(2, n, b, p, "c128")
    d0 = torch.from_numpy(x).cuda()
    d1 = torch.empty_like(d0)
    delta = 1.0 / n
    for fn, rf, orf in ((pl.dx, ref.dx, O.dx), (pl.dy, ref.dy, O.dy)):
        want = rf(x, delta)
        assert np.array_equal(orf(x, n, b, p, delta), want)
        fn(d0, d1, delta=delta)
        assert np.array_equal(d1.cpu().numpy(), want)


def test_c1_stated_field_against_reference_and_oracle():
    """Config 1: complex128 N=1024, P=2, B=32, Re and Im U[-1,1) from seed 0 (the
    counter-based generator shared by host and device): forward, inverse round trip and
    the periodic 5-point Laplacian with h = 1/N, against the reference pipeline, the C
    oracle and FP64 pocketfft."""
    import torch
    n, b, p = 1024, 32, 2
    ref = _ref(n, b, p)
    nat = O.uniform_field(0, n * n).reshape(n, n)
    buf = O.natural_to_real_layout(nat, b, p)
    pl = _plan(2, n, b, p, "c128")
    d_in = torch.empty(n * n, dtype=torch.complex128, device="cuda")
    from stencilfft_b200 import abi
    pl.fill(d_in, abi.ZM_FIELD_UNIFORM, 0)
    assert np.array_equal(to_host(d_in), buf)          # device generator == host generator
    want, _, _ = ref.fft(buf, 2)
    spec = O.natural_to_reciprocal_layout(np.fft.fft2(nat), b, p)
    assert relerr(want, spec) < 1e-12
    d_out, work, back = torch.empty_like(d_in), torch.empty_like(d_in), torch.empty_like(d_in)
    pl.forward_fft(d_in, d_out, work=work)
    assert relerr(to_host(d_out), want) < 1e-12
    assert relerr(to_host(d_out), spec) < 1e-12
    assert relerr(O.forward_fft(buf, 2, n, b, p), want) < 1e-12
    want_back, _, _ = ref.fft(want, 2, inverse=True, scale=1.0 / (n * n))
    pl.inverse_fft(d_out, back, scale=1.0 / (n * n), work=work)
    assert relerr(to_host(back), want_back) < 1e-12
    assert relerr(to_host(back), buf) < 1e-12
    # Laplacian with h = 1/N: the reference has no 1/h^2 factor, so scale its output
    lap_ref, _, _ = ref.laplace(buf, 2)
    d_lap = torch.empty_like(d_in)
    pl.laplace(d_in, d_lap, inv_h2=float(n * n))
    assert relerr(to_host(d_lap), lap_ref * float(n * n)) < 1e-12
    pl.laplace(d_in, d_lap, inv_h2=1.0)
    assert np.array_equal(to_host(d_lap), lap_ref)
    nat_lap = (np.roll(nat, 1, 0) + np.roll(nat, -1, 0) + np.roll(nat, 1, 1) + np.roll(nat, -1, 1)
               - 4 * nat)
    assert relerr(O.real_layout_to_natural(lap_ref, 2, n, b, p), nat_lap) < 1e-14


TIMING = [(2, 1024, 32, 2), (2, 4096, 32, 4), (3, 256, 16, 4)]


@pytest.mark.parametrize("dim,n,b,p", TIMING)
def test_reference_pipeline_timing(dim, n, b, p):
    """The GPU-vs-GPU bar: the reference's own pipeline (cuFFT + its kernels, all virtual
    ranks on this GPU, host-staged exchanges as it ships and, where built, the
    __GPU__AWARE__MPI__ form) against the library on the same field.  Reference times are
    barrier to barrier per call (its TOTAL timer, fft.cu:202-338); the library's are CUDA
    events over 10 calls.  Prints one JSON line per configuration; the parity of the two
    outputs is asserted."""
    import json
    import torch
    from stencilfft_b200 import Plan, abi
    ref = _ref(n, b, p)
    pl128 = Plan(dim, n, b, p, dtype="c128")
    u = pl128.empty()
    pl128.fill(u, abi.ZM_FIELD_GAUSSIAN, 2)
    buf = to_host(u)
    row = {"dim": dim, "n": n, "b": b, "p": p, "ranks": p ** dim}
    for aware in (False, True):
        if not R.available(n, b, p, aware):
            continue
        r = R.RefPipeline(n, b, p, aware)
        tag = "ref_aware" if aware else "ref_staged"
        spec, ms_f, log = r.fft(buf, dim, reps=2)
        _, ms_i, _ = r.fft(spec, dim, inverse=True, scale=1.0 / n ** dim, reps=2)
        lap, ms_l, _ = r.laplace(buf, dim, reps=2)
        row[tag] = {"fwd_ms": round(ms_f, 3), "inv_ms": round(ms_i, 3), "laplace_ms": round(ms_l, 3),
                    "stages_ns": {k: v[-1] for k, v in R.stage_times(log).items()}}
    for dt in ("c128", "c64"):
        pl = pl128 if dt == "c128" else Plan(dim, n, b, p, dtype=dt)
        x = u if dt == "c128" else u.to(torch.complex64)
        y, w, z = pl.empty(), pl.empty(), pl.empty()

        def t(fn, reps=10):
            fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps
        ms_f = t(lambda: pl.forward_fft(x, y, work=w))
        ms_i = t(lambda: pl.inverse_fft(y, z, scale=1.0 / n ** dim, work=w))
        ms_l = t(lambda: pl.laplace(x, z, inv_h2=1.0))
        row[dt] = {"fwd_ms": round(ms_f, 4), "inv_ms": round(ms_i, 4), "laplace_ms": round(ms_l, 4)}
        if dt == "c128":
            pl.forward_fft(x, y, work=w)
            assert relerr(to_host(y), spec) < 1e-12
            pl.laplace(x, z, inv_h2=1.0)
            assert relerr(to_host(z), lap) < 1e-15
    print("\nREFTIMING " + json.dumps(row))
