"""CPU tests of the oracle itself (no GPU).

The oracle is pinned three ways before any CUDA result is compared with it:
  * bit-exactly against the reference's own zmodel/utils.h index maps and the
    zmodel/utils.cu ramp fixture, compiled on the host into oracle/_ref;
  * against an independent FP64 FFT (numpy pocketfft) through those maps;
  * against the closed-form spectrum of the reference's ramp fixture (KAT).
"""
import numpy as np
import pytest

import oracle as O
from helpers import ramp_spectrum

# (dim, N, B, P): corners of the reference's run.sh / run3d.sh sweep plus small
# versions of the benchmark layouts.
GRID_2D = [(2, 64, 1, 2), (2, 64, 2, 2), (2, 64, 4, 2), (2, 64, 8, 2), (2, 64, 16, 2),
           (2, 64, 1, 4), (2, 64, 2, 4), (2, 64, 4, 4), (2, 128, 8, 4), (2, 128, 2, 2),
           (2, 256, 16, 4), (2, 256, 8, 2), (2, 256, 1, 2)]
GRID_3D = [(3, 16, 2, 2), (3, 16, 4, 2), (3, 32, 2, 4), (3, 32, 4, 2)]


def relerr(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rand_field(dim, n, seed=0):
    rng = np.random.default_rng(seed)
    shape = (n,) * dim
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


# ----------------------------------------------------- pin against reference

REF_SMALL = [(n, b, p) for (n, b, p) in
             [(16, 2, 2), (16, 4, 2), (32, 2, 4), (32, 4, 2), (64, 1, 2), (64, 2, 2), (64, 4, 2),
              (64, 8, 2), (64, 16, 2), (64, 1, 4), (64, 2, 4), (64, 4, 4), (128, 2, 2),
              (128, 8, 4), (256, 1, 2), (256, 8, 2), (256, 16, 4), (512, 16, 2), (512, 32, 4),
              (1024, 16, 2), (1024, 32, 2), (2048, 32, 2), (4096, 32, 4)]]


@pytest.mark.parametrize("n,b,p", REF_SMALL)
def test_index_maps_bit_exact_vs_reference_utils(n, b, p):
    ref = O.ref_host_lib(n, b, p)
    if ref is None:
        pytest.skip("reference host code not built (oracle/_ref)")
    d = O.derived(2, n, b, p)
    L = d["L"]
    # 1-D permutations over their whole domains
    for name in ("packed_to_block_cyclic", "block_cyclic_to_packed", "lp", "ct", "lp_inv", "ct_inv"):
        dom = L if name in ("packed_to_block_cyclic", "block_cyclic_to_packed", "lp", "lp_inv") else n
        f = getattr(ref, "zr_" + name)
        ours = [O.index_map(name, n, b, p, i) for i in range(0, dom, max(1, dom // 257))] \
            if name in ("lp", "ct", "lp_inv", "ct_inv") else None
        if ours is not None:
            theirs = [f(i) for i in range(0, dom, max(1, dom // 257))]
            assert ours == theirs, name
    # whole-grid maps (2D always; 3D where the grid is small)
    for dim in (2, 3):
        if n ** dim > (1 << 22):
            continue
        if dim == 3 and (L // b) % p:
            continue
        import ctypes
        mine = O.real_layout_map(dim, n, b, p)
        theirs = np.empty_like(mine)
        ref.zr_real_layout_map(dim, theirs.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(mine, theirs), f"real_to_global dim={dim}"
        mine = O.reciprocal_layout_map(dim, n, b, p)
        ref.zr_reciprocal_layout_map(dim, theirs.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(mine, theirs), f"reciprocal_to_global dim={dim}"


@pytest.mark.parametrize("n,b,p", [(16384, 64, 4), (4096, 32, 4), (2048, 32, 2)])
def test_index_maps_sampled_large(n, b, p):
    """Sampled scalar checks where the whole-grid table would be too large."""
    import ctypes
    ref = O.ref_host_lib(n, b, p)
    if ref is None:
        pytest.skip("reference host code not built (oracle/_ref)")
    rng = np.random.default_rng(1)
    ci = ctypes.c_int
    for _ in range(2000):
        ky, kx = (int(v) for v in rng.integers(0, n, 2))
        out = [ci() for _ in range(4)]
        ref.zr_global_to_reciprocal(ky, kx, *[ctypes.byref(o) for o in out])
        assert O.index_map("global_to_reciprocal", n, b, p, ky, kx) == tuple(o.value for o in out)
        gr, gc = (int(v) for v in rng.integers(0, n, 2))
        ref.zr_global_to_real(gr, gc, *[ctypes.byref(o) for o in out])
        assert O.index_map("global_to_real", n, b, p, gr, gc) == tuple(o.value for o in out)


@pytest.mark.parametrize("dim,n,b,p", [(2, 64, 4, 2), (2, 64, 2, 4), (2, 256, 16, 4),
                                       (2, 1024, 32, 2), (3, 16, 2, 2), (3, 32, 2, 4)])
def test_ramp_fixture_bit_exact_vs_reference_init_host(dim, n, b, p):
    import ctypes
    ref = O.ref_host_lib(n, b, p)
    if ref is None:
        pytest.skip("reference host code not built (oracle/_ref)")
    d = O.derived(dim, n, b, p)
    ours = O.init_ramp(dim, n, b, p)
    per = d["rank_elems"]
    for r in range(d["ranks"]):
        got = np.empty(per, dtype=np.complex128)
        ptr = got.ctypes.data_as(ctypes.c_void_p)
        if dim == 2:
            ref.zr_init_host(r // p, r % p, ptr)
        else:
            ref.zr_init_host_3d((r % (p * p)) // p, r % p, r // (p * p), ptr)
        assert np.array_equal(ours[r * per:(r + 1) * per], got), f"rank {r}"


# --------------------------------------------------------- FP64 FFT oracle

@pytest.mark.parametrize("dim,n,b,p", GRID_2D + GRID_3D)
def test_forward_inverse_vs_pocketfft(dim, n, b, p):
    x = rand_field(dim, n, seed=n + b + p)
    buf = O.natural_to_real_layout(x, b, p)
    out = O.forward_fft(buf, dim, n, b, p)
    X = O.reciprocal_layout_to_natural(out, dim, n, b, p)
    assert relerr(X, np.fft.fftn(x)) < 1e-13
    back = O.inverse_fft(out, dim, n, b, p, scale=1.0 / n ** dim)
    assert relerr(back, buf) < 1e-13


@pytest.mark.parametrize("dim,n,b,p", [(2, 64, 4, 2), (2, 128, 8, 4), (3, 16, 2, 2)])
def test_ramp_known_answer(dim, n, b, p):
    """Closed-form spectrum of the reference fixture x = global linear index."""
    buf = O.init_ramp(dim, n, b, p)
    X = O.reciprocal_layout_to_natural(O.forward_fft(buf, dim, n, b, p), dim, n, b, p)
    exp = ramp_spectrum(dim, n)
    assert relerr(X, exp) < 1e-13


@pytest.mark.parametrize("dim,n,b,p", [(2, 64, 4, 2), (2, 64, 1, 4), (3, 16, 2, 2), (3, 32, 4, 2)])
def test_permutation_only_mode_is_a_bijection(dim, n, b, p):
    """do_compute=false (the reference's __ZMODEL__COMPUTE__ off): pure data movement."""
    ramp = np.arange(n ** dim, dtype=np.float64) + 0j
    out = O.forward_fft(ramp, dim, n, b, p, do_compute=False)
    assert np.array_equal(np.sort(out.real), ramp.real)
    back = O.inverse_fft(out, dim, n, b, p, do_compute=False)
    assert np.array_equal(back, ramp)


# ----------------------------------------------------------------- stencils

@pytest.mark.parametrize("dim,n,b,p", GRID_2D + GRID_3D)
def test_laplace_is_periodic_laplacian(dim, n, b, p):
    x = rand_field(dim, n, seed=7)
    buf = O.natural_to_real_layout(x, b, p)
    got = O.real_layout_to_natural(O.laplace(buf, dim, n, b, p), dim, n, b, p)
    ref = sum(np.roll(x, s, axis=a) for a in range(dim) for s in (1, -1)) - 2 * dim * x
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max() * 10


@pytest.mark.parametrize("dim,n,b,p", [g for g in GRID_2D if g[2] >= 2])
def test_dx_dy_are_fourth_order_central_differences(dim, n, b, p):
    x = rand_field(2, n, seed=11)
    buf = O.natural_to_real_layout(x, b, p)
    h = 1.0 / n
    gx = O.real_layout_to_natural(O.dx(buf, n, b, p, h), 2, n, b, p)
    gy = O.real_layout_to_natural(O.dy(buf, n, b, p, h), 2, n, b, p)
    rx = (np.roll(x, 2, 1) - 8 * np.roll(x, 1, 1) + 8 * np.roll(x, -1, 1) - np.roll(x, -2, 1)) / (12 * h)
    ry = (np.roll(x, 2, 0) - 8 * np.roll(x, 1, 0) + 8 * np.roll(x, -1, 0) - np.roll(x, -2, 0)) / (12 * h)
    assert relerr(gx, rx) < 1e-14
    assert relerr(gy, ry) < 1e-14
    # real Scalar path of the reference (dx.cu operates on double)
    xr = np.ascontiguousarray(buf.real)
    assert np.array_equal(O.dx(xr, n, b, p, h), np.ascontiguousarray(O.dx(buf, n, b, p, h).real))


def test_dx_rejects_b1():
    with pytest.raises(ValueError):
        O.dx(np.zeros(64 * 64, np.complex128), 64, 1, 2)


def test_generator_is_counter_based():
    a = O.uniform_field(5, 1000)
    b = O.uniform_field(5, 500, first=500)
    assert np.array_equal(a[500:], b)
    assert np.all(np.abs(a.real) <= 1) and np.all(np.abs(a.imag) <= 1)
    g = O.gaussian_field(2, 200000)
    assert abs(g.real.mean()) < 0.01 and abs(g.real.std() - 1) < 0.01
