"""Batches of uneven-N 2D fields (zm_batch_*): one persistent launch per call.

* small mixed batches against the oracle, field by field (forward, inverse, generator);
* the spectral Poisson pipeline (forward -> divide by -|k|^2 -> inverse -> 5-point
  Laplacian residual) against the same pipeline in FP64 numpy;
* the batching workload: 96 complex64 fields (32 x 256^2, 32 x 512^2, 24 x 1024^2,
  8 x 2048^2), P = 2, B chosen by the autotuner, N(0,1) fields from seeds 100..195,
  the pipeline captured in a CUDA graph and replayed; per-field residual error vs FP64.
"""
import numpy as np
import pytest

import oracle as O
from helpers import TOL, relerr, to_host

pytestmark = pytest.mark.gpu

# (the VEC = 4 complex64 tiles, whose row stage runs fused with the vector-side sweeps, at
# M = 16, 64, 128, 256, 512: (64, 8, 2), (256, 32, 2), (512, 32, 4), (1024, 128, 2), (2048, 256, 2))
MIXED = [(64, 4, 2), (128, 8, 2), (256, 16, 2), (128, 2, 4), (512, 32, 4), (64, 16, 2), (256, 1, 2),
         (64, 8, 2), (256, 32, 2), (1024, 128, 2), (2048, 256, 2)]


def _batch(fields, dt):
    from stencilfft_b200 import Batch
    return Batch([f[0] for f in fields], [f[1] for f in fields], [f[2] for f in fields], dtype=dt)


def _fp64_poisson(rhs_nat, length=1.0):
    """phi and residual of the spectral Poisson solve in FP64 (natural layout)."""
    n = rhs_nat.shape[0]
    k = np.fft.fftfreq(n, 1.0 / n) * (2 * np.pi / length)
    ksq = k[:, None] ** 2 + k[None, :] ** 2
    ksq[0, 0] = 1.0
    s = np.fft.fft2(rhs_nat) / (-ksq)
    s[0, 0] = 0.0
    phi = np.fft.ifft2(s)
    h = length / n
    lap = (np.roll(phi, 1, 0) + np.roll(phi, -1, 0) + np.roll(phi, 1, 1) + np.roll(phi, -1, 1) - 4 * phi) / h ** 2
    return phi, lap - rhs_nat


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_batch_forward_inverse_fill_against_oracle(dt):
    import torch
    from stencilfft_b200 import Plan, abi
    bt = _batch(MIXED, dt)
    x, spec, back, work = bt.empty(), bt.empty(), bt.empty(), bt.empty()
    bt.fill(x, abi.ZM_FIELD_GAUSSIAN, 40)
    bt.forward_fft(x, spec)
    bt.inverse_fft(spec, back, work=work)
    assert bt.status() == 0
    for i, (n, b, p) in enumerate(MIXED):
        xi = to_host(bt.field(x, i))
        # the generator matches the single-field plan's, element for element
        pl = Plan(2, n, b, p, dtype=dt)
        ref_fill = pl.empty()
        pl.fill(ref_fill, abi.ZM_FIELD_GAUSSIAN, 40 + i)
        assert np.array_equal(xi, to_host(ref_fill)), i
        assert relerr(to_host(bt.field(spec, i)), O.forward_fft(xi, 2, n, b, p)) < TOL[dt], i
        assert relerr(to_host(bt.field(back, i)), xi) < TOL[dt], i
    # work = None: `in` is scratch, results unchanged
    spec2 = spec.clone()
    bt.inverse_fft(spec2, back)
    for i in range(len(MIXED)):
        assert relerr(to_host(bt.field(back, i)), to_host(bt.field(x, i))) < TOL[dt], i
    torch.cuda.synchronize()


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_batch_poisson_against_fp64(dt):
    from stencilfft_b200 import abi
    bt = _batch(MIXED, dt)
    rhs, phi, res, work = bt.empty(), bt.empty(), bt.empty(), bt.empty()
    bt.fill(rhs, abi.ZM_FIELD_GAUSSIAN, 7)
    bt.poisson(rhs, phi, res, work, length=2.0)
    assert bt.status() == 0
    tol = 1e-12 if dt == "c128" else 1e-5
    # the residual is a difference of nearly equal terms: phi's FP32 rounding, times the
    # 5-point stencil / h^2, is amplified by about 8 N / (2 pi)^2 relative to rhs
    tol_res = 1e-12 if dt == "c128" else 2e-4
    for i, (n, b, p) in enumerate(MIXED):
        r_nat = O.real_layout_to_natural(to_host(bt.field(rhs, i)), 2, n, b, p)
        phi_ref, res_ref = _fp64_poisson(r_nat, length=2.0)
        phi_nat = O.real_layout_to_natural(to_host(bt.field(phi, i)), 2, n, b, p)
        res_nat = O.real_layout_to_natural(to_host(bt.field(res, i)), 2, n, b, p)
        assert relerr(phi_nat, phi_ref) < tol, (i, relerr(phi_nat, phi_ref))
        assert relerr(res_nat, res_ref) < tol_res, (i, relerr(res_nat, res_ref))


def test_batch_rejects_bad_input():
    from stencilfft_b200 import Batch, ZmError
    with pytest.raises(ZmError):
        Batch([32], [2], [2], dtype="c64")          # below the batch range for complex64
    with pytest.raises(ZmError):
        Batch([8192], [32], [2], dtype="c64")       # above it
    with pytest.raises(ZmError):
        Batch([256], [128], [2], dtype="c64")       # P does not divide VEC
    bt = Batch([256, 512], [16, 32], [2, 2], dtype="c64")
    a = bt.empty()
    with pytest.raises(ZmError):
        bt.poisson(a, a, None, bt.empty())           # rhs and phi overlap


SIZES = [256] * 32 + [512] * 32 + [1024] * 24 + [2048] * 8


def test_batching_workload_graph():
    """The 96-field workload: B autotuned per N, the pipeline captured in a CUDA graph,
    replayed; per-field residual vs FP64 (rel-L2)."""
    import torch
    from stencilfft_b200 import Batch, abi, launch_count
    best = {n: Batch.autotune_b(n, 2, "c64", count=SIZES.count(n), reps=2)[0] for n in sorted(set(SIZES))}
    bt = Batch(SIZES, [best[n] for n in SIZES], [2] * len(SIZES), dtype="c64")
    rhs, phi, res, work = bt.empty(), bt.empty(), bt.empty(), bt.empty()
    bt.fill(rhs, abi.ZM_FIELD_GAUSSIAN, 100)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        bt.poisson(rhs, phi, res, work, length=1.0)
    l0 = launch_count()
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    assert launch_count() == l0    # replays launch nothing through the host API
    assert bt.status() == 0
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    reps = 10
    for _ in range(reps):
        graph.replay()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    worst = {}
    for i, n in enumerate(SIZES):
        r_nat = O.real_layout_to_natural(to_host(bt.field(rhs, i)), 2, n, best[n], 2)
        phi_ref, res_ref = _fp64_poisson(r_nat)
        phi_nat = O.real_layout_to_natural(to_host(bt.field(phi, i)), 2, n, best[n], 2)
        res_nat = O.real_layout_to_natural(to_host(bt.field(res, i)), 2, n, best[n], 2)
        e_phi, e_res = relerr(phi_nat, phi_ref), relerr(res_nat, res_ref)
        e_norm = abs(np.linalg.norm(res_nat) - np.linalg.norm(res_ref)) / np.linalg.norm(res_ref)
        w = worst.setdefault(n, [0.0, 0.0, 0.0])
        worst[n] = [max(w[0], e_phi), max(w[1], e_res), max(w[2], e_norm)]
    print(f"\nbatch of 96 fields (B per N {best}): {ms:.3f} ms per graph replay, "
          f"{96 / (ms * 1e-3):.0f} fields/s; worst per N of (phi rel-L2, residual rel-L2, "
          f"|residual norm| rel) vs FP64: " + ", ".join(f"{n}: ({a:.2e}, {b:.2e}, {c:.2e})"
                                                   for n, (a, b, c) in sorted(worst.items())))
    for n, (e_phi, e_res, e_norm) in worst.items():
        assert e_phi < 1e-5 and e_norm < 1e-5, (n, e_phi, e_norm)
        assert e_res < 1e-6 * n, (n, e_res)   # amplified rounding of phi (see above)
    del graph


def test_barrier_timeout_is_reported_not_hung():
    """Failure detection without a fault: a grid barrier that can never complete (one
    arrival more than the grid has) gives up after its 2 s limit, the kernel returns,
    the status reports it, and the context stays usable for the next call."""
    import time

    from stencilfft_b200 import abi
    bt = _batch(MIXED[:3], "c64")
    bt.barrier_probe(0)
    assert bt.status() == 0
    t0 = time.perf_counter()
    bt.barrier_probe(1)
    assert bt.status() == 1
    assert time.perf_counter() - t0 < 30
    assert bt.status() == 0                       # the flag was cleared
    x, y = bt.empty(), bt.empty()
    bt.fill(x, abi.ZM_FIELD_GAUSSIAN, 1)
    bt.forward_fft(x, y)
    assert bt.status() == 0
    for i, (n, b, p) in enumerate(MIXED[:3]):
        xi = to_host(bt.field(x, i))
        assert relerr(to_host(bt.field(y, i)), O.forward_fft(xi, 2, n, b, p)) < TOL["c64"]


def test_timeout_ends_only_its_own_launch():
    """A barrier timeout aborts only the launch it happened in: a call made after it,
    before anyone reads the status, still runs every step; the sticky flag then still
    reports the earlier timeout once, and is cleared."""
    from stencilfft_b200 import abi
    bt = _batch(MIXED[:3], "c64")
    bt.barrier_probe(1)                           # times out (2 s), flag left set
    x, y = bt.empty(), bt.empty()
    bt.fill(x, abi.ZM_FIELD_GAUSSIAN, 2)
    bt.forward_fft(x, y)
    for i, (n, b, p) in enumerate(MIXED[:3]):
        xi = to_host(bt.field(x, i))
        assert relerr(to_host(bt.field(y, i)), O.forward_fft(xi, 2, n, b, p)) < TOL["c64"]
    assert bt.status() == 1
    assert bt.status() == 0
