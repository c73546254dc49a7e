"""Benchmark of the interleaved block-cyclic FFT + stencil hot path on B200.

Workload (one step): the large 2D configuration -- N = 16384 (16384 x 16384), P = 4
(16 virtual ranks), B = 64 -- on a field that is a seeded sum of 32 random Fourier
modes (|k| <= N/8, unit complex Gaussian amplitudes) plus 1e-3 white noise:
    forward FFT -> inverse FFT (round trip, scale 1/N^2) -> 5-point Laplacian,
    4th-order dx and dy (h = 1/N) of the round-tripped field, the three stencils in
    one launch (zm_laplace_dx_dy; each output bit-identical to its own kernel).
The headline is the complex64 bulk form (compensated FP32 twiddles); the plain
complex128 form is measured beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is the device time of one step (ms, max over
ranks, lower is better).  With --gpus N > 1 (torchrun) every rank runs an independent
replica (the path is held on one GPU; there is no data-path collective).
The reference arm (--impl reference) times the same step on the host cores at the full
size in complex128: pocketfft (scipy.fft, the stand-in for the reference's FFTW baseline)
for the transforms and the oracle's OpenMP restatement of the reference's stencils.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N, P, B = 16384, 4, 64
NMODES, NOISE, MODE_SEED, NOISE_SEED = 32, 1e-3, 1, 1
METRIC = "fft_stencil_step_time"
WORKLOAD = ("2D N=16384 P=4 B=64: forward FFT + inverse FFT + 5-pt Laplacian + dx + dy "
            "(h=1/N, the three stencils in one launch) on 32 seeded Fourier modes + 1e-3 noise")


def modes_and_amps(n: int):
    """32 modes (kx, ky) uniform in the disc |k| <= n/8 (rejection sampling) and unit
    complex Gaussian amplitudes, drawn from numpy.random.default_rng(seed=1)."""
    import numpy as np
    rng = np.random.default_rng(MODE_SEED)
    kmax = n // 8
    modes = []
    while len(modes) < NMODES:
        kx, ky = (int(v) for v in rng.integers(-kmax, kmax + 1, 2))
        if kx * kx + ky * ky <= kmax * kmax:
            modes.append((kx, ky))
    amps = rng.standard_normal((NMODES, 2))
    return np.array(modes, dtype=np.int64), amps


def read_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(key: str):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary (profiles/traffic.txt):
    (bytes, source) -- the value is that capture's, not a measurement of this run."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None, None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == key:
            try:
                return float(parts[1]), "profiles/" + parts[2] if len(parts) > 2 else "profiles/traffic.txt"
            except ValueError:
                return None, None
    return None, None


class ClockSampler:
    """SM clock / throttle-reason sampling during the timed region: NVML polled every
    10 ms from a background thread (read-only queries), nvidia-smi at 200 ms as the
    fallback."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.thread = None
        self.rows = []

    def _nvml_loop(self, nv, h, stop):
        bits = [nv.nvmlClocksThrottleReasonHwSlowdown, nv.nvmlClocksThrottleReasonHwThermalSlowdown,
                nv.nvmlClocksThrottleReasonSwThermalSlowdown, nv.nvmlClocksThrottleReasonSwPowerCap]
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.rows.append((float(sm), float(mx), ["Active" if r & b else "Not Active" for b in bits]))
            except Exception:
                break
            stop.wait(0.01)

    def __enter__(self):
        try:
            import threading

            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self._stop = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h, self._stop), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self._stop.set()
            self.thread.join(timeout=5)
            return
        out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
        for line in (out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                self.rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue

    def summary(self):
        rows = self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        reasons = sorted({self.NAMES[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows),
                "source": "nvml, 10 ms" if self.thread is not None else "nvidia-smi, 200 ms"}


def max_over_ranks(value: float, dist=None, device: str = "cuda") -> float:
    """The largest `value` over all ranks of the default process group (itself when
    there is none).  Every rank must call it at the same point."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ CPU arm

def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class CpuStep:
    """The step on the host cores at the full size, N = 16384, complex128 (the
    reference's only precision; FP64 throughout).

    The reference's CPU baseline is FFTW through heFFTe (heffte/heffte_example_fftw.cpp),
    which is not installed; its stand-in is pocketfft (`scipy.fft.fft2` / `ifft2`, all
    host threads) on the natural-layout field.  The stencils are the oracle's OpenMP C
    restatement of the reference's laplace / dx / dy kernels with their halo exchanges
    (zmodel/stencils/laplace.cu:73-256, dx.cu:10-161, dy.cu:10-185) on the interleaved
    layout, all host threads.  One step = fft2 + ifft2 + Laplacian + dx + dy."""

    def __init__(self, threads: int | None = None):
        import numpy as np  # noqa: F401
        import oracle as O
        self.threads = threads or cpu_threads()
        O.set_threads(self.threads)
        self.x = O.uniform_field(0, N * N).reshape(N, N)
        self.buf = O.natural_to_real_layout(self.x, B, P)

    def run(self):
        """(ms of the two transforms, ms of the three stencils)."""
        import scipy.fft
        import oracle as O
        t0 = time.perf_counter()
        X = scipy.fft.fft2(self.x, workers=self.threads)
        back = scipy.fft.ifft2(X, workers=self.threads, overwrite_x=True)
        del X, back
        t1 = time.perf_counter()
        for f in (lambda: O.laplace(self.buf, 2, N, B, P), lambda: O.dx(self.buf, N, B, P, 1.0 / N),
                  lambda: O.dy(self.buf, N, B, P, 1.0 / N)):
            out = f()
            del out
        t2 = time.perf_counter()
        return (t1 - t0) * 1e3, (t2 - t1) * 1e3

    def describe(self, fft_ms: float, st_ms: float, runs: int) -> str:
        return (f"full workload N={N} complex128 on {self.threads} threads of {cpu_model()}: "
                f"pocketfft fft2+ifft2 (scipy.fft, the FFTW stand-in) {fft_ms:.0f} ms + oracle OpenMP "
                f"laplace+dx+dy on the interleaved layout {st_ms:.0f} ms; median of {runs} steps")


def cpu_baseline_sample(runs: int = 3):
    """The bounded CPU sample of the GPU arm: one warm-up step and the median of `runs`."""
    step = CpuStep()
    step.run()
    res = [step.run() for _ in range(runs)]
    tot = [a + b for a, b in res]
    k = tot.index(statistics.median(tot)) if runs % 2 else 0
    ms = statistics.median(tot)
    return ms, step.threads, step.describe(res[k][0], res[k][1], runs)


def run_reference(args, rank: int, world: int):
    """The reference arm: every step is the whole workload on the host cores (CpuStep)."""
    if rank != 0:
        return
    step = CpuStep()
    for _ in range(args.warmup):
        step.run()
    res = [step.run() for _ in range(args.steps)]
    tot = [a + b for a, b in res]
    v = statistics.mean(tot)
    med = statistics.median(tot)
    sample = step.describe(statistics.mean(a for a, _ in res), statistics.mean(b for _, b in res), args.steps)
    line = {"metric": METRIC, "value": round(v, 2), "unit": "ms", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 2), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (U[-1,1) seed 0)",
            "config": {"workload": WORKLOAD, "n": N, "p": P, "b": B, "dtype": "c128 (FP64, the reference's only form)"},
            "median_ms": round(med, 2),
            "cpu_baseline": {"value": round(v, 2), "unit": "ms", "cores": step.threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(v, 2), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm

def run_ours(args, rank: int, world: int):
    import numpy as np
    import torch
    from stencilfft_b200 import Plan, launch_count

    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_
    stream = torch.cuda.current_stream()
    modes, amps = modes_and_amps(N)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def run_dtype(dt: str, timed_steps: int, warmup: int, with_e2e: bool, spec_ref=None):
        pl = Plan(2, N, B, P, dtype=dt)
        u = pl.empty()
        pl.fill_modes(u, modes, amps, NOISE, NOISE_SEED)
        spec, back, work = pl.empty(), pl.empty(), pl.empty()
        lap, gx, gy = pl.empty(), pl.empty(), pl.empty()
        h = 1.0 / N
        marks = []

        def step(record=None):
            e = [ev() for _ in range(4)] if record is not None else None
            if e: e[0].record(stream)
            pl.forward_fft(u, spec, work=work)
            if e: e[1].record(stream)
            pl.inverse_fft(spec, back, scale=1.0 / (N * N), work=work)
            if e: e[2].record(stream)
            # Laplacian, dx, dy in one launch (each bit-identical to its own kernel)
            pl.laplace_dx_dy(back, lap, gx, gy, inv_h2=1.0 / (h * h), delta=h)
            if e: e[3].record(stream)
            if record is not None:
                record.append(e)

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        if dist: dist.barrier()
        torch.cuda.synchronize()
        l0 = launch_count()
        t0, t1 = ev(), ev()
        with ClockSampler(local) as cs:
            t0.record(stream)
            for _ in range(timed_steps):
                step(marks)
            t1.record(stream)
            torch.cuda.synchronize()
        launches = launch_count() - l0
        if dist: dist.barrier()
        ms = t0.elapsed_time(t1) / timed_steps
        stage = {k: statistics.mean(m[i].elapsed_time(m[i + 1]) for m in marks)
                 for i, k in enumerate(["fwd", "inv", "laplace_dx_dy"])}
        # accuracy of the round trip, in FP64 on the device
        err = float(torch.linalg.vector_norm((back - u).to(torch.complex128)) /
                    torch.linalg.vector_norm(u.to(torch.complex128)))
        res = {"ms": ms, "stage_ms": stage, "launches": launches, "clocks": cs.summary(),
               "roundtrip_rel_l2": err, "field_bytes": pl.field_bytes}
        if spec_ref is not None:
            # spectrum of this form against the other form's (complex128: FP64 arithmetic)
            s128 = spec.to(torch.complex128)
            d = torch.linalg.vector_norm(spec_ref - s128) / torch.linalg.vector_norm(s128)
            res["spec_rel_l2_vs_other"] = float(d)
            res["spec_max_abs_vs_other"] = float((spec_ref - s128).abs().max() / s128.abs().max())
            del s128
        elif dt == "c64":
            res["spec"] = spec.to(torch.complex128)
        if with_e2e:
            # Through the C ABI with host buffers: every step copies its input from pinned
            # host memory (H2D), runs the step and copies the three outputs back (D2H).
            # Consecutive steps are pipelined on three streams (H2D / compute / D2H) with
            # double-buffered device inputs and outputs, so step i's D2H overlaps step
            # i+1's H2D and compute; the time per step is the whole loop / steps.
            host_in = torch.empty(pl.total, dtype=pl.torch_dtype, pin_memory=True)
            host_in.copy_(u.cpu())
            host_out = [torch.empty(pl.total, dtype=pl.torch_dtype, pin_memory=True) for _ in range(3)]
            s_in, s_cp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
            dins = [u, pl.empty()]
            douts = [(lap, gx, gy), (pl.empty(), pl.empty(), pl.empty())]

            def run_steps(k, t0=None, t1=None):
                ev_cp, ev_out = [None] * k, [None] * k
                if t0 is not None:
                    t0.record(s_in)
                for i in range(k):
                    bi = i % 2
                    if i >= 2:
                        s_in.wait_event(ev_cp[i - 2])    # step i-2 has finished reading dins[bi]
                    with torch.cuda.stream(s_in):
                        dins[bi].copy_(host_in, non_blocking=True)
                    e_in = torch.cuda.Event()
                    e_in.record(s_in)
                    s_cp.wait_event(e_in)
                    if i >= 2:
                        s_cp.wait_event(ev_out[i - 2])   # step i-2's outputs are on the host
                    pl.forward_fft(dins[bi], spec, work=work, stream=s_cp)
                    pl.inverse_fft(spec, back, scale=1.0 / (N * N), work=work, stream=s_cp)
                    pl.laplace_dx_dy(back, *douts[bi], inv_h2=1.0 / (h * h), delta=h, stream=s_cp)
                    ev_cp[i] = torch.cuda.Event()
                    ev_cp[i].record(s_cp)
                    s_out.wait_event(ev_cp[i])
                    with torch.cuda.stream(s_out):
                        for hb, db in zip(host_out, douts[bi]):
                            hb.copy_(db, non_blocking=True)
                    ev_out[i] = torch.cuda.Event()
                    ev_out[i].record(s_out)
                if t1 is not None:
                    t1.record(s_out)

            run_steps(2)
            torch.cuda.synchronize()
            reps = max(2, timed_steps)
            a, b_ = ev(), ev()
            run_steps(reps, a, b_)
            torch.cuda.synchronize()
            res["e2e_ms"] = a.elapsed_time(b_) / reps
            res["e2e_steps"] = reps
            res["h2d"] = pl.field_bytes
            res["d2h"] = 3 * pl.field_bytes
            del host_in, host_out, dins, douts
        del u, spec, back, work, lap, gx, gy
        pl.close()
        torch.cuda.empty_cache()
        return res

    main = run_dtype("c64", args.steps, args.warmup, with_e2e=True)
    side = None
    try:
        side = run_dtype("c128", max(2, args.steps // 2), max(3, args.warmup), with_e2e=False,
                         spec_ref=main.pop("spec"))
    except Exception as ex:  # c128 at this N may be unsupported by the build
        side = {"error": str(ex).splitlines()[0]}
    main.pop("spec", None)
    torch.cuda.empty_cache()

    def gmax(v: float) -> float:
        return max_over_ranks(v, dist, "cuda")

    ms = gmax(main["ms"])
    e2e_ms = gmax(main["e2e_ms"])
    F = main["field_bytes"]
    peak, peak_kind = read_peaks()
    # dominant kernel: the three-stage fused line pass of the forward transform (2 launches
    # per forward call: x pass persistent, y pass on buddy-line CTA pairs)
    t_launch = main["stage_ms"]["fwd"] / 2
    achieved = (2 * F) / (t_launch * 1e-3) / 1e9
    traffic, traffic_src = read_traffic("k3_pass_fwd_c64_N16384")
    fft_flops = 5.0 * N * N * math.log2(N * N)
    # algorithmic bytes: 4F per 2D transform, 2F per stencil (6F for the three fused
    # stencils, which move 4F: one read, three writes)
    stages = {k: {"ms": round(v, 4), "GBps": round((4 * F if k in ("fwd", "inv") else 6 * F) / (v * 1e-3) / 1e9, 1)}
              for k, v in main["stage_ms"].items()}
    st = main["stage_ms"]["laplace_dx_dy"]
    stages["laplace_dx_dy"]["moved_GBps"] = round(4 * F / (st * 1e-3) / 1e9, 1)
    stages["laplace_dx_dy"]["note"] = "three stencils in one launch: 6F algorithmic, 4F moved"
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cms, cores, sample = cpu_baseline_sample()
        cpu = {"value": round(cms, 2), "unit": "ms", "cores": cores, "kind": "port", "sample": sample}
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(ms, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64", "data": "synthetic (32 seeded Fourier modes + 1e-3 noise)",
        "config": {"workload": WORKLOAD, "n": N, "p": P, "b": B, "dtype": "c64 (compensated FP32 twiddles)",
                   "l2": "inputs larger than L2 (2 GiB field per buffer)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "kernel": "k3_pass_kernel<6,8,fwd> (x pass persistent, y pass on buddy-line CTA pairs)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic, "traffic_source": f"committed ncu capture ({traffic_src})",
                     "algorithmic_bytes_per_launch": 2 * F},
        "stages": stages,
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": main["h2d"],
                "d2h_bytes_per_step": main["d2h"], "steps": main["e2e_steps"],
                "how": "C ABI with pinned host buffers; H2D, compute and D2H of consecutive steps "
                       "pipelined on three streams"},
        "gpu_launches": main["launches"],
        "clocks": main["clocks"],
        "gflops": {"fwd": round(fft_flops / (main["stage_ms"]["fwd"] * 1e-3) / 1e9, 1),
                   "inv": round(fft_flops / (main["stage_ms"]["inv"] * 1e-3) / 1e9, 1),
                   "convention": "5 N^2 log2(N^2) per transform"},
        "accuracy": {"c64_roundtrip_rel_l2": main["roundtrip_rel_l2"],
                     "c64_fwd_rel_l2_vs_c128": side.get("spec_rel_l2_vs_other"),
                     "c64_fwd_max_abs_rel_vs_c128": side.get("spec_max_abs_vs_other")},
        "c128": ({"ms": round(side["ms"], 4), "stage_ms": {k: round(v, 4) for k, v in side["stage_ms"].items()},
                  "roundtrip_rel_l2": side["roundtrip_rel_l2"],
                  "c128_over_c64": round(side["ms"] / main["ms"], 3)} if "ms" in side else side),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_profile_case(args):
    """Small profiling case (N = 8192, c64 by default, 512 MiB per buffer; or the 3D
    Laplacian at N = 512): one warm-up and one measured call of each stage, for
    `ncu -k ... -s/-c` captures."""
    import torch
    from stencilfft_b200 import Plan, abi
    if args.profile_ops == "fft3d":
        # 3D forward + inverse transform with a workspace, N = 512, P = 4, B = 32 (1 GiB per
        # c64 field, three fields)
        n3 = 512
        pl3 = Plan(3, n3, 32, P, dtype=args.profile_dtype)
        u3, s3, w3 = pl3.empty(), pl3.empty(), pl3.empty()
        pl3.fill(u3, abi.ZM_FIELD_GAUSSIAN, 2)
        for _ in range(2):
            pl3.forward_fft(u3, s3, work=w3)
            pl3.inverse_fft(s3, u3, scale=1.0 / n3 ** 3, work=w3)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": {"dim": 3, "n": n3, "p": P, "b": 32, "dtype": args.profile_dtype,
                                           "ops": "fft3d", "field_bytes": pl3.field_bytes}}))
        return
    if args.profile_ops == "batch":
        # the 96-field Poisson batch (32 x 256^2, 32 x 512^2, 24 x 1024^2, 8 x 2048^2; P = 2,
        # B = N / 8), two calls
        from stencilfft_b200 import Batch
        sizes = [256] * 32 + [512] * 32 + [1024] * 24 + [2048] * 8
        bt = Batch(sizes, [n // 8 for n in sizes], [2] * len(sizes), dtype=args.profile_dtype)
        rhs, phi, res, work = bt.empty(), bt.empty(), bt.empty(), bt.empty()
        bt.fill(rhs, abi.ZM_FIELD_GAUSSIAN, 100)
        for _ in range(2):
            bt.poisson(rhs, phi, res, work, length=1.0)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": {"ops": "batch", "fields": len(sizes), "dtype": args.profile_dtype,
                                           "elems": bt.total}}))
        return
    if args.profile_ops == "layout":
        # natural -> interleaved converter, a reciprocal-space pointwise operator and the
        # natural <-> reciprocal converters, N = 8192
        n = args.profile_n
        pl = Plan(2, n, B, P, dtype=args.profile_dtype)
        nat, buf = pl.empty(), pl.empty()
        pl.fill(nat, abi.ZM_FIELD_GAUSSIAN, 3)
        for _ in range(2):
            pl.natural_to_real(nat, buf)
            pl.spectral_apply(buf, abi.ZM_SPECTRAL_GAUSSIAN, n / 16)
            pl.natural_to_reciprocal(nat, buf)
            pl.reciprocal_to_natural(buf, nat)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": {"n": n, "p": P, "b": B, "dtype": args.profile_dtype,
                                           "ops": "layout", "field_bytes": pl.field_bytes}}))
        return
    if args.profile_ops == "lap3d":
        # 3D 7-point Laplacian, N = 512, P = 4, B = 32 (1 GiB per c64 field, two fields)
        n3 = 512
        pl3 = Plan(3, n3, 32, P, dtype=args.profile_dtype)
        u3, o3 = pl3.empty(), pl3.empty()
        pl3.fill(u3, abi.ZM_FIELD_GAUSSIAN, 2)
        for _ in range(2):
            pl3.laplace(u3, o3, inv_h2=float(n3 * n3))
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": {"dim": 3, "n": n3, "p": P, "b": 32, "dtype": args.profile_dtype,
                                           "ops": "lap3d", "field_bytes": pl3.field_bytes}}))
        return
    n = args.profile_n
    pl = Plan(2, n, B, P, dtype=args.profile_dtype)
    modes, amps = modes_and_amps(n)
    u = pl.empty()
    pl.fill_modes(u, modes, amps, NOISE, NOISE_SEED)
    if args.profile_ops == "inv":
        # inverse transform only (with a workspace): three buffers on the device
        back, work = pl.empty(), pl.empty()
        for _ in range(2):
            pl.inverse_fft(u, back, scale=1.0 / (n * n), work=work)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": {"n": n, "p": P, "b": B, "dtype": args.profile_dtype,
                                           "ops": "inv", "field_bytes": pl.field_bytes}}))
        return
    if args.profile_ops == "stencils":
        # the three 2D stencils in one launch (Laplacian, dx, dy): four buffers
        lap, gx, gy = pl.empty(), pl.empty(), pl.empty()
        for _ in range(2):
            pl.laplace_dx_dy(u, lap, gx, gy, inv_h2=float(n * n), delta=1.0 / n)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": {"n": n, "p": P, "b": B, "dtype": args.profile_dtype,
                                           "ops": "stencils", "field_bytes": pl.field_bytes}}))
        return
    if args.profile_ops == "fwd":
        # forward transform only (with a workspace, as in the timed step): three buffers
        spec, work = pl.empty(), pl.empty()
        for _ in range(2):
            pl.forward_fft(u, spec, work=work)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": {"n": n, "p": P, "b": B, "dtype": args.profile_dtype,
                                           "ops": "fwd", "field_bytes": pl.field_bytes}}))
        return
    spec, back, work = pl.empty(), pl.empty(), pl.empty()
    lap, gx, gy = pl.empty(), pl.empty(), pl.empty()
    for _ in range(2):
        pl.forward_fft(u, spec, work=work)
        pl.inverse_fft(spec, back, scale=1.0 / (n * n), work=work)
        pl.laplace_dx_dy(back, lap, gx, gy, inv_h2=float(n * n), delta=1.0 / n)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": {"n": n, "p": P, "b": B, "dtype": args.profile_dtype,
                                       "field_bytes": pl.field_bytes}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--profile-case", action="store_true",
                    help="run the small profiling case only (for ncu captures)")
    ap.add_argument("--profile-n", type=int, default=8192)
    ap.add_argument("--profile-dtype", default="c64")
    ap.add_argument("--profile-ops", choices=["all", "fwd", "inv", "stencils", "lap3d", "fft3d", "batch", "layout"],
                    default="all")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile_case:
        run_profile_case(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
