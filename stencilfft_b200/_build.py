"""Build libzmodel_b200.so in-tree (nvcc, sm_100a only).

    python -m stencilfft_b200._build        # or stencilfft_b200._build.build()

Each .cu is compiled separately (in parallel) for ``-gencode arch=compute_100a,code=sm_100a``
with ``-lineinfo`` and linked into ``stencilfft_b200/lib/libzmodel_b200.so``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "lib"
LIB = OUT_DIR / "libzmodel_b200.so"
BUILD_DIR = ROOT / "_build" / "zmodel_b200"

SOURCES = ["zm_api.cu", "zm_fft.cu", "zm_stencil.cu", "zm_layout.cu", "zm_static.cu", "zm_batch.cu", "zm_fft2_c64_fwd.cu",
           "zm_fft2_c64_inv.cu", "zm_fft2_c128_fwd.cu", "zm_fft2_c128_inv.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else (shutil.which("nvcc") or "nvcc")


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "zmodel_b200.h"]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(verbose: bool = False, extra: list[str] | None = None, force: bool = False) -> Path:
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    extra = extra or []
    objs = []
    jobs = []
    for s in SOURCES:
        src = CSRC / s
        obj = BUILD_DIR / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append([nvcc(), *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        return r

    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        list(ex.map(run, jobs))
    if jobs or not LIB.exists() or force:
        run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"])
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = [a for a in sys.argv[1:] if a not in ("-v", "--force")]
    print(build(verbose=v, extra=extra, force="--force" in sys.argv))
