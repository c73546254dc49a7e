"""The C++ compat header (include/zmodel_compat.hpp): the reference's example() call
sequence compiles against it (CPU) and reproduces the oracle on the GPU."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from stencilfft_b200 import abi

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "compat_example.cpp"


def _build(tmp_path) -> Path:
    exe = tmp_path / "compat_example"
    libdir = abi.library_path().parent
    cmd = ["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include", str(SRC),
           f"-L{libdir}", "-lzmodel_b200", "-L/usr/local/cuda/lib64", "-lcudart",
           f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_compat_header_compiles_and_links(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_compat_example_matches_oracle(tmp_path):
    exe = _build(tmp_path)
    n, b, p = 256, 16, 2
    rng = np.random.default_rng(3)
    x = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    buf = O.natural_to_real_layout(x, b, p)
    paths = [tmp_path / f for f in ("in.bin", "lap.bin", "spec.bin", "back.bin")]
    buf.astype(np.complex128).tofile(paths[0])
    r = subprocess.run([str(exe), *map(str, paths), str(n), str(b), str(p)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lap = np.fromfile(paths[1], dtype=np.complex128)
    spec = np.fromfile(paths[2], dtype=np.complex128)
    back = np.fromfile(paths[3], dtype=np.complex128)
    ref_lap = O.laplace(buf, 2, n, b, p)
    assert np.array_equal(lap, ref_lap)
    ref_spec = O.forward_fft(ref_lap, 2, n, b, p)
    assert np.linalg.norm(spec - ref_spec) / np.linalg.norm(ref_spec) < 1e-12
    assert np.linalg.norm(back - ref_lap) / np.linalg.norm(ref_lap) < 1e-12
    ky, kx = O.index_map("reciprocal_to_global", n, b, p, 0, 0, 1, 2)
    assert f"({ky}, {kx})" in r.stdout
