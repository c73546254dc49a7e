"""CPU checks of the reference GPU runner's host side (no GPU needed).

* The in-process MPI stand-in (oracle/refgpu/mpi_shim.cpp) delivers what MPI would for
  the reference's call pattern: row / column communicators from MPI_Comm_split,
  MPI_Alltoall over each, the four halo MPI_Sendrecv of communicate_laplace and
  MPI_Reduce(MAX), on P*P host threads for P = 1..4.
* Every runner library built from the reference sources loads, reports the layout it
  was compiled for and exports only the driver's entry points.
"""
import ctypes
import re
import subprocess

import pytest

from oracle import refgpu as R

HERE = R.HERE


def _selftest_lib():
    subprocess.run(["make", "-C", str(HERE), "libzr_mpi_selftest.so"], check=True,
                   stdout=subprocess.DEVNULL)
    L = ctypes.CDLL(str(HERE / "libzr_mpi_selftest.so"))
    L.zr_mpi_selftest.argtypes = [ctypes.c_int]
    L.zr_mpi_selftest.restype = ctypes.c_int
    return L


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_mpi_standin_collectives(p):
    assert _selftest_lib().zr_mpi_selftest(p) == 0


def test_stage_time_parser():
    log = "FFT0 1200 ns\nPACK0 300 ns\nFFT0 1100 ns\nTOTAL 5000 ns\n\nnoise\n"
    assert R.stage_times(log) == {"FFT0": [1200, 1100], "PACK0": [300], "TOTAL": [5000]}


def _built():
    return sorted(R.REF_DIR.glob("libzref_gpu_*.so"))


@pytest.mark.skipif(not _built(), reason="reference GPU runner not built")
def test_runner_libraries_load_and_report_their_layout():
    for path in _built():
        m = re.match(r"libzref_gpu_N(\d+)_B(\d+)_P(\d+)(_aware)?\.so", path.name)
        n, b, p, aware = int(m[1]), int(m[2]), int(m[3]), bool(m[4])
        pipe = R.RefPipeline(n, b, p, aware)
        assert (pipe.n, pipe.b, pipe.p, pipe.gpu_aware) == (n, b, p, aware)
        out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True,
                             text=True, check=True).stdout
        exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
        assert {"zr_config", "zr_fft", "zr_laplace", "zr_dxdy"} <= exported
        assert not any(s.startswith("MPI_") for s in exported), path.name
