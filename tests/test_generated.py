"""The generated dispatch sources (zm_fft2_<dtype>_<dir>.cu) are what gen_fused.py writes
from its variant and configuration tables, so the tables documented there are the ones
compiled into the library."""
import shutil
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parents[1] / "stencilfft_b200" / "csrc"
GENERATED = ["zm_fft2_c64_fwd.cu", "zm_fft2_c64_inv.cu", "zm_fft2_c128_fwd.cu", "zm_fft2_c128_inv.cu"]


def test_generated_dispatch_is_up_to_date(tmp_path):
    shutil.copy(CSRC / "gen_fused.py", tmp_path / "gen_fused.py")
    subprocess.run([sys.executable, "gen_fused.py"], cwd=tmp_path, check=True)
    for name in GENERATED:
        assert (tmp_path / name).read_text() == (CSRC / name).read_text(), name


def test_three_stage_variants_listed_for_the_bench_size():
    """The 2^14-point complex64 lines (VEC = 64, M = 256) list the three-stage kernels and
    the out-of-place configurations use them."""
    src = (CSRC / "zm_fft2_c64_fwd.cu").read_text()
    assert "launch_k3<6, 8, false, true, false>" in src     # persistent
    assert "launch_k3<6, 8, false, false, true>" in src     # buddy-line pairs
    inv = (CSRC / "zm_fft2_c64_inv.cu").read_text()
    assert "launch_k3<6, 8, true, true, false>" in inv
