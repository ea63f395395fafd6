"""The reference-arithmetic sweep divides its window sums by the window side with
Markstein's correction (three instructions) instead of a division.  Its results are
bit-exact only if that equals the IEEE division for every input: compiled from the
library's own header, it is compared with x / n for every float bit pattern and every
window side 3..15 on the GPU."""
import pathlib
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = pathlib.Path(__file__).resolve().parent


def test_window_division_equals_ieee_division_for_every_float(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "div_win_check"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-o", str(exe),
                    str(HERE / "cuda" / "div_win_check.cu")], check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 7, r.stdout + r.stderr
    for line in lines:
        assert " 0 differences" in line and "no error" in line, line
    assert r.returncode == 0
