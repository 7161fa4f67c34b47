"""The row steppers of the peeled row pass, checked on the host: along every
row of many shapes (coprime and not, both index widths) the values they carry
from column to column equal the C2R and R2C row shuffle functors evaluated at
each column (tests/cxx/row_stepper.cu, compiled by nvcc as host code)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_row_steppers_match_the_functors(tmp_path):
    nvcc = next((c for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc")
                 if c and os.path.exists(c)), None)
    if nvcc is None:
        pytest.skip("nvcc not found")
    exe = str(tmp_path / "row_stepper")
    build = subprocess.run([nvcc, "-std=c++17", "-O2", "-x", "cu", "-I" + os.path.join(ROOT, "213transpose_b200", "csrc"),
                            "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cxx", "row_stepper.cu"),
                            "-o", exe], capture_output=True, text=True)
    assert build.returncode == 0, build.stderr[-2000:]
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.startswith("ok"), run.stdout + run.stderr
