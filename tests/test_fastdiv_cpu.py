"""The kernels' divide-by-invariant-integer helper (FastDiv) agrees with
integer / and % on the host for every divisor up to 70000."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "phase-field-dislocation-dynamics-pfdd-2.x_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_fastdiv_matches_integer_division(tmp_path):
    exe = str(tmp_path / "fastdiv_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, os.path.join(HERE, "fastdiv_check.cpp"), "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
