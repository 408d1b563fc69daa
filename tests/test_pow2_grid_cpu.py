"""The host test that selects the reciprocal instantiation of the kernels
(sams::pow2_grid): it must accept exactly the uniform Cartesian grids whose
spacings and mu0 are powers of two (the 256^3 cube, Orszag-Tang 128 x 128 x
4) and refuse the others (1/250, the Harris grid's 5/128, an offset axis,
mu0 = 4 pi 1e-7), and every reciprocal it returns must reproduce the
division bit for bit, subnormal quotients included.  Compiled as host code."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not present")
def test_pow2_grid_accepts_exactly_the_power_of_two_grids(tmp_path):
    exe = str(tmp_path / "pow2_grid")
    r = subprocess.run(["nvcc", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                        "-I", os.path.join(ROOT, "sams_b200", "csrc"),
                        os.path.join(ROOT, "tests", "cpp", "pow2_grid.cu"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and '"bad": 0' in r.stdout, r.stdout + r.stderr
