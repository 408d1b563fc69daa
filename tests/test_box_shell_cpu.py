"""The ghost-shell walk the fused x / y sweep uses to complete its
out-of-place arrays (sams::BoxShell): compiled as host code and checked to
produce every box point outside the inner cube exactly once.  A point it
missed would keep a stale value wherever no boundary fill overwrites it, so
this is checked directly rather than through the parity runs."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not present")
def test_box_shell_covers_the_shell_exactly_once(tmp_path):
    exe = str(tmp_path / "box_shell")
    r = subprocess.run(["nvcc", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                        "-I", os.path.join(ROOT, "sams_b200", "csrc"),
                        os.path.join(ROOT, "tests", "cpp", "box_shell.cu"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and '"bad": 0' in r.stdout, r.stdout + r.stderr
