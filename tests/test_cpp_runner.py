"""The C++ runner API (include/sams/): a reference-style initial-condition
package driven by SAMS::runner<LARE::LARE3D, ...>.

The host-only test checks event order, harness variable ranges, the
boundary-condition table and the IC values; the GPU test steps the runner on
the device and checks every field bit for bit against the oracle started from
the same initial state (tests/cpp/runner_ot.cpp).
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def runner_bin(tmp_path_factory, oracle_lib):
    from sams_b200 import build as sb
    lib = sb.build()
    libdir = os.path.dirname(lib)
    odir = os.path.join(ROOT, "oracle", "_build")
    exe = str(tmp_path_factory.mktemp("cpp") / "runner_ot")
    cmd = ["g++", "-std=c++20", "-O2", "-ffp-contract=off", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle"),
           os.path.join(ROOT, "tests", "cpp", "runner_ot.cpp"), "-o", exe,
           "-L", libdir, "-lsams_lare", "-L", odir, "-llare_oracle",
           "-Wl,-rpath," + libdir + ":" + odir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout + r.stderr


def test_runner_setup_host(runner_bin):
    rc, out = _run(runner_bin, "--check-setup")
    assert rc == 0, out
    assert '"check_setup": "ok"' in out


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps,shape", [(3, (24, 20, 4)), (4, (40, 32, 12))])
def test_runner_gpu_matches_oracle(runner_bin, nsteps, shape):
    rc, out = _run(runner_bin, "--run", nsteps, *shape)
    assert rc == 0, out
    assert '"mismatches": 0' in out and '"time_ok": true' in out, out
