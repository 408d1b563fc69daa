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


# the reference tree, read in place where oracle/Makefile found it
def _ref_tree():
    from oracle import lare_oracle as lo
    return lo.reference_tree() or ""


REF_OT = os.path.join(_ref_tree(), "src", "InitialConditions", "OrszagTang")


@pytest.mark.skipif(not os.path.isdir(REF_OT), reason="reference tree not present on this machine")
def test_reference_ic_package_compiles_and_sets_up(tmp_path):
    """The reference's own Orszag-Tang IC package, compiled unchanged from its
    tree against include/sams/ (its includes of harness.h, runner.h,
    shared_data.h and builtInBoundaryConditions.h resolve to one-line shims),
    sets up a runner on the host: 128 x 128 x 2, gamma = 5/3, every variable
    periodic on every edge, fields as the package writes them."""
    from sams_b200 import build as sb
    lib = sb.build()
    shim = tmp_path / "shim"
    shim.mkdir()
    for h in ("harness.h", "runner.h", "shared_data.h", "builtInBoundaryConditions.h"):
        (shim / h).write_text('#include "sams/lare3d.hpp"\n')
    exe = str(tmp_path / "ref_ic")
    cmd = ["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), "-I", str(shim), "-I", REF_OT,
           os.path.join(ROOT, "tests", "cpp", "reference_ic_setup.cpp"), os.path.join(REF_OT, "OrszagTang.cpp"),
           "-o", exe, "-L", os.path.dirname(lib), "-lsams_lare", "-Wl,-rpath," + os.path.dirname(lib)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    rc, out = _run(exe)
    assert rc == 0, out
    assert '"nx": 128, "ny": 128, "nz": 2' in out and '"periodic_slots": 78' in out, out
