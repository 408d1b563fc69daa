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


# The reference's own LARE-compatible IC package (src/InitialConditions/LARE,
# compiled unchanged by tests/cpp/Makefile where the reference tree exists;
# the binary travels with the checkout).
LARE_IC = os.path.join(ROOT, "tests", "cpp", "_build", "lare_ic_runner")


@pytest.mark.skipif(not os.path.exists(LARE_IC), reason="reference LARE IC driver not built on this machine")
def test_reference_lare_ic_package_boundary_table():
    """Its LAREBoundaryConditions (host functions) become device descriptors:
    the LARE BC_OTHER planes on all 13 variables' 6 edges, except dm in y and
    z, where the package's dm function does nothing (it only handles x)."""
    rc, out = _run(LARE_IC, "--check-setup")
    assert rc == 0, out
    assert '"lare_other_slots": 74, "none_slots": 4, "dm_y_z_none": true' in out, out


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(LARE_IC), reason="reference LARE IC driver not built on this machine")
@pytest.mark.parametrize("name", ["ot_lare_12x10x6_s5", "rf_lare_10x8x6_s4"])
def test_reference_lare_ic_package_on_gpu_matches_reference(name, tmp_path):
    """The runner with the reference's LARE IC package steps on the GPU and
    equals the reference's own run of that package (the *_lare_* fixtures:
    the same seeded state, BC_OTHER on every edge) bit for bit."""
    import numpy as np
    from sams_b200 import lare
    from tests.golden.make_golden import STATE, load
    z, meta = load(name)
    nx, ny, nz = meta["nx"], meta["ny"], meta["nz"]
    out = str(tmp_path / "state.bin")
    rc, log = _run(LARE_IC, "--run", meta["case"], nx, ny, nz, meta["steps"], meta["seed"], out)
    assert rc == 0, log
    assert f'"steps": {meta["steps"]}' in log and '"lare_other_slots": 74' in log, log
    boxes = np.fromfile(out, dtype="<f8").reshape(lare.NFIELDS, nx + 5, ny + 5, nz + 5)
    for f in STATE:
        ref = z[f]
        m = ~np.isnan(ref)
        got = boxes[lare.FIELD[f]]
        assert np.array_equal(got[m], ref[m]), f"{name}: {f} differs (max {np.abs(got[m] - ref[m]).max():.3e})"
