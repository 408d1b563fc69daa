"""GPU timestep (libsams_lare.so through its C ABI) against the reference.

Bit-for-bit against the reference's own outputs (tests/golden, made by the
compiled reference) and against the CPU checker at further sizes; at the
benchmark's full size through properties that do not depend on size (mass
conservation on a periodic grid, run-to-run determinism, graph == stream).
"""
import numpy as np
import pytest

from sams_b200 import lare
from tests.golden.make_golden import CASES, GEO_DOMAIN, STATE, apply_options, load

pytestmark = pytest.mark.gpu


def _solver(case, nx, ny, nz, seed=1, b0=0.0, rke=0, options=None):
    p, b = lare.case_setup(case, nx, ny, nz, b0)
    p.rke = rke
    if options:
        apply_options(p, options, b)
    s = lare.LARE3D(p, b)
    s.upload_all(lare.case_fields(case, p, seed=seed, b0=b0))
    return s


def _assert_state_equal(s, ref_field, label):
    for f in STATE:
        ref = ref_field(f)
        m = ~np.isnan(ref)
        got = s.download(f)
        if not np.array_equal(got[m], ref[m]):
            diff = np.abs(got[m] - ref[m])
            rel = diff.max() / max(np.abs(ref[m]).max(), 1e-300)
            raise AssertionError(f"{label}: {f} differs, max abs {diff.max():.3e}, rel {rel:.3e}")


@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_gpu_matches_reference_golden(name):
    z, meta = load(name)
    s = _solver(meta["case"], meta["nx"], meta["ny"], meta["nz"], meta["seed"], meta["b0"], options=meta)
    dts = []
    for _ in range(meta["steps"]):
        s.step(1)
        dts.append(s.dt)
    assert np.array_equal(np.array(dts), z["dts"]), (dts, z["dts"])
    _assert_state_equal(s, lambda f: z[f], name)
    assert s.steps == meta["steps"]
    assert s.time == pytest.approx(meta["time"], rel=0, abs=0)


@pytest.mark.parametrize("case,n,steps", [
    ("ot", (24, 20, 8), 30),
    ("ot", (33, 17, 5), 10),
    ("rf", (16, 16, 16), 10),
    ("rf", (20, 12, 9), 6),
    ("harris", (24, 16, 8), 10),
    ("rf", (8, 8, 2), 5),          # fewer than three cells in z: ordered edge copies
    ("ot", (2, 9, 5), 5),          # ... in x
    ("harris", (12, 1, 6), 4),     # ... one cell in y, walls
    # z lines long enough for the fused out-of-place x / y sweep kernel
    ("rf", (12, 10, 24), 4),
    ("harris", (10, 12, 28), 3),
    ("ot", (9, 7, 26), 4),
    ("ot", (2, 9, 24), 4),         # ... with fewer than three cells along the sweep
    ("rf", (8, 2, 26), 3),
])
def test_gpu_matches_checker(case, n, steps, oracle_lib):
    lo = oracle_lib
    nx, ny, nz = n
    s = _solver(case, nx, ny, nz, seed=9)
    p, b = lo.case_setup(case, nx, ny, nz)
    o = lo.Oracle(p, b, lo.case_fields(case, p, seed=9))
    for _ in range(steps):
        s.step(1)
        o.step(1)
        assert s.dt == o.dt
    _assert_state_equal(s, lambda f: _masked(o.field(f), f, nx, ny, nz), f"{case}{n}")


def _masked(box, f, nx, ny, nz):
    out = np.full(box.shape, np.nan)
    sl = lare.field_slices(f, nx, ny, nz)
    out[sl] = box[sl]
    return out


def test_gpu_matches_checker_64cube_resistive(oracle_lib):
    lo = oracle_lib
    s = _solver("rf", 64, 64, 64, seed=2)
    p, b = lo.case_setup("rf", 64, 64, 64)
    o = lo.Oracle(p, b, lo.case_fields("rf", p, seed=2))
    s.step(4)
    o.step(4)
    assert s.dt == o.dt
    _assert_state_equal(s, lambda f: _masked(o.field(f), f, 64, 64, 64), "rf64")


def test_graph_equals_stream_and_is_deterministic():
    a = _solver("ot", 32, 32, 4)
    b = _solver("ot", 32, 32, 4)
    a.step(12)
    b.step(12, graph=True)
    a.synchronize()
    b.synchronize()
    for f in STATE:
        assert np.array_equal(a.download(f), b.download(f)), f
    assert a.dt == b.dt and a.time == b.time


def test_full_size_256_cube_conserves_mass_and_is_deterministic():
    """The benchmark configuration (256^3 random field, resistive) at full
    size: total mass sum(rho * cv) over the periodic domain is conserved to
    1e-13 relative, and two solves from the same state agree bit for bit."""
    n = 256
    p, b = lare.case_setup("rf", n, n, n)
    fields = lare.case_fields("rf", p, seed=1)
    cv = (1.0 / n) ** 3
    m0 = fields[0][3:n + 3, 3:n + 3, 3:n + 3].sum() * cv
    runs = []
    for _ in range(2):
        s = lare.LARE3D(p, b)
        s.upload_all(fields)
        s.step(3, graph=True)
        s.synchronize()
        runs.append(s.download("rho"))
        s.close()
    assert np.array_equal(runs[0], runs[1])
    m1 = runs[0][3:n + 3, 3:n + 3, 3:n + 3].sum() * cv
    assert abs(m1 - m0) / m0 < 1e-13


@pytest.mark.parametrize("case,n,steps", [("rf", (20, 16, 12), 5), ("ot", (24, 20, 8), 8), ("harris", (16, 12, 6), 4),
                                          ("ot", (16, 12, 2), 4)])
def test_gpu_matches_checker_with_rke(case, n, steps, oracle_lib):
    """The remap kinetic-energy correction: delta_ke is gathered in the
    reference's serial order, so the GPU equals the checker bit for bit."""
    lo = oracle_lib
    nx, ny, nz = n
    s = _solver(case, nx, ny, nz, seed=4, rke=1)
    p, b = lo.case_setup(case, nx, ny, nz)
    p.rke = 1
    o = lo.Oracle(p, b, lo.case_fields(case, p, seed=4))
    for _ in range(steps):
        s.step(1, graph=True)
        o.step(1)
        assert s.dt == o.dt
    _assert_state_equal(s, lambda f: _masked(o.field(f), f, nx, ny, nz), f"rke {case}{n}")


def test_gpu_resistive_with_inconsistent_energy_ghosts(oracle_lib):
    """Energy ghosts that are not their boundary values at the start (as an
    IC package may leave them): the resistive predictor reads the step-start
    pressures, like the reference, not ones recomputed after the sub-steps
    refill the ghosts."""
    lo = oracle_lib
    n = (12, 10, 8)
    p, b = lare.case_setup("rf", *n)
    fields = lare.case_fields("rf", p, seed=3)
    for f in (1, 2):
        inner = fields[f][3:-2, 3:-2, 3:-2].copy()
        fields[f] *= 1.25
        fields[f][3:-2, 3:-2, 3:-2] = inner
    s = lare.LARE3D(p, b)
    s.upload_all(fields)
    op, ob = lo.case_setup("rf", *n)
    o = lo.Oracle(op, ob, fields)
    for _ in range(3):
        s.step(1)
        o.step(1)
        assert s.dt == o.dt
    _assert_state_equal(s, lambda f: _masked(o.field(f), f, *n), "rf ghosts")


@pytest.mark.parametrize("case,n,steps,geometry,rke", [("ot", (24, 20, 8), 6, 1, 0), ("rf", (16, 12, 10), 4, 2, 0),
                                                       ("harris", (16, 12, 6), 4, 1, 1), ("rf", (12, 10, 2), 3, 2, 1),
                                                       ("rf", (10, 8, 24), 3, 2, 0), ("ot", (12, 8, 25), 3, 1, 0)])
def test_gpu_matches_checker_in_curvilinear_geometry(case, n, steps, geometry, rke, oracle_lib):
    """Cylindrical and spherical geometry (metric factors on r in [1, 2],
    theta in [0.5, 1.5]) against the checker, bit for bit."""
    lo = oracle_lib
    nx, ny, nz = n
    opts = {"geometry": geometry, "rke": rke, "domain": GEO_DOMAIN}
    s = _solver(case, nx, ny, nz, seed=6, options=opts)
    p, b = lo.case_setup(case, nx, ny, nz)
    apply_options(p, opts)
    o = lo.Oracle(p, b, lo.case_fields(case, p, seed=6))
    for _ in range(steps):
        s.step(1, graph=True)
        o.step(1)
        assert s.dt == o.dt
    _assert_state_equal(s, lambda f: _masked(o.field(f), f, nx, ny, nz), f"geometry {geometry} {case}{n}")


# The LARE BC_OTHER conditions (walls at the x edges for the velocities,
# plane copies elsewhere) on every edge, as the reference's
# LARE3DInitialConditions package installs them, against the C restatement
# (itself pinned to the reference's own run of that package by the
# *_lare_* fixtures): sizes with fused x / y sweeps (nz >= 24), 2.5-D and a
# power-of-two grid.
@pytest.mark.parametrize("case,n,steps", [
    ("ot", (20, 16, 8), 8), ("rf", (12, 10, 26), 4), ("harris", (10, 12, 28), 3),
    ("ot", (16, 12, 2), 4), ("rf", (16, 16, 16), 4),
])
def test_gpu_lare_other_bcs_match_checker(case, n, steps, oracle_lib):
    lo = oracle_lib
    nx, ny, nz = n
    opts = {"lare_bcs": 1}
    s = _solver(case, nx, ny, nz, seed=5, options=opts)
    p, b = lo.case_setup(case, nx, ny, nz)
    apply_options(p, opts, b)
    o = lo.Oracle(p, b, lo.case_fields(case, p, seed=5))
    for _ in range(steps):
        s.step(1)
        o.step(1)
        assert s.dt == o.dt
    _assert_state_equal(s, lambda f: _masked(o.field(f), f, nx, ny, nz), f"lare bcs {case}{n}")
    s.close()


@pytest.mark.parametrize("n,j_max", [((16, 12, 24), 0.5), ((16, 12, 24), 1.0), ((12, 10, 6), 2.0)])
def test_gpu_matches_checker_with_current_dependent_eta(n, j_max, oracle_lib):
    """eta = eta_bg + eta0 where |J| > j_max (lagran.cpp:445-476), on a grid
    with the fused resistive march (nz = 24) and a thin one, against the
    checker bit for bit.  (The configurations use eta0 = 0, where the
    kernels skip |J|'s square root.)"""
    lo = oracle_lib
    nx, ny, nz = n
    p, b = lare.case_setup("rf", nx, ny, nz)
    p.eta0, p.j_max = 2e-3, j_max
    s = lare.LARE3D(p, b)
    s.upload_all(lare.case_fields("rf", p, seed=9))
    po, bo = lo.case_setup("rf", nx, ny, nz)
    po.eta0, po.j_max = 2e-3, j_max
    o = lo.Oracle(po, bo, lo.case_fields("rf", po, seed=9))
    for _ in range(4):
        s.step(1, graph=True)
        o.step(1)
        assert s.dt == o.dt
    _assert_state_equal(s, lambda f: _masked(o.field(f), f, nx, ny, nz), f"rf{n} j_max {j_max}")
