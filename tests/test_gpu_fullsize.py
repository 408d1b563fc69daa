"""The benchmark configurations at their full sizes, bit for bit against the
CPU checker (oracle/lare_oracle.c, itself pinned to the reference):

  C0  Orszag-Tang 128 x 128 x 4, all 200 steps of the configuration
  C1  random-field cube 256^3, resistive (the throughput benchmark), 2 steps
  C2  Harris sheet 512 x 256 x 64 with conducting y walls, resistive, 2 steps

plus the total energy budget (internal + kinetic + magnetic) within 1e-10
relative of the checker's.  The checker runs on the host's cores (seconds per
step at 256^3), so these are the slowest GPU tests.
"""
import numpy as np
import pytest

from sams_b200 import lare

pytestmark = pytest.mark.gpu

STATE = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz", "bx", "by", "bz"]


def _interior(a, n):
    nx, ny, nz = n
    return a[3:nx + 3, 3:ny + 3, 3:nz + 3]


def energy_budget(get, p):
    """Internal, kinetic and magnetic energy over the interior cells of a
    Cartesian grid (cell volume dx dy dz).  Velocities are node values (the
    cell's upper corner), B the average of a cell's two faces."""
    n = (p.nx, p.ny, p.nz)
    dv = ((p.x_max - p.x_min) / p.nx) * ((p.y_max - p.y_min) / p.ny) * ((p.z_max - p.z_min) / p.nz)
    rho = _interior(get("rho"), n)
    internal = (rho * (_interior(get("energy_electron"), n) + _interior(get("energy_ion"), n))).sum() * dv
    v2 = sum(_interior(get(c), n) ** 2 for c in ("vx", "vy", "vz"))
    kinetic = 0.5 * (rho * v2).sum() * dv
    bx, by, bz = get("bx"), get("by"), get("bz")
    nx, ny, nz = n
    bxc = 0.5 * (bx[3:nx + 3, 3:ny + 3, 3:nz + 3] + bx[2:nx + 2, 3:ny + 3, 3:nz + 3])
    byc = 0.5 * (by[3:nx + 3, 3:ny + 3, 3:nz + 3] + by[3:nx + 3, 2:ny + 2, 3:nz + 3])
    bzc = 0.5 * (bz[3:nx + 3, 3:ny + 3, 3:nz + 3] + bz[3:nx + 3, 3:ny + 3, 2:nz + 2])
    magnetic = ((bxc ** 2 + byc ** 2 + bzc ** 2) / (2.0 * p.mu0)).sum() * dv
    return internal, kinetic, magnetic


def _run_both(oracle_lib, case, n, steps, seed):
    lo = oracle_lib
    p, b = lare.case_setup(case, *n)
    fields = lare.case_fields(case, p, seed=seed)
    s = lare.LARE3D(p, b)
    s.upload_all(fields)
    op, ob = lo.case_setup(case, *n)
    o = lo.Oracle(op, ob, fields)
    del fields
    dts_gpu, dts_cpu = [], []
    for _ in range(steps):
        s.step(1, graph=True)
        dts_gpu.append(s.dt)
        o.step(1)
        dts_cpu.append(o.dt)
    return s, o, p, dts_gpu, dts_cpu


def _check(s, o, p, dts_gpu, dts_cpu, label):
    assert dts_gpu == dts_cpu, label
    n = (p.nx, p.ny, p.nz)
    for f in STATE:
        sl = lare.field_slices(f, *n)
        got, want = s.download(f)[sl], o.field(f)[sl]
        if not np.array_equal(got, want):
            d = np.abs(got - want).max()
            raise AssertionError(f"{label}: {f} differs (max abs {d:.3e})")
    eg = energy_budget(s.download, p)
    ec = energy_budget(o.field, p)
    for name, a, c in zip(("internal", "kinetic", "magnetic"), eg, ec):
        assert abs(a - c) <= 1e-10 * abs(c), (label, name, a, c)
    assert abs(sum(eg) - sum(ec)) <= 1e-10 * abs(sum(ec)), label


def test_c0_orszag_tang_all_200_steps(oracle_lib):
    s, o, p, dg, dc = _run_both(oracle_lib, "ot", (128, 128, 4), 200, 1)
    _check(s, o, p, dg, dc, "C0 ot 128x128x4 x200")
    assert s.steps == 200 and s.time == o.time
    s.close()


def test_c1_random_field_256_cube(oracle_lib):
    s, o, p, dg, dc = _run_both(oracle_lib, "rf", (256, 256, 256), 2, 1)
    _check(s, o, p, dg, dc, "C1 rf 256^3 x2")
    s.close()


def test_c2_harris_512x256x64(oracle_lib):
    s, o, p, dg, dc = _run_both(oracle_lib, "harris", (512, 256, 64), 2, 1)
    _check(s, o, p, dg, dc, "C2 harris 512x256x64 x2")
    s.close()
