"""The single-solve benchmark configurations at their full sizes AND full
stated step counts, against records written by the reference itself
(tests/golden/make_longrun.py, tests/golden/longrun.py):

  C0  Orszag-Tang 128 x 128 x 4, 200 steps
  C1  random-field cube 256^3, resistive (the throughput benchmark), 500 steps
  C2  Harris sheet 512 x 256 x 64, conducting y walls, resistive, 1000 steps

Each run steps on the GPU one graph step at a time (reading dt back after
each, as the runner's step log does), then checks the dt history, every
state field's SHA-256 over its own index range (bit-identical), the samples
(reported within the 1e-10 relative L-infinity tolerance when a hash
differs), mass conservation to 1e-13 relative (C0, C1: periodic in every
dimension) and the energy budget to 1e-10 of the reference's.  The late
steps are where the limiter branches, the small-velocity branch of the
edge viscosity (dv dt / dx < 1e-14) and, in C2, the walls under a developed
current sheet come into play.
"""
import os
import sys

import numpy as np
import pytest

from sams_b200 import lare

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import longrun as lr  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative L-infinity for the sample report
MASS_TOL = 1e-13


def _run(name):
    meta, fields = lr.load(name)
    case, nx, ny, nz, steps, seed = (meta[k] for k in ("case", "nx", "ny", "nz", "steps", "seed"))
    p, b = lare.case_setup(case, nx, ny, nz)
    ic = lare.case_fields(case, p, seed=seed)
    dv = ((p.x_max - p.x_min) / nx) * ((p.y_max - p.y_min) / ny) * ((p.z_max - p.z_min) / nz)
    m0 = lr.mass(ic[0], nx, ny, nz, dv)
    s = lare.LARE3D(p, b)
    s.upload_all(ic)
    del ic
    dts = []
    for _ in range(steps):
        s.step(1, graph=True)
        dts.append(s.dt)
    s.synchronize()
    return meta, fields, p, s, dts, m0, dv


def _check(name, periodic):
    meta, fields, p, s, dts, m0, dv = _run(name)
    nx, ny, nz = meta["nx"], meta["ny"], meta["nz"]
    try:
        assert s.steps == meta["steps"] and s.time == meta["time"], (s.steps, s.time, meta["time"])
        first = next((i for i, (a, c) in enumerate(zip(dts, meta["dts"])) if a != c), None)
        assert first is None, f"{name}: dt differs first at step {first + 1}: {dts[first]!r} vs {meta['dts'][first]!r}"
        boxes = {}
        diffs = []
        for f in lr.STATE:
            boxes[f] = s.download(f)
            local = boxes[f][lare.field_slices(f, nx, ny, nz)]
            h, idx, want = fields[f]
            got = local[tuple(idx)]
            if lr.digest(local) != h:
                scale = max(np.abs(want).max(), np.finfo(float).tiny)
                rel = np.abs(got - want).max() / scale
                diffs.append(f"{f}: hash differs, sampled rel L-inf {rel:.3e} ({'within' if rel <= TOL else 'beyond'} {TOL})")
            else:
                assert np.array_equal(got, want), f"{name} {f}: hash equal but samples differ"
        assert not diffs, f"{name}: " + "; ".join(diffs)
        eb = lr.energy_budget(lambda f: boxes[f], nx, ny, nz, dv, p.mu0)
        for k, v in zip(("internal", "kinetic", "magnetic"), eb):
            ref = meta["energy"][k]
            assert abs(v - ref) <= TOL * abs(ref), (name, k, v, ref)
        m1 = lr.mass(boxes["rho"], nx, ny, nz, dv)
        assert m1 == meta["mass_final"] or abs(m1 - meta["mass_final"]) <= MASS_TOL * abs(m0), (m1, meta["mass_final"])
        if periodic:
            assert abs(m1 - m0) <= MASS_TOL * abs(m0), f"{name}: mass drift {(m1 - m0) / m0:.3e}"
    finally:
        s.close()


def test_c0_orszag_tang_200_steps_against_reference_record():
    _check("c0_ot_128x128x4_s200", periodic=True)


def test_c1_random_field_256_cube_500_steps_against_reference_record():
    _check("c1_rf_256cube_s500", periodic=True)


def test_c2_harris_1000_steps_against_reference_record():
    _check("c2_harris_512x256x64_s1000", periodic=False)
