"""The CPU checker (oracle/lare_oracle.c) against the reference.

Golden fixtures in tests/golden/ were produced by the reference itself
(tests/golden/make_golden.py runs the compiled reference LARE3D); where the
reference binary is present (this build container) the checker is also
compared with it directly on further cases.  The bar is bit-for-bit.
"""
import os

import numpy as np
import pytest

from oracle import lare_oracle as lo
from tests.golden.make_golden import CASES, GEO_DOMAIN, STATE, apply_options, load


def _run_checker(case, nx, ny, nz, steps, seed, b0, options=None):
    p, b = lo.case_setup(case, nx, ny, nz, b0)
    apply_options(p, options or {}, b)
    o = lo.Oracle(p, b, lo.case_fields(case, p, seed=seed, b0=b0))
    dts = []
    for _ in range(steps):
        o.step(1)
        dts.append(o.dt)
    return o, dts


@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_checker_matches_reference_golden(name, oracle_lib):
    z, meta = load(name)
    o, dts = _run_checker(meta["case"], meta["nx"], meta["ny"], meta["nz"], meta["steps"], meta["seed"], meta["b0"],
                          meta)
    assert np.array_equal(np.array(dts), z["dts"]), "dt history differs"
    for f in STATE:
        ref = z[f]
        m = ~np.isnan(ref)
        got = o.field(f)
        assert np.array_equal(got[m], ref[m]), f"{name}: field {f} differs (max {np.abs(got[m]-ref[m]).max()})"


@pytest.mark.skipif(not os.path.exists(lo.REF_BIN), reason="reference harness binary not built here")
@pytest.mark.parametrize("case,n,steps,rke,geometry", [
    ("ot", (9, 11, 5), 12, 0, 0), ("rf", (8, 8, 8), 6, 0, 0), ("harris", (10, 8, 4), 6, 0, 0),
    ("rf", (8, 8, 2), 3, 0, 0), ("ot", (2, 9, 5), 3, 0, 0), ("ot", (9, 11, 5), 6, 1, 0),
    ("harris", (10, 8, 4), 4, 1, 0), ("ot", (9, 11, 5), 6, 0, 1), ("rf", (8, 6, 6), 3, 0, 2),
    ("harris", (10, 8, 4), 3, 1, 2)])
def test_checker_matches_reference_binary(case, n, steps, rke, geometry, tmp_path, oracle_lib):
    """rke = 1: the reference on one thread (its atomic adds in loop order);
    geometry 1/2: cylindrical/spherical on r in [1, 2], theta in [0.5, 1.5]."""
    from oracle.dumpio import Dump
    nx, ny, nz = n
    dump = str(tmp_path / "ref.dump")
    extra = (["--rke"] if rke else []) + (["--geometry", str(geometry), "--domain"] + [repr(x) for x in GEO_DOMAIN]
                                           if geometry else [])
    lo.run_reference(case, nx, ny, nz, steps, dump, seed=11, extra=extra, threads=1 if rke else None)
    d = Dump(dump)
    opts = {"rke": rke, "geometry": geometry, "domain": GEO_DOMAIN if geometry else None}
    o, dts = _run_checker(case, nx, ny, nz, steps, 11, 0.0, opts)
    assert dts == d.header["dts"]
    for f in lo.FIELD_NAMES:
        ref = d.box(f)
        m = ~np.isnan(ref)
        assert np.array_equal(o.field(f)[m], ref[m]), f
    # grid metrics as LARE3D::grid builds them
    for name in ["cv", "cvc", "dxab", "dyab", "dzab", "dxac", "dyac", "dzac"]:
        ref = d.box(name)
        m = ~np.isnan(ref)
        assert np.array_equal(o.named(name)[m], ref[m]), name


def test_planted_error_is_caught(oracle_lib):
    """A mistake planted in the checker's input state must show up in the
    comparison (guards against a vacuous test)."""
    z, meta = load("ot_12x10x6_s5")
    p, b = lo.case_setup("ot", meta["nx"], meta["ny"], meta["nz"])
    fields = lo.case_fields("ot", p)
    fields[0][7, 7, 4] *= 1.0 + 1e-12
    o = lo.Oracle(p, b, fields)
    o.step(meta["steps"])
    ref = z["rho"]
    m = ~np.isnan(ref)
    assert not np.array_equal(o.field("rho")[m], ref[m])


def test_periodic_mass_conservation_checker(oracle_lib):
    p, b = lo.case_setup("ot", 16, 16, 4)
    o = lo.Oracle(p, b, lo.case_fields("ot", p))
    cv = o.named("cv")[3:-2, 3:-2, 3:-2]
    m0 = (o.field("rho")[3:-2, 3:-2, 3:-2] * cv).sum()
    o.step(20)
    m1 = (o.field("rho")[3:-2, 3:-2, 3:-2] * cv).sum()
    assert abs(m1 - m0) / m0 < 1e-13


@pytest.mark.skipif(not os.path.exists(lo.REF_BIN), reason="reference harness binary not built here")
def test_checker_matches_reference_with_inconsistent_ghosts(tmp_path, oracle_lib):
    """Initial energies whose ghost cells are not their boundary values (an IC
    package may fill ghosts analytically): in a resistive run the predictor
    must use the pressures of the step's start, before the sub-steps refill
    the energies' ghosts."""
    from oracle.dumpio import Dump
    n = (10, 8, 6)
    p, b = lo.case_setup("rf", *n)
    fields = lo.case_fields("rf", p, seed=3)
    for f in (1, 2):  # e_e, e_i: ghosts scaled, interior untouched
        inner = fields[f][3:-2, 3:-2, 3:-2].copy()
        fields[f] *= 1.25
        fields[f][3:-2, 3:-2, 3:-2] = inner
    ic = tmp_path / "ic.bin"
    with open(ic, "wb") as fh:
        for a in fields:
            fh.write(np.ascontiguousarray(a).tobytes())
    dump = str(tmp_path / "ref.dump")
    lo.run_reference("rf", *n, 3, dump, ic=str(ic))
    d = Dump(dump)
    o = lo.Oracle(p, b, fields)
    dts = []
    for _ in range(3):
        o.step(1)
        dts.append(o.dt)
    assert dts == d.header["dts"]
    for f in lo.FIELD_NAMES:
        ref = d.box(f)
        m = ~np.isnan(ref)
        assert np.array_equal(o.field(f)[m], ref[m]), f


def test_longrun_records_are_complete():
    """The long-run records written from the reference (tests/golden/*.longrun.npz)
    cover every single-solve configuration at its stated step count."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import longrun as lr
    for name, case, nx, ny, nz, steps, seed in lr.RUNS:
        meta, fields = lr.load(name)
        got = (meta["case"], meta["nx"], meta["ny"], meta["nz"], meta["steps"], meta["seed"])
        assert got == (case, nx, ny, nz, steps, seed)
        assert len(meta["dts"]) == steps and set(fields) == set(lr.STATE)
        assert all(len(h) == 64 and len(v) == lr.NSAMPLES for h, _, v in fields.values())
