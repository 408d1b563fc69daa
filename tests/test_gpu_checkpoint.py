"""Checkpoint / restart (sams_lare_save / sams_lare_load, SAMSDUMP1 files).

A run that is saved, reloaded into a fresh solver and continued equals the
run that never stopped, bit for bit (fields, dt, time, step count); the
reference's own state after three steps (tests/golden/ot_12x10x6_at3.dump,
written by tests/golden/make_golden.py from the compiled reference) restarts
on the GPU and reaches the reference's state after five steps; and a GPU
checkpoint reads back with the oracle's dump reader.
"""
import os

import numpy as np
import pytest

from oracle.dumpio import Dump
from sams_b200 import lare
from tests.golden.make_golden import STATE, load

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _solver(case, n, seed):
    p, b = lare.case_setup(case, *n)
    s = lare.LARE3D(p, b)
    s.upload_all(lare.case_fields(case, p, seed=seed))
    return s


@pytest.mark.parametrize("case,n,first,rest", [("rf", (20, 16, 12), 3, 4), ("harris", (24, 16, 8), 2, 3),
                                                ("ot", (16, 12, 2), 1, 3)])
def test_restart_equals_uninterrupted_run(case, n, first, rest, tmp_path):
    a = _solver(case, n, seed=5)
    a.step(first + rest, graph=True)
    b = _solver(case, n, seed=5)
    b.step(first)
    path = str(tmp_path / "ckpt.dump")
    b.save(path)
    b.close()
    p, bc = lare.case_setup(case, *n)
    c = lare.LARE3D(p, bc)                # fresh solver: nothing but the file
    c.load(path)
    assert c.steps == first
    c.step(rest, graph=True)
    assert (c.dt, c.time, c.steps) == (a.dt, a.time, a.steps)
    for f in STATE:
        sl = lare.field_slices(f, *n)
        assert np.array_equal(c.download(f)[sl], a.download(f)[sl]), f
    a.close()
    c.close()


def test_restart_from_the_reference_state():
    z, meta = load("ot_12x10x6_s5")
    p, b = lare.case_setup("ot", 12, 10, 6)
    s = lare.LARE3D(p, b)
    s.load(os.path.join(HERE, "golden", "ot_12x10x6_at3.dump"))
    assert s.steps == 3 and s.dt == z["dts"][2]
    dts = []
    for _ in range(2):
        s.step(1)
        dts.append(s.dt)
    assert np.array_equal(np.array(dts), z["dts"][3:5])
    for f in STATE:
        ref = z[f]
        m = ~np.isnan(ref)
        assert np.array_equal(s.download(f)[m], ref[m]), f
    assert s.time == meta["time"]
    s.close()


def test_checkpoint_reads_back_with_the_oracle_reader(tmp_path):
    n = (14, 10, 6)
    s = _solver("rf", n, seed=8)
    s.step(2)
    path = str(tmp_path / "c.dump")
    s.save(path)
    d = Dump(path)
    assert d.header["step"] == 2 and d.header["dt"] == s.dt and d.header["time"] == s.time
    for f in STATE + ["vx1", "vy1", "vz1", "dm"]:
        sl = lare.field_slices(f, *n)
        assert np.array_equal(d.box(f)[sl], s.download(f)[sl]), f
    s.close()


def test_load_rejects_other_grids_and_bad_files(tmp_path):
    s = _solver("ot", (12, 10, 6), seed=1)
    other = str(tmp_path / "other.dump")
    t = _solver("ot", (12, 10, 4), seed=1)
    t.save(other)
    t.close()
    with pytest.raises(lare.LareError) as e:
        s.load(other)
    assert e.value.status == -1
    bad = tmp_path / "bad.dump"
    bad.write_bytes(b"not a dump\n")
    with pytest.raises(lare.LareError):
        s.load(str(bad))
    with pytest.raises(lare.LareError):
        s.load(str(tmp_path / "missing.dump"))
    s.close()
