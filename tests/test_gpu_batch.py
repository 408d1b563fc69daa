"""Batched solves: every solve in a batch must give exactly what it gives
alone (same kernels, same per-solve dt), through adds, removes and tuning."""
import numpy as np
import pytest

from sams_b200 import lare
from tests.golden.make_golden import GEO_DOMAIN, apply_options

pytestmark = pytest.mark.gpu

STATE = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz", "bx", "by", "bz"]

MIX = [("ot", (16, 12, 4), 1, 0.0), ("ot", (24, 24, 4), 2, 0.9 / (4 * np.pi) ** 0.5),
       ("rf", (12, 12, 12), 3, 0.0), ("harris", (16, 12, 6), 4, 0.0), ("ot", (40, 8, 5), 5, 0.0),
       ("ot", (20, 16, 2), 6, 0.0), ("rf", (10, 2, 8), 7, 0.0)]


def _solo(case, n, seed, b0, steps, rke=0, geometry=0):
    p, b = lare.case_setup(case, *n, b0)
    p.rke = rke
    if geometry:
        apply_options(p, {"geometry": geometry, "domain": GEO_DOMAIN})
    s = lare.LARE3D(p, b)
    s.upload_all(lare.case_fields(case, p, seed=seed, b0=b0))
    s.step(steps)
    out = {f: s.download(f) for f in STATE}
    st = (s.dt, s.time, s.steps)
    s.close()
    return out, st


def _add(batch, case, n, seed, b0, rke=0, geometry=0):
    p, b = lare.case_setup(case, *n, b0)
    p.rke = rke
    if geometry:
        apply_options(p, {"geometry": geometry, "domain": GEO_DOMAIN})
    return batch.add(p, b, lare.case_fields(case, p, seed=seed, b0=b0))


def _check_equal(batch, sid, case, n, ref, ref_state):
    dt, tm, st = batch.state(sid)
    assert (dt, tm, st) == ref_state, (case, n)
    for f in STATE:
        sl = lare.field_slices(f, *n)
        got = batch.download(sid, f)[sl]
        assert np.array_equal(got, ref[f][sl]), f"{case}{n}: {f}"


@pytest.mark.parametrize("graph", [False, True])
def test_batch_equals_solo(graph):
    steps = 6
    bt = lare.Batch()
    ids = [_add(bt, *m) for m in MIX]
    bt.step(steps, graph=graph)
    bt.synchronize()
    for sid, (case, n, seed, b0) in zip(ids, MIX):
        ref, st = _solo(case, n, seed, b0, steps)
        _check_equal(bt, sid, case, n, ref, st)
    bt.close()


def test_batch_add_remove_midrun_and_autotune_restores():
    bt = lare.Batch()
    a = _add(bt, *MIX[0])
    b = _add(bt, *MIX[2])
    bt.step(3, graph=True)
    bt.remove(a)                       # a leaves after 3 steps
    c = _add(bt, *MIX[3])              # c joins (fresh)
    before = {f: bt.download(b, f) for f in STATE}
    state_b = bt.state(b)
    tile, bps, ms = bt.autotune(trial_steps=1)
    assert tile in (1, 2, 4, 8) and bps in (2, 4, 8) and ms > 0
    assert bt.state(b) == state_b
    for f in STATE:
        assert np.array_equal(bt.download(b, f), before[f]), f
    bt.step(4, graph=True)
    bt.synchronize()
    ref_b, st_b = _solo(*MIX[2], steps=7)
    _check_equal(bt, b, MIX[2][0], MIX[2][1], ref_b, st_b)
    ref_c, st_c = _solo(*MIX[3], steps=4)
    _check_equal(bt, c, MIX[3][0], MIX[3][1], ref_c, st_c)
    bt.close()


def test_batch_mixing_rke_and_plain_solves_equals_solo():
    """Solves with and without the remap kinetic-energy correction share a
    batch: the correction's launches run for the batch and leave the others'
    state alone."""
    mix = [("rf", (12, 12, 12), 3, 0.0, 1), ("ot", (24, 24, 4), 2, 0.0, 0), ("harris", (16, 12, 6), 4, 0.0, 1),
           ("ot", (20, 16, 2), 6, 0.0, 1)]
    bt = lare.Batch()
    ids = [_add(bt, *m) for m in mix]
    bt.step(5, graph=True)
    bt.synchronize()
    for sid, (case, n, seed, b0, rke) in zip(ids, mix):
        ref, st = _solo(case, n, seed, b0, 5, rke)
        _check_equal(bt, sid, case, n, ref, st)
    bt.close()


def test_batch_mixing_geometries_equals_solo():
    """Cartesian, cylindrical and spherical solves in one batch."""
    mix = [("ot", (20, 16, 4), 1, 0.0, 0, 1), ("rf", (12, 10, 8), 2, 0.0, 0, 2), ("ot", (16, 12, 4), 3, 0.0, 1, 0),
           ("harris", (12, 10, 6), 4, 0.0, 0, 1)]
    bt = lare.Batch()
    ids = [_add(bt, *m) for m in mix]
    bt.step(4, graph=True)
    bt.synchronize()
    for sid, (case, n, seed, b0, rke, geo) in zip(ids, mix):
        ref, st = _solo(case, n, seed, b0, 4, rke, geo)
        _check_equal(bt, sid, case, n, ref, st)
    bt.close()


def test_batch_with_lare_other_bcs_equals_solo():
    """Solves whose every edge carries the LARE BC_OTHER conditions, batched
    with periodic ones: each equals its solo run."""
    mix = [("ot", (16, 12, 4), 1, 0.0, True), ("rf", (12, 12, 12), 3, 0.0, True),
           ("ot", (20, 16, 2), 6, 0.0, True), ("ot", (24, 24, 4), 2, 0.0, False)]
    steps = 5
    bt = lare.Batch()
    ids, refs = [], []
    for case, n, seed, b0, lbc in mix:
        opts = {"lare_bcs": 1} if lbc else {}
        p, b = lare.case_setup(case, *n, b0)
        apply_options(p, opts, b)
        ids.append(bt.add(p, b, lare.case_fields(case, p, seed=seed, b0=b0)))
        s = lare.LARE3D(p, b)
        s.upload_all(lare.case_fields(case, p, seed=seed, b0=b0))
        s.step(steps)
        refs.append(({f: s.download(f) for f in STATE}, (s.dt, s.time, s.steps)))
        s.close()
    bt.step(steps, graph=True)
    bt.synchronize()
    for sid, (case, n, seed, b0, lbc), (ref, st) in zip(ids, mix, refs):
        _check_equal(bt, sid, case, n, ref, st)
    bt.close()



def test_config3_batch_equals_each_plain_run():
    """The batched workload at its configured size: 64 Orszag-Tang solves
    n x n x 4, n = round(64 * 8^u) (u seeded), B0 uniform in [0.5, 1.5]/sqrt(4 pi),
    3 batched steps; every solve equals its own plain run bit for bit."""
    import math
    rng = np.random.default_rng(2024)
    ns = [int(round(64 * 8 ** u)) for u in rng.random(64)]
    b0s = rng.uniform(0.5, 1.5, 64) / math.sqrt(4 * math.pi)
    steps = 3
    bt = lare.Batch()
    ids = [_add(bt, "ot", (n, n, 4), 1, b0) for n, b0 in zip(ns, b0s)]
    bt.step(steps, graph=True)
    bt.synchronize()
    for sid, n, b0 in zip(ids, ns, b0s):
        ref, st = _solo("ot", (n, n, 4), 1, b0, steps)
        _check_equal(bt, sid, "ot", (n, n, 4), ref, st)
    bt.close()
