"""Serving on several GPUs through the router: solves placed on different
servers must each equal the same solve run alone, bit for bit, and the
placement must spread a burst.  One GPU is enough to check this: the router
is given the same device twice, i.e. two independent servers (threads,
streams, budgets) on one GPU; their kernels never wait on each other."""
import time

import numpy as np
import pytest

from sams_b200 import lare

pytestmark = pytest.mark.gpu

STATE = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz", "bx", "by", "bz"]
REQS = [("rf", (16, 16, 16), 12, 1), ("rf", (20, 16, 12), 9, 2), ("ot", (32, 24, 4), 15, 3),
        ("harris", (24, 16, 8), 10, 4), ("rf", (24, 24, 24), 7, 5), ("ot", (48, 16, 6), 5, 6)]


def _solo(case, n, steps, seed):
    p, b = lare.case_setup(case, *n)
    s = lare.LARE3D(p, b)
    s.upload_all(lare.case_fields(case, p, seed=seed))
    s.step(steps)
    out = {f: s.download(f) for f in STATE}
    s.close()
    return out


def test_routed_results_equal_solo_and_spread():
    rt = lare.Router(1 << 30, devices=(0, 0))
    tickets, outs = [], []
    for case, n, steps, seed in REQS:
        p, b = lare.case_setup(case, *n)
        out = [np.zeros(lare.box_shape(*n)) for _ in range(9)]
        tickets.append(rt.submit(p, b, lare.case_fields(case, p, seed=seed), steps, out))
        outs.append(out)
        time.sleep(0.005)
    placed = [rt.placement(t) for t in tickets]
    assert set(placed) == {0, 1}
    rt.drain(300)
    st = rt.stats()
    assert st["completed"] == len(REQS) and st["failed"] == 0
    assert st["pending_cell_updates"] == 0 and st["queued_bytes"] == 0
    per = [rt.server_stats(q)["completed"] for q in range(2)]
    assert sum(per) == len(REQS) and min(per) >= 1
    for t, out, (case, n, steps, seed) in zip(tickets, outs, REQS):
        assert rt.poll(t)[0] == "done"
        ref = _solo(case, n, steps, seed)
        for q, f in enumerate(STATE):
            sl = lare.field_slices(f, *n)
            assert np.array_equal(out[q][sl], ref[f][sl]), f"{case}{n} {f}"
    rt.close()


def test_router_fetch_cancel_release():
    rt = lare.Router(1 << 30, devices=(0, 0))
    p, b = lare.case_setup("rf", 12, 12, 12)
    keep = rt.submit(p, b, lare.case_fields("rf", p, seed=2), 6)      # result kept by its server
    long_ = rt.submit(p, b, lare.case_fields("rf", p, seed=3), 100000)
    rt.cancel(long_)
    rt.drain(300)
    assert rt.poll(long_)[0] == "cancelled"
    assert rt.poll(keep)[0] == "done"
    ref = _solo("rf", (12, 12, 12), 6, 2)
    for q, f in enumerate(STATE):
        sl = lare.field_slices(f, 12, 12, 12)
        assert np.array_equal(rt.fetch(keep, q)[sl], ref[f][sl]), f
    rt.release(keep)
    rt.release(long_)
    with pytest.raises(lare.LareError):
        rt.poll(keep)
    st = rt.stats()
    assert st["completed"] == 1 and st["p50_latency_s"] > 0
    rt.close()
