"""Serving: continuous batching under a device-memory budget.  Solves that
arrive while others run are admitted when memory frees up and stepped in
the same batch; each result must equal the same solve run alone, bit for
bit.  A solve that goes non-finite fails alone."""
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


@pytest.mark.parametrize("budget_mb,max_cells", [(4096, 0), (60, 0), (4096, 9000)])
def test_served_results_equal_solo(budget_mb, max_cells):
    """budget 4 GB: everything runs concurrently; 60 MB: admissions wait for
    earlier solves to finish (continuous batching under a tight budget);
    a 9000-cell cap: at most two of these solves run at once, in arrival
    order (the 13824-cell one runs alone)."""
    srv = lare.Server(budget_mb << 20, max_cells=max_cells)
    tickets = []
    outs = []
    for case, n, steps, seed in REQS:
        p, b = lare.case_setup(case, *n)
        out = [np.zeros(lare.box_shape(*n)) for _ in range(9)]
        tickets.append(srv.submit(p, b, lare.case_fields(case, p, seed=seed), steps, out))
        outs.append(out)
        time.sleep(0.01)  # staggered arrivals
    srv.drain(300)
    st = srv.stats()
    assert st["completed"] == len(REQS) and st["failed"] == 0
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0
    for t, out, (case, n, steps, seed) in zip(tickets, outs, REQS):
        assert srv.poll(t)[0] == "done"
        ref = _solo(case, n, steps, seed)
        for q, f in enumerate(STATE):
            sl = lare.field_slices(f, *n)
            assert np.array_equal(out[q][sl], ref[f][sl]), f"{case}{n} {f}"
    srv.close()


def test_failed_solve_is_isolated_and_kept_results_fetchable():
    srv = lare.Server(1 << 30)
    p, b = lare.case_setup("rf", 12, 12, 12)
    bad = lare.case_fields("rf", p, seed=1)
    bad[0][:] = 0.0                       # zero density: the CFL timestep is not finite
    tb = srv.submit(p, b, bad, 70)
    good = srv.submit(p, b, lare.case_fields("rf", p, seed=2), 8)  # result kept by the server
    srv.drain(300)
    assert srv.poll(tb)[0] == "failed"
    assert srv.poll(good)[0] == "done"
    ref = _solo("rf", (12, 12, 12), 8, 2)
    for q, f in enumerate(STATE):
        sl = lare.field_slices(f, 12, 12, 12)
        assert np.array_equal(srv.fetch(good, q)[sl], ref[f][sl]), f
    srv.release(good)
    srv.close()
    tiny = lare.Server(1 << 20)           # 1 MB: a 16^3 solve can never fit
    p16, b16 = lare.case_setup("rf", 16, 16, 16)
    with pytest.raises(lare.LareError) as e:
        tiny.submit(p16, b16, lare.case_fields("rf", p16), 1)
    assert e.value.status == -7
    tiny.close()


def test_cancel_queued_and_running_requests():
    """A cap of one running 16^3 solve: the first request runs long, the
    next two wait.  Cancelling the running one and one queued one leaves the
    last to run alone, and its result still equals its solo run."""
    srv = lare.Server(1 << 30, max_cells=16 * 16 * 16)
    p, b = lare.case_setup("rf", 16, 16, 16)
    long_run = srv.submit(p, b, lare.case_fields("rf", p, seed=1), 100000)
    queued = srv.submit(p, b, lare.case_fields("rf", p, seed=2), 5)
    out = [np.zeros(lare.box_shape(16, 16, 16)) for _ in range(9)]
    last = srv.submit(p, b, lare.case_fields("rf", p, seed=3), 6, out)
    for _ in range(2000):
        if srv.poll(long_run)[0] == "running":
            break
        time.sleep(0.005)
    assert srv.poll(queued)[0] == "queued"
    srv.cancel(queued)
    assert srv.poll(queued)[0] == "cancelled"
    srv.cancel(long_run)
    srv.drain(300)
    assert srv.poll(long_run)[0] == "cancelled"
    assert srv.poll(last)[0] == "done"
    ref = _solo("rf", (16, 16, 16), 6, 3)
    for q, f in enumerate(STATE):
        sl = lare.field_slices(f, 16, 16, 16)
        assert np.array_equal(out[q][sl], ref[f][sl]), f
    with pytest.raises(lare.LareError):
        srv.cancel(last)              # already finished
    for t in (long_run, queued, last):
        srv.release(t)
    srv.close()


def test_served_mix_with_a_192_cube_equals_solo():
    """A config-4-shaped mix (random-field cubes, resistive, one of edge 192)
    arriving while others run, under a cell cap that makes the 192^3 solve
    wait for room: each result equals its solo run bit for bit."""
    reqs = [("rf", (64, 64, 64), 6, 11), ("rf", (192, 192, 192), 4, 12), ("rf", (32, 32, 32), 9, 13),
            ("rf", (96, 96, 96), 5, 14)]
    srv = lare.Server(40 << 30, max_cells=8_000_000)
    tickets, outs = [], []
    for case, n, steps, seed in reqs:
        p, b = lare.case_setup(case, *n)
        out = [np.zeros(lare.box_shape(*n)) for _ in range(9)]
        tickets.append(srv.submit(p, b, lare.case_fields(case, p, seed=seed), steps, out))
        outs.append(out)
        time.sleep(0.02)
    srv.drain(600)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for t, out, (case, n, steps, seed) in zip(tickets, outs, reqs):
        assert srv.poll(t)[0] == "done"
        ref = _solo(case, n, steps, seed)
        for q, f in enumerate(STATE):
            sl = lare.field_slices(f, *n)
            assert np.array_equal(out[q][sl], ref[f][sl]), f"{case}{n} {f}"
    srv.close()


def test_own_stream_solves_fail_and_cancel_alone():
    """Solves whose z lines fill the fused kernels (here nz = 24) step on
    their own streams beside the batched ones.  One of them goes non-finite
    and another is cancelled while running: both leave alone, and a fused
    and a batched solve that share the GPU with them still equal their solo
    runs bit for bit."""
    srv = lare.Server(4 << 30)
    p24, b24 = lare.case_setup("rf", 16, 12, 24)
    p12, b12 = lare.case_setup("rf", 12, 12, 12)
    bad = lare.case_fields("rf", p24, seed=1)
    bad[0][:] = 0.0                       # zero density: the CFL timestep is not finite
    tb = srv.submit(p24, b24, bad, 70)
    long_run = srv.submit(p24, b24, lare.case_fields("rf", p24, seed=2), 100000)
    out24 = [np.zeros(lare.box_shape(16, 12, 24)) for _ in range(9)]
    out12 = [np.zeros(lare.box_shape(12, 12, 12)) for _ in range(9)]
    g24 = srv.submit(p24, b24, lare.case_fields("rf", p24, seed=3), 9, out24)
    g12 = srv.submit(p12, b12, lare.case_fields("rf", p12, seed=4), 11, out12)
    for _ in range(2000):
        if srv.poll(long_run)[0] == "running":
            break
        time.sleep(0.005)
    srv.cancel(long_run)
    srv.drain(300)
    assert srv.poll(tb)[0] == "failed"
    assert srv.poll(long_run)[0] == "cancelled"
    for t, out, n, steps, seed in ((g24, out24, (16, 12, 24), 9, 3), (g12, out12, (12, 12, 12), 11, 4)):
        assert srv.poll(t)[0] == "done"
        ref = _solo("rf", n, steps, seed)
        for q, f in enumerate(STATE):
            sl = lare.field_slices(f, *n)
            assert np.array_equal(out[q][sl], ref[f][sl]), f"{n} {f}"
    st = srv.stats()
    assert st["completed"] == 2 and st["failed"] == 1
    srv.close()
