"""Multi-GPU serving router, host side: the placement rule (least outstanding
work among the servers where the solve fits now, then fewest committed
bytes, then lowest index; budget errors) and the solve-size figure it
charges.  No device is touched."""
import pytest

from sams_b200 import lare

GB = 1 << 30


def test_least_outstanding_work_wins():
    assert lare.route_pick([5e9, 1e9, 3e9], [1 * GB, 1 * GB, 1 * GB], [100 * GB] * 3, GB) == 1


def test_ties_go_to_fewest_committed_bytes_then_lowest_index():
    assert lare.route_pick([1e9, 1e9, 1e9], [3 * GB, 2 * GB, 2 * GB], [100 * GB] * 3, GB) == 1
    assert lare.route_pick([0.0, 0.0], [0, 0], [100 * GB] * 2, GB) == 0


def test_a_server_where_the_solve_fits_now_beats_a_less_loaded_full_one():
    # server 0 has less work queued but its budget is committed; server 1 can admit now
    assert lare.route_pick([1e9, 9e9], [95 * GB, 10 * GB], [100 * GB] * 2, 10 * GB) == 1
    # when it fits nowhere now, the least outstanding work among those that can ever hold it
    assert lare.route_pick([1e9, 9e9], [95 * GB, 95 * GB], [100 * GB] * 2, 10 * GB) == 0


def test_budgets_too_small_are_skipped_and_none_raises_budget():
    assert lare.route_pick([0.0, 5e9], [0, 0], [1 * GB, 100 * GB], 2 * GB) == 1
    with pytest.raises(lare.LareError) as e:
        lare.route_pick([0.0, 0.0], [0, 0], [GB, GB], 2 * GB)
    assert e.value.status == -7


def test_sequential_placements_spread_equal_solves():
    """What the router does on a burst of equal solves: each placement adds
    the solve's work and bytes to its server, so the burst spreads evenly."""
    n, work, size = 4, 2.0e9, 3 * GB
    pending, committed = [0.0] * n, [0] * n
    picks = []
    for _ in range(8):
        q = lare.route_pick(pending, committed, [100 * GB] * n, size)
        pending[q] += work
        committed[q] += size
        picks.append(q)
    assert picks == [0, 1, 2, 3, 0, 1, 2, 3]


def test_solve_bytes_grows_with_the_grid():
    p1, _ = lare.case_setup("rf", 16, 16, 16)
    p2, _ = lare.case_setup("rf", 32, 32, 32)
    b1, b2 = lare.solve_bytes(p1), lare.solve_bytes(p2)
    assert 0 < b1 < b2
    # at least the 13 fields' boxes
    assert b2 >= 13 * 8 * 37 ** 3
