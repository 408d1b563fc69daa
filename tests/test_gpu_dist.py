"""One solve cut along x into slabs (sams_lare_dist_*): the result must equal
the undivided solve's bit for bit, and the reference's own outputs where a
fixture exists.  One GPU is enough: every slab gets its own solver, stream
and host thread on device 0, and slabs meet only through stream-ordered
copies and events (no kernel waits on another)."""
import numpy as np
import pytest

from sams_b200 import lare
from tests.golden.make_golden import GEO_DOMAIN, STATE, apply_options, load

pytestmark = pytest.mark.gpu


def _setup(case, n, b0=0.0, options=None, x_bc=None):
    p, b = lare.case_setup(case, *n, b0)
    if options:
        apply_options(p, options)
    if x_bc is not None:
        for f in range(lare.NFIELDS):
            for e in range(2):
                b.kind[f][0][e] = x_bc
    return p, b


def _pair(case, n, parts, seed=1, b0=0.0, options=None, x_bc=None):
    p, b = _setup(case, n, b0, options, x_bc)
    ic = lare.case_fields(case, p, seed=seed, b0=b0)
    one = lare.LARE3D(p, b)
    one.upload_all(ic)
    dist = lare.DistLARE3D(p, b, devices=[0] * parts)
    dist.upload_all(ic)
    return one, dist


def _assert_equal(one, dist, n, label):
    for f in STATE:
        sl = lare.field_slices(f, *n)
        a, b = one.download(f)[sl], dist.download(f)[sl]
        if not np.array_equal(a, b):
            d = np.abs(a - b)
            where = np.unravel_index(np.argmax(d), d.shape)
            raise AssertionError(f"{label}: {f} differs, max abs {d.max():.3e} at box index {where}")


@pytest.mark.parametrize("case,n,parts,steps,opts", [
    ("ot", (12, 10, 6), 2, 5, None),
    ("ot", (13, 10, 6), 3, 5, None),               # uneven slabs 5, 4, 4
    ("rf", (16, 8, 8), 3, 4, None),                # resistive, power-of-two grid
    ("rf", (20, 12, 9), 4, 4, None),
    ("harris", (12, 10, 6), 3, 4, None),           # conducting walls in y
    ("ot", (12, 10, 2), 2, 4, None),               # two cells in z
    ("ot", (12, 10, 6), 2, 4, {"geometry": 1, "domain": GEO_DOMAIN}),
    ("rf", (12, 8, 6), 2, 3, {"geometry": 2, "domain": GEO_DOMAIN}),
    ("rf", (64, 32, 32), 4, 3, None),
    ("rf", (12, 8, 24), 3, 3, None),               # fused out-of-place x / y sweeps
    ("ot", (10, 8, 24), 2, 3, {"geometry": 1, "domain": GEO_DOMAIN}),
])
def test_slabs_equal_undivided_solve(case, n, parts, steps, opts):
    one, dist = _pair(case, n, parts, options=opts)
    for k in range(steps):
        one.step(1)
        dist.step(1)
        assert dist.state()[0] == one.dt, f"dt of step {k + 1}"
    _assert_equal(one, dist, n, f"{case}{n}/{parts}")
    dt, tm, st = dist.state()
    assert (dt, tm, st) == (one.dt, one.time, one.steps)


@pytest.mark.parametrize("kind", [2, 3])  # zero-gradient, mirror x edges: filled on the end slabs
def test_non_periodic_x_edges(kind):
    n = (12, 10, 6)
    one, dist = _pair("ot", n, 3, x_bc=kind)
    one.step(4)
    dist.step(4)
    _assert_equal(one, dist, n, f"x bc {kind}")


def test_several_steps_per_call_and_golden():
    z, meta = load("ot_12x10x6_s5")
    p, b = _setup(meta["case"], (meta["nx"], meta["ny"], meta["nz"]), meta["b0"], meta)
    dist = lare.DistLARE3D(p, b, devices=[0, 0])
    dist.upload_all(lare.case_fields(meta["case"], p, seed=meta["seed"], b0=meta["b0"]))
    assert dist.slab(0) == (1, 6) and dist.slab(1) == (7, 6)
    dist.step(meta["steps"])
    for f in STATE:
        ref = z[f]
        m = ~np.isnan(ref)
        assert np.array_equal(dist.download(f)[m], ref[m]), f


def test_rke_is_refused():
    p, b = lare.case_setup("ot", 12, 10, 6)
    p.rke = 1
    with pytest.raises(lare.LareError) as e:
        lare.DistLARE3D(p, b, devices=[0, 0])
    assert e.value.status == -4
