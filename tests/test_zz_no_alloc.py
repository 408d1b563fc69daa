"""The allocation-free entry point, sams_lare_step_noalloc.

It is for callers that cannot call cudaMalloc while they run (their device
memory comes from their own pool, or their footprint must not grow): they
hand over their own device buffers for the 13 fields and the step's scratch
comes from a fixed static array in the library.  Here the caller's buffers
are torch tensors; the check is that two calls in a row give exactly what
the regular entry point (sams_lare_create + sams_lare_step) gives for the
same steps, and that grids larger than the static array are refused.

This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from sams_b200 import lare

pytestmark = pytest.mark.gpu

STATE = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz", "bx", "by", "bz"]


def _noalloc_fn():
    L = lare.lib()
    fn = L.sams_lare_step_noalloc
    fn.argtypes = [ctypes.POINTER(lare.Params), ctypes.POINTER(lare.Bcs), ctypes.c_void_p * lare.NFIELDS,
                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int64,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


# The long-z grids run the kernels that need many z values on this entry
# point's dense rows: nz = 31 and nz = 290 run the out-of-place x / y sweep
# (and its pointer swap on the caller's buffers), nz = 290 also the separate
# z-sweep kernels used when a z line does not fit one block.
@pytest.mark.parametrize("case,n,calls", [("ot", (24, 20, 8), (3, 2)), ("rf", (16, 14, 12), (2, 2)),
                                          ("harris", (20, 12, 6), (2, 3)), ("ot", (16, 12, 2), (2, 2)),
                                          ("rf", (10, 8, 31), (2, 2)), ("ot", (6, 5, 290), (2, 1))])
def test_noalloc_matches_regular_entry_point(case, n, calls):
    import torch

    fn = _noalloc_fn()
    nx, ny, nz = n
    p, b = lare.case_setup(case, nx, ny, nz)
    fields = lare.case_fields(case, p, seed=4)
    reg = lare.LARE3D(p, b)
    reg.upload_all(fields)
    dev = [torch.from_numpy(f.copy()).cuda() for f in fields]   # caller-owned device buffers
    ptrs = (ctypes.c_void_p * lare.NFIELDS)(*[t.data_ptr() for t in dev])
    dt = ctypes.c_double(0.0)
    tm = ctypes.c_double(0.0)
    torch.cuda.synchronize()
    for k in calls:                                              # two calls in a row
        rc = fn(ctypes.byref(p), ctypes.byref(b), ptrs, ctypes.byref(dt), ctypes.byref(tm), k, None)
        assert rc == 0, lare.lib().sams_lare_last_error().decode()
        reg.step(k)
        reg.synchronize()
        assert dt.value == reg.dt
        assert tm.value == reg.time
        for f in STATE:
            sl = lare.field_slices(f, nx, ny, nz)
            got = dev[lare.FIELD[f]].cpu().numpy()[sl]
            want = reg.download(f)[sl]
            assert np.array_equal(got, want), f"{case} field {f} after {k} more steps"
    reg.close()


def test_noalloc_rejects_grids_beyond_the_static_array():
    import torch

    fn = _noalloc_fn()
    p, b = lare.case_setup("ot", 96, 96, 64)
    one = torch.zeros(8, dtype=torch.float64, device="cuda")     # never touched: refused before use
    ptrs = (ctypes.c_void_p * lare.NFIELDS)(*([one.data_ptr()] * lare.NFIELDS))
    dt, tm = ctypes.c_double(0.0), ctypes.c_double(0.0)
    rc = fn(ctypes.byref(p), ctypes.byref(b), ptrs, ctypes.byref(dt), ctypes.byref(tm), 1, None)
    assert rc == -1
    assert "too large" in lare.lib().sams_lare_last_error().decode()
