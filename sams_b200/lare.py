"""Python access to the B200 LARE3D library through its C ABI
(include/sams_lare.h).

The reference drives LARE3D as a package of a SAMS::runner
(src/PhysicsPackages/LARE/shared_data.h:229-508); here a :class:`LARE3D`
object owns one GPU-resident solve and exposes the same life cycle: set up
parameters and boundary conditions, fill the initial state, step, read the
state back.  All arithmetic happens in libsams_lare.so on the GPU; there is
no CPU fallback, and constructing a solver without the library or without a
GPU raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsams_lare.so")

NFIELDS = 13
FIELD_NAMES = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz",
               "vx1", "vy1", "vz1", "bx", "by", "bz", "dm"]
FIELD = {n: i for i, n in enumerate(FIELD_NAMES)}
STAGGER = [(0, 0, 0)] * 3 + [(1, 1, 1)] * 6 + [(1, 0, 0), (0, 1, 0), (0, 0, 1), (0, 0, 0)]
BC = {"none": 0, "periodic": 1, "zero_gradient": 2, "mirror": 3, "clamp": 4}
CASES = {"ot": 0, "rf": 1, "harris": 2}

STATUS = {0: "ok", -1: "invalid argument", -2: "out of memory", -3: "CUDA error",
          -4: "unsupported option", -5: "non-finite timestep", -6: "timeout", -7: "over budget"}


class Params(ctypes.Structure):
    """sams_lare_params (include/sams_lare_layout.h)."""
    _fields_ = [("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64),
                ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
                ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
                ("z_min", ctypes.c_double), ("z_max", ctypes.c_double),
                ("gas_gamma", ctypes.c_double), ("mu0", ctypes.c_double),
                ("visc1", ctypes.c_double), ("visc2", ctypes.c_double),
                ("dt_multiplier", ctypes.c_double),
                ("eta_background", ctypes.c_double), ("eta0", ctypes.c_double),
                ("j_max", ctypes.c_double),
                ("resistive_mhd", ctypes.c_int32), ("rke", ctypes.c_int32),
                ("geometry", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Bcs(ctypes.Structure):
    """sams_lare_bcs: one condition per (field, dim, edge)."""
    _fields_ = [("kind", ctypes.c_int32 * 2 * 3 * NFIELDS),
                ("value", ctypes.c_double * 2 * 3 * NFIELDS)]


class LareError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None
_P = ctypes.POINTER(ctypes.c_double)


def lib():
    """Load libsams_lare.so (building it first if this checkout has no
    built copy and nvcc is present)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    i64 = ctypes.c_int64
    L.sams_lare_last_error.restype = ctypes.c_char_p
    L.sams_lare_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(Bcs), ctypes.c_int, ctypes.POINTER(vp)]
    L.sams_lare_destroy.argtypes = [vp]
    L.sams_lare_set_stream.argtypes = [vp, vp]
    L.sams_lare_set_bc.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    L.sams_lare_upload_field.argtypes = [vp, ctypes.c_int, _P]
    L.sams_lare_download_field.argtypes = [vp, ctypes.c_int, _P]
    L.sams_lare_upload_field_device.argtypes = [vp, ctypes.c_int, vp]
    L.sams_lare_download_field_device.argtypes = [vp, ctypes.c_int, vp]
    L.sams_lare_step.argtypes = [vp, i64]
    L.sams_lare_step_graph.argtypes = [vp, i64]
    L.sams_lare_synchronize.argtypes = [vp]
    L.sams_lare_get_dt.argtypes = [vp, _P]
    L.sams_lare_get_time.argtypes = [vp, _P]
    L.sams_lare_get_step.argtypes = [vp, ctypes.POINTER(i64)]
    L.sams_lare_field_device_ptr.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(i64),
                                             ctypes.POINTER(i64)]
    L.sams_lare_device_bytes.argtypes = [vp, ctypes.POINTER(i64)]
    L.sams_lare_launches_per_step.argtypes = [vp, ctypes.POINTER(i64)]
    L.sams_lare_phase_times.argtypes = [vp, _P]
    L.sams_lare_fp64_rates.argtypes = [ctypes.c_int, _P]
    L.sams_lare_save.argtypes = [vp, ctypes.c_char_p]
    L.sams_lare_load.argtypes = [vp, ctypes.c_char_p]
    L.sams_lare_case_setup.argtypes = [ctypes.c_int, i64, i64, i64, ctypes.c_double,
                                       ctypes.POINTER(Params), ctypes.POINTER(Bcs)]
    L.sams_lare_case_fields.argtypes = [ctypes.c_int, ctypes.POINTER(Params), ctypes.c_uint64, ctypes.c_double,
                                        ctypes.POINTER(_P)]
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise LareError(rc, lib().sams_lare_last_error().decode())


def box_shape(nx, ny, nz):
    return (nx + 5, ny + 5, nz + 5)


FP64_KINDS = ("add", "mul", "fma", "div", "sqrt", "rcp")


def fp64_rates(device=0):
    """Measured FP64 throughput of `device` (thread-level operations per
    second) by kind: add, mul, fma, IEEE div, sqrt (with one multiply),
    correctly rounded reciprocal (with one multiply)."""
    out = (ctypes.c_double * 6)()
    _check(lib().sams_lare_fp64_rates(device, out))
    return dict(zip(FP64_KINDS, list(out)))


def field_slices(field, nx, ny, nz):
    """Box slices covering a field's own local range."""
    idx = FIELD[field] if isinstance(field, str) else field
    return tuple(slice(0 if s else 1, n + 5) for s, n in zip(STAGGER[idx], (nx, ny, nz)))


def case_setup(case, nx, ny, nz, b0=0.0):
    """Parameters and boundary conditions of a named workload."""
    p, b = Params(), Bcs()
    _check(lib().sams_lare_case_setup(CASES.get(case, case), nx, ny, nz, b0, ctypes.byref(p), ctypes.byref(b)))
    return p, b


def case_fields(case, params, seed=1, b0=0.0):
    """Initial state of a named workload as 13 box arrays."""
    shape = box_shape(params.nx, params.ny, params.nz)
    arrs = [np.zeros(shape) for _ in range(NFIELDS)]
    ptrs = (_P * NFIELDS)(*[a.ctypes.data_as(_P) for a in arrs])
    _check(lib().sams_lare_case_fields(CASES.get(case, case), ctypes.byref(params), seed, b0, ptrs))
    return arrs


class LARE3D:
    """One LARE3D solve resident on a GPU (the reference package's name and
    role, shared_data.h:330-345)."""

    name = "LARE3D"
    coreSimulation = True
    timeSimulation = True

    def __init__(self, params, bcs, device=0):
        self.params = params
        self.shape = box_shape(params.nx, params.ny, params.nz)
        h = ctypes.c_void_p()
        _check(lib().sams_lare_create(ctypes.byref(params), ctypes.byref(bcs), device, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().sams_lare_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_bc(self, field, dim, edge, kind, value=0.0):
        f = FIELD[field] if isinstance(field, str) else field
        k = BC[kind] if isinstance(kind, str) else kind
        _check(lib().sams_lare_set_bc(self._h, f, dim, edge, k, value))

    def upload(self, field, arr):
        f = FIELD[field] if isinstance(field, str) else field
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"expected box shape {self.shape}, got {a.shape}")
        _check(lib().sams_lare_upload_field(self._h, f, a.ctypes.data_as(_P)))
        _check(lib().sams_lare_synchronize(self._h))

    def upload_all(self, fields):
        for f, a in enumerate(fields):
            self.upload(f, a)

    def download(self, field, out=None):
        f = FIELD[field] if isinstance(field, str) else field
        if out is None:
            out = np.empty(self.shape)
        _check(lib().sams_lare_download_field(self._h, f, out.ctypes.data_as(_P)))
        return out

    def save(self, path):
        """Checkpoint: the 13 fields, step count, time and last dt as a
        SAMSDUMP1 file (readable by oracle.dumpio.Dump)."""
        _check(lib().sams_lare_save(self.handle, str(path).encode()))

    def load(self, path):
        """Restart from a SAMSDUMP1 file of the same grid (a checkpoint, or a
        dump of the reference's own state)."""
        _check(lib().sams_lare_load(self.handle, str(path).encode()))

    def step(self, n=1, graph=False):
        if graph:
            _check(lib().sams_lare_step_graph(self._h, n))
        else:
            _check(lib().sams_lare_step(self._h, n))

    def synchronize(self):
        _check(lib().sams_lare_synchronize(self._h))

    @property
    def dt(self):
        v = ctypes.c_double()
        _check(lib().sams_lare_get_dt(self._h, ctypes.byref(v)))
        return v.value

    @property
    def time(self):
        v = ctypes.c_double()
        _check(lib().sams_lare_get_time(self._h, ctypes.byref(v)))
        return v.value

    @property
    def steps(self):
        v = ctypes.c_int64()
        _check(lib().sams_lare_get_step(self._h, ctypes.byref(v)))
        return v.value

    @property
    def device_bytes(self):
        v = ctypes.c_int64()
        _check(lib().sams_lare_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    @property
    def launches_per_step(self):
        v = ctypes.c_int64()
        _check(lib().sams_lare_launches_per_step(self._h, ctypes.byref(v)))
        return v.value

    def phase_times(self):
        """Run one step; device ms of (lagrangian, corrector, remap_x,
        remap_y, remap_z)."""
        out = (ctypes.c_double * 5)()
        _check(lib().sams_lare_phase_times(self._h, out))
        return list(out)

    def set_stream(self, stream_ptr):
        _check(lib().sams_lare_set_stream(self._h, ctypes.c_void_p(stream_ptr)))


def _bind_batch(L):
    if getattr(L, "_batch_bound", False):
        return
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    ip = ctypes.POINTER(ctypes.c_int)
    L.sams_lare_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.sams_lare_batch_destroy.argtypes = [vp]
    L.sams_lare_batch_set_stream.argtypes = [vp, vp]
    L.sams_lare_batch_add.argtypes = [vp, ctypes.POINTER(Params), ctypes.POINTER(Bcs), ip]
    L.sams_lare_batch_remove.argtypes = [vp, ctypes.c_int]
    L.sams_lare_batch_upload_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, _P]
    L.sams_lare_batch_download_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, _P]
    L.sams_lare_batch_step.argtypes = [vp, i64]
    L.sams_lare_batch_step_graph.argtypes = [vp, i64]
    L.sams_lare_batch_synchronize.argtypes = [vp]
    L.sams_lare_batch_get_state.argtypes = [vp, ctypes.c_int, _P, _P, ctypes.POINTER(i64)]
    L.sams_lare_batch_set_tuning.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.sams_lare_batch_autotune.argtypes = [vp, ctypes.c_int, ip, ip, _P]
    L.sams_lare_batch_device_bytes.argtypes = [vp, ctypes.POINTER(i64)]
    L._batch_bound = True


class Batch:
    """Many independent LARE3D solves stepped together on one GPU (each
    phase one persistent launch over all solves' tiles; each solve keeps its
    own CFL timestep)."""

    def __init__(self, device=0):
        L = lib()
        _bind_batch(L)
        h = ctypes.c_void_p()
        _check(L.sams_lare_batch_create(device, ctypes.byref(h)))
        self._h = h
        self.shapes = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().sams_lare_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, params, bcs, fields=None):
        i = ctypes.c_int()
        _check(lib().sams_lare_batch_add(self._h, ctypes.byref(params), ctypes.byref(bcs), ctypes.byref(i)))
        self.shapes[i.value] = box_shape(params.nx, params.ny, params.nz)
        if fields is not None:
            for f, a in enumerate(fields):
                self.upload(i.value, f, a)
            self.synchronize()
        return i.value

    def remove(self, sid):
        _check(lib().sams_lare_batch_remove(self._h, sid))
        self.shapes.pop(sid, None)

    def upload(self, sid, field, arr):
        f = FIELD[field] if isinstance(field, str) else field
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != self.shapes[sid]:
            raise ValueError(f"expected box shape {self.shapes[sid]}, got {a.shape}")
        self._keep = a  # the copy is asynchronous
        _check(lib().sams_lare_batch_upload_field(self._h, sid, f, a.ctypes.data_as(_P)))
        _check(lib().sams_lare_batch_synchronize(self._h))

    def download(self, sid, field, out=None):
        f = FIELD[field] if isinstance(field, str) else field
        if out is None:
            out = np.empty(self.shapes[sid])
        _check(lib().sams_lare_batch_download_field(self._h, sid, f, out.ctypes.data_as(_P)))
        return out

    def step(self, n=1, graph=False):
        if graph:
            _check(lib().sams_lare_batch_step_graph(self._h, n))
        else:
            _check(lib().sams_lare_batch_step(self._h, n))

    def synchronize(self):
        _check(lib().sams_lare_batch_synchronize(self._h))

    def state(self, sid):
        dt, tm, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        _check(lib().sams_lare_batch_get_state(self._h, sid, ctypes.byref(dt), ctypes.byref(tm), ctypes.byref(st)))
        return dt.value, tm.value, st.value

    def set_tuning(self, tile_planes, blocks_per_sm):
        _check(lib().sams_lare_batch_set_tuning(self._h, tile_planes, blocks_per_sm))

    def autotune(self, trial_steps=2):
        t, b, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(lib().sams_lare_batch_autotune(self._h, trial_steps, ctypes.byref(t), ctypes.byref(b),
                                              ctypes.byref(ms)))
        return t.value, b.value, ms.value

    @property
    def device_bytes(self):
        v = ctypes.c_int64()
        _check(lib().sams_lare_batch_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    def set_stream(self, stream_ptr):
        _check(lib().sams_lare_batch_set_stream(self._h, ctypes.c_void_p(stream_ptr)))


class ServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("queued", ctypes.c_int64), ("running", ctypes.c_int64),
                ("p50_latency_s", ctypes.c_double), ("p99_latency_s", ctypes.c_double),
                ("mean_latency_s", ctypes.c_double), ("cell_updates", ctypes.c_double),
                ("wall_s", ctypes.c_double), ("cell_updates_per_s", ctypes.c_double),
                ("device_bytes_in_use", ctypes.c_int64), ("pending_cell_updates", ctypes.c_double),
                ("queued_bytes", ctypes.c_int64)]


SERVE_STATUS = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


def _bind_serve(L):
    if getattr(L, "_serve_bound", False):
        return
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    L.sams_lare_serve_create.argtypes = [ctypes.c_int, i64, ctypes.POINTER(vp)]
    L.sams_lare_serve_submit.argtypes = [vp, ctypes.POINTER(Params), ctypes.POINTER(Bcs), ctypes.POINTER(_P), i64,
                                         ctypes.POINTER(_P), ctypes.POINTER(i64)]
    L.sams_lare_serve_set_max_cells.argtypes = [vp, i64]
    L.sams_lare_serve_poll.argtypes = [vp, i64, ctypes.POINTER(ctypes.c_int), _P]
    L.sams_lare_serve_fetch.argtypes = [vp, i64, ctypes.c_int, _P]
    L.sams_lare_serve_release.argtypes = [vp, i64]
    L.sams_lare_serve_cancel.argtypes = [vp, i64]
    L.sams_lare_serve_drain.argtypes = [vp, ctypes.c_double]
    L.sams_lare_serve_get_stats.argtypes = [vp, ctypes.POINTER(ServeStats)]
    L.sams_lare_serve_destroy.argtypes = [vp]
    L.sams_lare_serve_solve_bytes.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(i64)]
    L.sams_lare_router_create.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, i64, ctypes.POINTER(vp)]
    L.sams_lare_router_submit.argtypes = L.sams_lare_serve_submit.argtypes
    L.sams_lare_router_placement.argtypes = [vp, i64, ctypes.POINTER(ctypes.c_int)]
    for name in ("set_max_cells", "poll", "fetch", "release", "cancel", "drain", "get_stats", "destroy"):
        getattr(L, "sams_lare_router_" + name).argtypes = getattr(L, "sams_lare_serve_" + name).argtypes
    L.sams_lare_router_server_stats.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ServeStats)]
    L.sams_lare_route_pick.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(i64),
                                       ctypes.POINTER(i64), i64, ctypes.POINTER(ctypes.c_int)]
    L._serve_bound = True


def solve_bytes(params):
    """Device bytes one solve takes while a server runs it."""
    L = lib()
    _bind_serve(L)
    v = ctypes.c_int64()
    _check(L.sams_lare_serve_solve_bytes(ctypes.byref(params), ctypes.byref(v)))
    return v.value


def route_pick(pending_cell_updates, committed_bytes, budget_bytes, request_bytes):
    """The multi-GPU router's placement rule (host only): index of the server
    a solve of `request_bytes` goes to, given each server's outstanding work
    and committed bytes."""
    L = lib()
    _bind_serve(L)
    n = len(pending_cell_updates)
    pend = (ctypes.c_double * n)(*pending_cell_updates)
    comm = (ctypes.c_int64 * n)(*committed_bytes)
    bud = (ctypes.c_int64 * n)(*budget_bytes)
    idx = ctypes.c_int(-1)
    _check(L.sams_lare_route_pick(n, pend, comm, bud, int(request_bytes), ctypes.byref(idx)))
    return idx.value


class Server:
    """Continuous-batching LARE3D server on one GPU (include/sams_lare.h,
    serving section).  Submitted solves are admitted as device memory within
    `budget_bytes` frees up, stepped together with every other running solve
    (large ones on their own streams, small and thin ones in one batched
    step), and their final state copied back when their step count is
    reached."""

    _prefix = "sams_lare_serve_"

    def __init__(self, budget_bytes, device=0, max_cells=0):
        L = lib()
        _bind_serve(L)
        h = ctypes.c_void_p()
        _check(L.sams_lare_serve_create(device, int(budget_bytes), ctypes.byref(h)))
        self._h = h
        self._keep = {}
        if max_cells:
            self.set_max_cells(max_cells)

    def _fn(self, name):
        return getattr(lib(), self._prefix + name)

    def set_max_cells(self, max_cells):
        """Cap the interior cells of the solves running at once (0 = none)."""
        _check(self._fn("set_max_cells")(self._h, int(max_cells)))

    def close(self):
        if getattr(self, "_h", None):
            self._fn("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, params, bcs, ic, nsteps, out=None):
        ic = [np.ascontiguousarray(a, dtype=np.float64) for a in ic]
        ip = (_P * NFIELDS)(*[a.ctypes.data_as(_P) for a in ic])
        op = None
        if out is not None:
            op = (_P * 9)(*[a.ctypes.data_as(_P) for a in out])
        t = ctypes.c_int64()
        _check(self._fn("submit")(self._h, ctypes.byref(params), ctypes.byref(bcs), ip, int(nsteps),
                                            op, ctypes.byref(t)))
        self._keep[t.value] = (ic, out, box_shape(params.nx, params.ny, params.nz))
        return t.value

    def poll(self, ticket):
        st, lat = ctypes.c_int(), ctypes.c_double()
        _check(self._fn("poll")(self._h, ticket, ctypes.byref(st), ctypes.byref(lat)))
        return SERVE_STATUS[st.value], lat.value

    def fetch(self, ticket, index):
        out = np.empty(self._keep[ticket][2])
        _check(self._fn("fetch")(self._h, ticket, index, out.ctypes.data_as(_P)))
        return out

    def cancel(self, ticket):
        """Withdraw a queued or running request (its status becomes
        "cancelled"; a running one leaves before the next batched step)."""
        _check(self._fn("cancel")(self._h, ticket))

    def release(self, ticket):
        _check(self._fn("release")(self._h, ticket))
        self._keep.pop(ticket, None)

    def drain(self, timeout_s=600.0):
        _check(self._fn("drain")(self._h, float(timeout_s)))

    def stats(self):
        s = ServeStats()
        _check(self._fn("get_stats")(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in ServeStats._fields_}


class Router(Server):
    """Serving on several GPUs (include/sams_lare.h, "Serving on several
    GPUs"): one continuous-batching server per entry of `devices` and a host
    router that places each submitted solve on the least-loaded one.  Same
    calls as Server; `placement(ticket)` says which server took a solve."""

    _prefix = "sams_lare_router_"

    def __init__(self, budget_bytes_per_device, devices=(0,), max_cells=0):
        L = lib()
        _bind_serve(L)
        devs = (ctypes.c_int * len(devices))(*devices)
        h = ctypes.c_void_p()
        _check(L.sams_lare_router_create(devs, len(devices), int(budget_bytes_per_device), ctypes.byref(h)))
        self._h = h
        self._keep = {}
        self.devices = tuple(devices)
        if max_cells:
            self.set_max_cells(max_cells)

    def placement(self, ticket):
        idx = ctypes.c_int(-1)
        _check(lib().sams_lare_router_placement(self._h, ticket, ctypes.byref(idx)))
        return idx.value

    def server_stats(self, index):
        s = ServeStats()
        _check(lib().sams_lare_router_server_stats(self._h, index, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in ServeStats._fields_}


def _bind_dist(L):
    if getattr(L, "_dist_bound", False):
        return
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    L.sams_lare_dist_partition.argtypes = [i64, ctypes.c_int, ctypes.POINTER(i64)]
    L.sams_lare_dist_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(Bcs), ctypes.POINTER(ctypes.c_int),
                                        ctypes.c_int, ctypes.POINTER(vp)]
    L.sams_lare_dist_slab.argtypes = [vp, ctypes.c_int, ctypes.POINTER(i64), ctypes.POINTER(i64)]
    L.sams_lare_dist_upload_field.argtypes = [vp, ctypes.c_int, _P]
    L.sams_lare_dist_download_field.argtypes = [vp, ctypes.c_int, _P]
    L.sams_lare_dist_step.argtypes = [vp, i64]
    L.sams_lare_dist_get_state.argtypes = [vp, _P, _P, ctypes.POINTER(i64)]
    L.sams_lare_dist_destroy.argtypes = [vp]
    L._dist_bound = True


def dist_partition(nx, nparts):
    """Cell offsets of the x slabs of a distributed solve: slab q covers
    cells offsets[q]+1 .. offsets[q+1] (host only)."""
    L = lib()
    _bind_dist(L)
    out = (ctypes.c_int64 * (nparts + 1))()
    _check(L.sams_lare_dist_partition(int(nx), int(nparts), out))
    return list(out)


class DistLARE3D:
    """One LARE3D solve cut along x into slabs over several GPUs (the
    reference's MPI decomposition, include/harness/mpiManager.h:1246-1277):
    slab q runs on devices[q]; ghost planes move between slabs by peer
    copies at every boundary fill.  Whole-grid box arrays in and out, as for
    LARE3D."""

    name = "LARE3D"

    def __init__(self, params, bcs, devices):
        L = lib()
        _bind_dist(L)
        self.params = params
        self.shape = box_shape(params.nx, params.ny, params.nz)
        devs = (ctypes.c_int * len(devices))(*devices)
        h = ctypes.c_void_p()
        _check(L.sams_lare_dist_create(ctypes.byref(params), ctypes.byref(bcs), devs, len(devices),
                                       ctypes.byref(h)))
        self._h = h
        self.devices = tuple(devices)

    def close(self):
        if getattr(self, "_h", None):
            lib().sams_lare_dist_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def slab(self, part):
        first, n = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().sams_lare_dist_slab(self._h, part, ctypes.byref(first), ctypes.byref(n)))
        return first.value, n.value

    def upload(self, field, arr):
        idx = FIELD[field] if isinstance(field, str) else field
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.shape == self.shape
        _check(lib().sams_lare_dist_upload_field(self._h, idx, a.ctypes.data_as(_P)))

    def upload_all(self, fields):
        for f, a in enumerate(fields):
            self.upload(f, a)

    def download(self, field, out=None):
        idx = FIELD[field] if isinstance(field, str) else field
        out = np.empty(self.shape) if out is None else out
        _check(lib().sams_lare_dist_download_field(self._h, idx, out.ctypes.data_as(_P)))
        return out

    def step(self, n=1):
        _check(lib().sams_lare_dist_step(self._h, int(n)))

    def state(self):
        dt, tm, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        _check(lib().sams_lare_dist_get_state(self._h, ctypes.byref(dt), ctypes.byref(tm), ctypes.byref(st)))
        return dt.value, tm.value, st.value
