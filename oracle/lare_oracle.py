"""Python access to the CPU checker (oracle/lare_oracle.c) and to the
reference harness binary (oracle/_ref/lare_ref).

TEST INFRASTRUCTURE ONLY: imported by tests/, bench.py's CPU-baseline leg
and __graft_entry__.smoke(), never by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "_build", "liblare_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "lare_ref")
REF_BENCH_BIN = os.path.join(HERE, "_ref", "lare_ref_bench")
REF_BENCH_BIN_V4 = os.path.join(HERE, "_ref", "lare_ref_bench_v4")
AVX512_V4 = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def host_isa():
    """'x86-64-v4' when this host's CPU has the AVX-512 subsets of that level,
    else 'x86-64-v3'."""
    try:
        with open("/proc/cpuinfo") as f:
            flags = set()
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        return "x86-64-v3"
    return "x86-64-v4" if all(x in flags for x in AVX512_V4) else "x86-64-v3"


def reference_bench_binary():
    """The reference's release build for the widest ISA this host runs (the
    reference builds with -march=native), and that ISA."""
    isa = host_isa()
    if isa == "x86-64-v4" and os.path.exists(REF_BENCH_BIN_V4):
        return REF_BENCH_BIN_V4, isa
    return REF_BENCH_BIN, "x86-64-v3"

NFIELDS = 13
FIELD_NAMES = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz",
               "vx1", "vy1", "vz1", "bx", "by", "bz", "dm"]
# staggering per field and dimension (1 = half cell), include/sams_lare_layout.h
STAGGER = [(0, 0, 0)] * 3 + [(1, 1, 1)] * 6 + [(1, 0, 0), (0, 1, 0), (0, 0, 1), (0, 0, 0)]
CASES = {"ot": 0, "rf": 1, "harris": 2}


class Params(ctypes.Structure):
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
    _fields_ = [("kind", ctypes.c_int32 * 2 * 3 * NFIELDS),
                ("value", ctypes.c_double * 2 * 3 * NFIELDS)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.lo_create.restype = vp
        L.lo_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(Bcs)]
        L.lo_destroy.argtypes = [vp]
        L.lo_set_fields.argtypes = [vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        L.lo_get_field.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.lo_get_named.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
        L.lo_step.argtypes = [vp, ctypes.c_int64]
        L.lo_step_phase.argtypes = [vp, ctypes.c_int]
        L.lo_dt.restype = ctypes.c_double
        L.lo_dt.argtypes = [vp]
        L.lo_time.restype = ctypes.c_double
        L.lo_time.argtypes = [vp]
        L.lo_steps.restype = ctypes.c_int64
        L.lo_steps.argtypes = [vp]
        L.sams_lare_case_setup.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                           ctypes.c_double, ctypes.POINTER(Params), ctypes.POINTER(Bcs)]
        L.sams_lare_case_fields.argtypes = [ctypes.c_int, ctypes.POINTER(Params), ctypes.c_uint64,
                                            ctypes.c_double, ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        _lib = L
    return _lib


def build(ref_tree=None):
    """Build the checker, and the reference harness when `ref_tree` (the
    reference source tree; default: the SAMS_REFERENCE_TREE environment
    variable) is given."""
    ref_tree = ref_tree or os.environ.get("SAMS_REFERENCE_TREE")
    cmd = ["make", "-s", "-C", HERE, "-j8"] + (["REF=" + ref_tree] if ref_tree else [])
    subprocess.run(cmd, check=True)


def reference_tree():
    """The reference source tree the harness was last built from, or None
    (recorded by oracle/Makefile; absent where the tree never was)."""
    try:
        with open(os.path.join(HERE, "_ref", "ref_tree.txt")) as f:
            path = f.read().strip()
    except OSError:
        return None
    return path if path and os.path.isdir(path) else None


def box_shape(nx, ny, nz):
    return (nx + 5, ny + 5, nz + 5)


def _ptrs(arrs):
    P = ctypes.POINTER(ctypes.c_double)
    return (P * NFIELDS)(*[a.ctypes.data_as(P) for a in arrs])


def case_setup(case, nx, ny, nz, b0=0.0):
    p, b = Params(), Bcs()
    rc = lib().sams_lare_case_setup(CASES.get(case, case), nx, ny, nz, b0, ctypes.byref(p), ctypes.byref(b))
    if rc != 0:
        raise ValueError(f"case_setup failed for {case} {nx}x{ny}x{nz}")
    return p, b


def case_fields(case, params, seed=1, b0=0.0):
    shape = box_shape(params.nx, params.ny, params.nz)
    arrs = [np.zeros(shape) for _ in range(NFIELDS)]
    rc = lib().sams_lare_case_fields(CASES.get(case, case), ctypes.byref(params), seed, b0, _ptrs(arrs))
    if rc != 0:
        raise ValueError("case_fields failed")
    return arrs


class Oracle:
    """The C restatement of the LARE3D timestep on box buffers."""

    def __init__(self, params, bcs, fields):
        self.params, self.bcs = params, bcs
        self.shape = box_shape(params.nx, params.ny, params.nz)
        self.h = lib().lo_create(ctypes.byref(params), ctypes.byref(bcs))
        if not self.h:
            raise ValueError("lo_create failed")
        arrs = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
        if lib().lo_set_fields(self.h, _ptrs(arrs)) != 0:
            raise ValueError("lo_set_fields failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().lo_destroy(self.h)
            self.h = None

    def step(self, n=1):
        lib().lo_step(self.h, n)

    def step_phase(self, phase):
        lib().lo_step_phase(self.h, phase)

    def field(self, f):
        idx = FIELD_NAMES.index(f) if isinstance(f, str) else f
        out = np.empty(self.shape)
        lib().lo_get_field(self.h, idx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def named(self, name):
        out = np.empty(self.shape)
        rc = lib().lo_get_named(self.h, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if rc != 0:
            raise KeyError(name)
        return out

    @property
    def dt(self):
        return lib().lo_dt(self.h)

    @property
    def time(self):
        return lib().lo_time(self.h)

    @property
    def steps(self):
        return lib().lo_steps(self.h)


def field_slices(field, nx, ny, nz):
    """Box slices of a field's own local range (centred -1..n+2, half-cell
    -2..n+2)."""
    idx = FIELD_NAMES.index(field) if isinstance(field, str) else field
    return tuple(slice(0 if s else 1, n + 5) for s, n in zip(STAGGER[idx], (nx, ny, nz)))


def run_reference(case, nx, ny, nz, steps, dump, seed=1, b0=0.0, ic=None, extra=(), binary=None, threads=None):
    """Run the reference harness binary; returns its JSON summary line.
    threads=1 gives the reference's serial order of floating-point atomic
    adds (the rke correction), i.e. a deterministic result."""
    import json
    import os
    cmd = [binary or REF_BIN, "--case", case, "--nx", str(nx), "--ny", str(ny), "--nz", str(nz),
           "--steps", str(steps), "--seed", str(seed), "--quiet"]
    if b0:
        cmd += ["--b0", repr(b0)]
    if dump:
        cmd += ["--dump", dump]
    if ic:
        cmd += ["--ic", ic]
    cmd += list(extra)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads)) if threads else None
    out = subprocess.run(cmd, check=True, capture_output=True, text=True, env=env).stdout
    return json.loads(out.strip().splitlines()[-1])
