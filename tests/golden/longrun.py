"""Records of the reference's state after the benchmark configurations' full
step counts, and the checks made against them.

A full-size state (1.2 GB at 256^3) cannot be committed, so a record keeps,
per state field over its own index range, the SHA-256 of its float64 bytes
plus 1024 seeded sample points, and for the run the dt history, the final
time, the total mass sum(rho * cv) and the energy budget (internal, kinetic,
magnetic).  `make_longrun.py` writes the records from the reference itself;
the GPU test (tests/test_gpu_longrun.py) steps the same workloads the same
number of steps and compares:

  * every field's hash (the bar: bit-identical), and on a mismatch the
    samples against the 1e-10 relative L-infinity tolerance (relative to the
    field's largest sampled magnitude) to say how far it is off;
  * the dt history exactly;
  * total mass against the initial state's to 1e-13 relative (periodic
    domains; the remap and the Lagrangian step conserve it);
  * the energy budget to 1e-10 relative of the reference's.
"""
import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
STATE = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz", "bx", "by", "bz"]
NSAMPLES = 1024
SAMPLE_SEED = 20261204

# (name, case, nx, ny, nz, steps, seed): the benchmark configurations that run
# one solve, at their stated sizes and step counts
RUNS = [
    ("c0_ot_128x128x4_s200", "ot", 128, 128, 4, 200, 1),
    ("c1_rf_256cube_s500", "rf", 256, 256, 256, 500, 1),
    ("c2_harris_512x256x64_s1000", "harris", 512, 256, 64, 1000, 1),
]


def path(name):
    return os.path.join(HERE, name + ".longrun.npz")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def sample_index(shape, field_index):
    rng = np.random.default_rng(SAMPLE_SEED + field_index)
    return np.stack([rng.integers(0, s, NSAMPLES) for s in shape]).astype(np.int32)


def energy_budget(get, nx, ny, nz, dv, mu0):
    """Internal, kinetic and magnetic energy over the interior cells of a
    Cartesian grid of cell volume dv.  `get(name)` returns a field's box
    (-2..n+2 per dimension).  Velocities are node values (the cell's upper
    corner), B the average of a cell's two faces."""
    def inner(a):
        return a[3:nx + 3, 3:ny + 3, 3:nz + 3]
    rho = inner(get("rho"))
    internal = (rho * (inner(get("energy_electron")) + inner(get("energy_ion")))).sum() * dv
    v2 = sum(inner(get(c)) ** 2 for c in ("vx", "vy", "vz"))
    kinetic = 0.5 * (rho * v2).sum() * dv
    bx, by, bz = get("bx"), get("by"), get("bz")
    bxc = 0.5 * (bx[3:nx + 3, 3:ny + 3, 3:nz + 3] + bx[2:nx + 2, 3:ny + 3, 3:nz + 3])
    byc = 0.5 * (by[3:nx + 3, 3:ny + 3, 3:nz + 3] + by[3:nx + 3, 2:ny + 2, 3:nz + 3])
    bzc = 0.5 * (bz[3:nx + 3, 3:ny + 3, 3:nz + 3] + bz[3:nx + 3, 3:ny + 3, 2:nz + 2])
    magnetic = ((bxc ** 2 + byc ** 2 + bzc ** 2) / (2.0 * mu0)).sum() * dv
    return internal, kinetic, magnetic


def mass(rho_box, nx, ny, nz, dv):
    return float(rho_box[3:nx + 3, 3:ny + 3, 3:nz + 3].sum() * dv)


def field_record(local):
    """Hash and samples of one field over its own index range: `local` maps
    a field name to that range's array."""
    out = {}
    for q, f in enumerate(STATE):
        a = local(f)
        idx = sample_index(a.shape, q)
        out[f] = (digest(a), idx, a[tuple(idx)])
    return out


def save(name, meta, fields):
    arrays = {"meta": np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)}
    for f, (h, idx, vals) in fields.items():
        arrays[f + ".idx"] = idx
        arrays[f + ".val"] = vals
        meta.setdefault("sha256", {})[f] = h
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(path(name), **arrays)


def load(name):
    z = np.load(path(name))
    meta = json.loads(bytes(z["meta"]).decode())
    fields = {f: (meta["sha256"][f], z[f + ".idx"], z[f + ".val"]) for f in STATE}
    return meta, fields
