"""Generate the golden fixtures in this directory from the REFERENCE itself.

Runs oracle/_ref/lare_ref (the unmodified reference LARE3D sources compiled
by oracle/Makefile, driven by its own SAMS::runner) on small seeded cases and
stores, per case, the nine state fields over their own index ranges plus the
dt history.  The reference tree is needed only to (re)generate; the .npz
files are committed and used by tests on machines without it.

    python tests/golden/make_golden.py [name ...]
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import lare_oracle as lo  # noqa: E402
from oracle import dumpio  # noqa: E402
from oracle.dumpio import Dump  # noqa: E402

GEO_DOMAIN = [1.0, 2.0, 0.5, 1.5, 0.0, 0.5]
# (name, case, nx, ny, nz, steps, seed, b0[, options]); options: rke (0/1),
# geometry (0/1/2) and domain [x0, x1, y0, y1, z0, z1]
CASES = [
    ("ot_12x10x6_s5", "ot", 12, 10, 6, 5, 1, 0.0),
    ("ot_7x5x3_s3", "ot", 7, 5, 3, 3, 1, 0.0),
    ("ot_b0_10x10x4_s4", "ot", 10, 10, 4, 4, 1, 0.9 / (4 * np.pi) ** 0.5),
    ("rf_10x8x6_s4", "rf", 10, 8, 6, 4, 7, 0.0),
    ("harris_12x10x6_s4", "harris", 12, 10, 6, 4, 3, 0.0),
    # dimensions with fewer than three cells: 2.5-D (the reference's own
    # Orszag-Tang runs nz = 2) and 2-D; edge copies read their own output here
    ("ot_12x10x2_s4", "ot", 12, 10, 2, 4, 1, 0.0),
    ("ot_8x6x1_s3", "ot", 8, 6, 1, 3, 1, 0.0),
    ("harris_10x2x4_s3", "harris", 10, 2, 4, 3, 3, 0.0),
    # the remap kinetic-energy correction on (rke): the reference run on one
    # thread, where its atomic adds happen in loop order
    ("ot_rke_12x10x6_s5", "ot", 12, 10, 6, 5, 1, 0.0, {"rke": 1}),
    ("rf_rke_10x8x6_s4", "rf", 10, 8, 6, 4, 7, 0.0, {"rke": 1}),
    # cylindrical (1) and spherical (2) geometry on r in [1, 2], theta in
    # [0.5, 1.5], third coordinate in [0, 0.5]
    ("ot_cyl_12x10x6_s5", "ot", 12, 10, 6, 5, 1, 0.0, {"geometry": 1, "domain": GEO_DOMAIN}),
    ("rf_sph_10x8x6_s3", "rf", 10, 8, 6, 3, 7, 0.0, {"geometry": 2, "domain": GEO_DOMAIN}),
    ("harris_cyl_10x8x4_s3", "harris", 10, 8, 4, 3, 3, 0.0, {"geometry": 1, "domain": GEO_DOMAIN}),
    ("ot_sph_rke_10x8x6_s4", "ot", 10, 8, 6, 4, 1, 0.0, {"geometry": 2, "domain": GEO_DOMAIN, "rke": 1}),
    # Cartesian grids whose spacings are all one power of two (1/16, 1/8, 1,
    # 1/2): the GPU divides by multiplying with exact reciprocals there
    ("ot_p2_16x8x4_s4", "ot", 16, 8, 4, 4, 1, 0.0),
    ("rf_p2_rke_16x8x8_s4", "rf", 16, 8, 8, 4, 7, 0.0, {"rke": 1}),
    ("harris_p2_16x8x4_s3", "harris", 16, 8, 4, 3, 3, 0.0, {"domain": [-8.0, 8.0, -4.0, 4.0, 0.0, 2.0]}),
    # the LARE BC_OTHER conditions of the reference's LARE3DInitialConditions
    # package on every edge (walls in x for the velocities, plane copies
    # elsewhere), registered by that package itself in the reference run
    ("ot_lare_12x10x6_s5", "ot", 12, 10, 6, 5, 1, 0.0, {"lare_bcs": 1}),
    ("rf_lare_10x8x6_s4", "rf", 10, 8, 6, 4, 7, 0.0, {"lare_bcs": 1}),
    ("ot_lare_8x6x2_s3", "ot", 8, 6, 2, 3, 1, 0.0, {"lare_bcs": 1}),
    ("harris_lare_p2_16x8x4_s3", "harris", 16, 8, 4, 3, 3, 0.0,
     {"lare_bcs": 1, "domain": [-8.0, 8.0, -4.0, 4.0, 0.0, 2.0]}),
    ("ot_lare_rke_12x10x6_s4", "ot", 12, 10, 6, 4, 1, 0.0, {"lare_bcs": 1, "rke": 1}),
]
STATE = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz", "bx", "by", "bz"]
# (file, case, nx, ny, nz, steps, seed): the reference's full harness state
# (13 variables, step, time, last dt) after `steps` steps as a SAMSDUMP1
# restart file; ot_12x10x6_at3 continues to ot_12x10x6_s5 above.
RESTARTS = [("ot_12x10x6_at3.dump", "ot", 12, 10, 6, 3, 1)]
HARNESS = ["rho", "energy_electron", "energy_ion", "vx", "vy", "vz", "vx1", "vy1", "vz1", "bx", "by", "bz", "dm"]


def main(only=()):
    """Regenerate every fixture, or only the cases named in `only`."""
    lo.build()
    if not os.path.exists(lo.REF_BIN):
        raise SystemExit("reference harness not built (needs the reference tree)")
    for name, case, nx, ny, nz, steps, seed, b0, *opt in CASES:
        if only and name not in only:
            continue
        o = opt[0] if opt else {}
        rke, geometry, domain = o.get("rke", 0), o.get("geometry", 0), o.get("domain")
        lare_bcs = o.get("lare_bcs", 0)
        extra = (["--rke"] if rke else []) + (["--geometry", str(geometry)] if geometry else [])
        extra += ["--lare-bcs"] if lare_bcs else []
        if domain:
            extra += ["--domain"] + [repr(x) for x in domain]
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "d.dump")
            summary = lo.run_reference(case, nx, ny, nz, steps, path, seed=seed, b0=b0,
                                       extra=extra, threads=1 if rke else None)
            d = Dump(path)
            out = {}
            for f in STATE:
                out[f] = d.box(f)
            out["dts"] = np.array(d.header["dts"])
            meta = dict(case=case, nx=nx, ny=ny, nz=nz, steps=steps, seed=seed, b0=b0, rke=rke, geometry=geometry,
                        domain=domain, lare_bcs=lare_bcs,
                        time=summary["time"], generator="oracle/_ref/lare_ref (reference LARE3D)")
            out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            print(name, "dt", d.header["dt"])
    for fname, case, nx, ny, nz, steps, seed in RESTARTS:
        if only and fname not in only:
            continue
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "d.dump")
            lo.run_reference(case, nx, ny, nz, steps, path, seed=seed)
            d = Dump(path)
            header = {k: d.header[k] for k in ("nx", "ny", "nz", "step", "phase", "time", "dt", "dts")}
            header["generator"] = "oracle/_ref/lare_ref (reference LARE3D), harness variables only"
            dumpio.write(os.path.join(HERE, fname), header, {n: d.get(n) for n in HARNESS})
            print(fname, "step", d.header["step"], "dt", d.header["dt"])


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    return z, meta


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))


SAMS_BC_LARE_OTHER = 5  # include/sams_lare_layout.h


def apply_options(p, meta, b=None):
    """Set a case's rke / geometry / domain options (from a fixture's meta) on
    a parameter block of either ctypes binding, and, given its boundary
    conditions `b`, the LARE BC_OTHER condition on every edge of every field
    where the case asks for it (lare_bcs)."""
    p.rke = meta.get("rke", 0)
    p.geometry = meta.get("geometry", 0)
    d = meta.get("domain")
    if d:
        p.x_min, p.x_max, p.y_min, p.y_max, p.z_min, p.z_max = d
    if b is not None and meta.get("lare_bcs"):
        for f in range(len(b.kind)):
            for dim in range(3):
                for e in range(2):
                    b.kind[f][dim][e] = SAMS_BC_LARE_OTHER
    return p
