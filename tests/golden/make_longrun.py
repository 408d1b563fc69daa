"""Write the long-run records (tests/golden/*.longrun.npz) from the REFERENCE.

Runs oracle/_ref/lare_ref (the unmodified reference LARE3D sources compiled
by oracle/Makefile, driven by its own SAMS::runner) on each benchmark
configuration for its full stated step count, with the seeded initial state
the GPU tests use, and records the final state's hashes, samples, dt
history, mass and energy budget (tests/golden/longrun.py).  The 256^3 and
512x256x64 runs take tens of minutes on an 8-core host.

    python tests/golden/make_longrun.py [name ...] [--dump name=PATH ...]

--dump reuses a SAMSDUMP1 file the reference harness already wrote for that
run (lare_ref ... --dump PATH) instead of running it again.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import longrun as lr  # noqa: E402
from oracle import lare_oracle as lo  # noqa: E402
from oracle.dumpio import Dump  # noqa: E402


def cell_volume(p):
    return ((p.x_max - p.x_min) / p.nx) * ((p.y_max - p.y_min) / p.ny) * ((p.z_max - p.z_min) / p.nz)


def record(name, case, nx, ny, nz, steps, seed, dump_path):
    p, _ = lo.case_setup(case, nx, ny, nz)
    dv = cell_volume(p)
    ic = lo.case_fields(case, p, seed=seed)
    m0 = lr.mass(ic[0], nx, ny, nz, dv)
    del ic
    d = Dump(dump_path)
    assert d.header["step"] == steps, (name, d.header["step"])
    fields = lr.field_record(lambda f: d.get(f)[0])
    boxes = {}

    def box(f):
        if f not in boxes:
            boxes[f] = d.box(f)
        return boxes[f]
    eb = lr.energy_budget(box, nx, ny, nz, dv, p.mu0)
    meta = dict(case=case, nx=nx, ny=ny, nz=nz, steps=steps, seed=seed,
                time=d.header["time"], dts=list(d.header["dts"]),
                mass_initial=m0, mass_final=lr.mass(box("rho"), nx, ny, nz, dv),
                energy=dict(zip(("internal", "kinetic", "magnetic"), eb)),
                generator="oracle/_ref/lare_ref (reference LARE3D, -O2 -ffp-contract=off)")
    lr.save(name, meta, fields)
    print(name, "steps", steps, "dt", meta["dts"][-1], "mass drift", (meta["mass_final"] - m0) / m0)


def main(argv):
    dumps, only = {}, []
    it = iter(argv)
    for a in it:
        if a == "--dump":
            k, v = next(it).split("=", 1)
            dumps[k] = v
        else:
            only.append(a)
    for name, case, nx, ny, nz, steps, seed in lr.RUNS:
        if only and name not in only:
            continue
        if name in dumps:
            record(name, case, nx, ny, nz, steps, seed, dumps[name])
            continue
        if not os.path.exists(lo.REF_BIN):
            raise SystemExit("reference harness not built (needs the reference tree)")
        with tempfile.TemporaryDirectory() as td:
            dp = os.path.join(td, "d.dump")
            lo.run_reference(case, nx, ny, nz, steps, dp, seed=seed)
            record(name, case, nx, ny, nz, steps, seed, dp)


if __name__ == "__main__":
    main(sys.argv[1:])
