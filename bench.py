#!/usr/bin/env python
"""Benchmark of the B200 LARE3D timestep (one JSON line on rank 0).

Workload: the plain 256^3 periodic random-field cube (resistive MHD,
eta = 1e-4, seeded initial state), FP64.  A "step" is one full LARE3D
timestep (Lagrangian predictor + corrector + x/y/z remap) of that cube.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`value` is device-timed throughput in cell-updates/s with the state resident
in HBM; `e2e` is the same solve through the C ABI from pinned host buffers
(state upload, K steps each reading back dt, state download).  Under torchrun
every rank runs its own independent solve (replicas; the path does not shard
within a solve), time = max over ranks.  `--impl reference` times the
reference LARE3D CPU code (oracle/_ref/lare_ref_bench, built from the
reference sources) on this host's cores for the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 cell-updates/s plain vs batched (1 B200, 1e-10 rel); p50/p99 solve latency"
UNIT = "cell-updates/s"
# Compulsory FP64 HBM traffic of one cell-update: state read/write per
# phase, 8 B per value (dt pass 72, predictor 96, corrector 144, three sweeps
# 3 x 176 = 840 B), plus two resistive sub-steps 2 x 72 in resistive runs.
ALGO_BYTES_IDEAL, ALGO_BYTES_RESISTIVE = 840, 984


class Workload:
    """One single-solve configuration: case, grid, algorithmic bytes per
    cell-update and its description (seeded synthetic initial state)."""

    def __init__(self, name, case, grid, algo_bytes, text, tag):
        self.name, self.case, self.grid, self.algo_bytes, self.text, self.tag = \
            name, case, tuple(grid), algo_bytes, text, tag

    @property
    def cells(self):
        return float(self.grid[0]) * self.grid[1] * self.grid[2]


def workload(args):
    """--config c0 / c1 / c2, or the random-field cube of edge --edge (c1's
    form; 256 = c1 itself)."""
    if args.config == "c0":
        return Workload("c0", "ot", (128, 128, 4), ALGO_BYTES_IDEAL,
                        "plain LARE3D step, Orszag-Tang 128x128x4 periodic [0,1]^2 x [0,4/128], gamma=5/3, "
                        "B0=1/sqrt(4 pi), visc1=0.1, visc2=0.5, ideal MHD", "ot128x128x4")
    if args.config == "c2":
        return Workload("c2", "harris", (512, 256, 64), ALGO_BYTES_RESISTIVE,
                        "plain LARE3D step, Harris current sheet 512x256x64 over [-10,10]x[-5,5]x[0,2.5], "
                        "beta=0.1, 1% seeded velocity perturbation, eta=1e-3, conducting y walls", "harris512x256x64")
    n = args.edge
    return Workload("c1" if n == 256 else f"rf{n}", "rf", (n, n, n), ALGO_BYTES_RESISTIVE,
                    f"plain LARE3D step, {n}^3 periodic random-field cube [0,1]^3, rho=1, p=0.1, "
                    "|B|rms=0.1, |v|rms=0.05, k=1..8, gamma=5/3, eta=1e-4 (resistive), seeded synthetic IC",
                    f"rf{n}")


def l2_note(w):
    """How the timed inputs relate to the 126 MB L2 of a B200."""
    nx, ny, nz = w.grid
    field_mb = (nx + 5) * (ny + 5) * (((nz + 6) + 7) // 8 * 8) * 8 / 1e6
    if field_mb * 32 > 126:
        return f"inputs larger than L2 (each field {field_mb:.0f} MB, 32 x {field_mb:.0f} MB resident)"
    return f"inputs fit in L2 (each field {field_mb:.1f} MB): not a full-size run"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sams", choices=["sams", "reference"])
    ap.add_argument("--edge", type=int, default=256, help="cube edge of the plain workload")
    ap.add_argument("--config", default="c1", choices=["c0", "c1", "c2"],
                    help="single-solve configuration of the plain line (c1: the 256^3 random-field cube)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=300, help="steps per solve of the batched workload (its configuration: 300)")
    ap.add_argument("--only-batched", action="store_true",
                    help="run only the batched workload's timed steps (for profiling) and print its line")
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-lookahead", type=int, default=4,
                    help="generated requests kept queued ahead of admission")
    ap.add_argument("--only-served", action="store_true",
                    help="run only the served workload (config 4) and print its line")
    ap.add_argument("--serve-max-cells", type=int, default=16 << 20)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if args.impl == "sams":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(w):
    """DRAM bytes per step from the committed ncu summary of this workload,
    if one exists (profiles/lare_step_<tag>_traffic.json)."""
    path = os.path.join(ROOT, "profiles", f"lare_step_{w.tag}_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)["dram_bytes_per_step"]
    except Exception:
        return None


def fp64_roof(w, ms_per_step, rates):
    """The step's FP64 compute roof: its fp64-pipe warp instructions (ncu
    sm__inst_executed_pipe_fp64 over one step of this workload, committed in
    profiles/lare_step_<tag>_fp64.json) at the measured fused multiply-add
    rate (one warp instruction = 32 thread operations), against the step's
    measured time."""
    path = os.path.join(ROOT, "profiles", f"lare_step_{w.tag}_fp64.json")
    try:
        with open(path) as f:
            inst = float(json.load(f)["fp64_pipe_warp_inst_per_step"])
    except Exception:
        return None
    if not rates or not rates.get("fma"):
        return None
    roof_ms = inst * 32 / (rates["fma"] * 1e9) * 1e3
    return {"fp64_pipe_warp_inst_per_step": inst, "roof_ms": roof_ms, "frac": roof_ms / ms_per_step,
            "source": os.path.relpath(path, ROOT)}


def cpu_reference(w, steps, threads=None):
    """Time the reference LARE3D CPU code (or, without its binary, the C
    restatement) on this host for `steps` steps of workload w."""
    from oracle import lare_oracle as lo
    threads = threads or os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="spread")
    binary, isa = lo.reference_bench_binary()
    nx, ny, nz = w.grid
    if os.path.exists(binary):
        cmd = [binary, "--case", w.case, "--nx", str(nx), "--ny", str(ny), "--nz", str(nz),
               "--steps", str(steps), "--seed", "1", "--quiet"]
        out = subprocess.run(cmd, check=True, capture_output=True, text=True, env=env).stdout
        rec = json.loads(out.strip().splitlines()[-1])
        return rec["step_seconds"], "reference", threads, isa
    # the C restatement (ctypes, OpenMP)
    p, b = lo.case_setup(w.case, nx, ny, nz)
    o = lo.Oracle(p, b, lo.case_fields(w.case, p, seed=1))
    secs = []
    for _ in range(steps):
        t0 = time.perf_counter()
        o.step(1)
        secs.append(time.perf_counter() - t0)
    return secs, "port", threads, "-O2 C restatement"


def max_over_ranks(pg, ms, device):
    """The slowest rank's time: replicas finish together only when the last
    one does.  Every rank takes part (the same collective on every rank)."""
    if pg is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, cells, steps, ms):
    """Whole-job cell-updates/s of `world` independent replicas, each
    advancing `cells` cells `steps` steps, in `ms` (max over ranks)."""
    return world * cells * steps / (ms / 1e3)


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    w = workload(args)
    total = args.warmup + args.steps
    secs, kind, threads, isa = cpu_reference(w, total)
    timed = secs[args.warmup:]
    cells = w.cells
    value = cells * len(timed) / sum(timed)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(timed) / len(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": w.text, "case": w.case, "grid": list(w.grid), "parallelism": "cpu-openmp"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "isa": isa,
                         "sample": f"{len(timed)} timed steps of the {w.name} workload after {args.warmup} "
                                   "warm-up steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_sams(args, world, rank, local, pg):
    import torch
    from sams_b200 import lare

    torch.cuda.set_device(local)
    w = workload(args)
    cells = w.cells
    p, b = lare.case_setup(w.case, *w.grid)
    fields = lare.case_fields(w.case, p, seed=1 + rank)
    # a dedicated stream: the solver launches on it and the events bracket it
    stream = torch.cuda.Stream(device=local)

    # ---------------- device-resident throughput ----------------
    s = lare.LARE3D(p, b, device=local)
    s.set_stream(stream.cuda_stream)
    s.upload_all(fields)
    for _ in range(args.warmup):
        s.step(1, graph=True)
    s.synchronize()
    launches = s.launches_per_step
    if pg is not None:
        pg.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.step(1, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = max_over_ranks(pg, e0.elapsed_time(e1), "cuda")
    if pg is not None:
        pg.barrier()
    s.synchronize()
    ms_per_step = ms / args.steps
    value = replica_throughput(world, cells, args.steps, ms)
    phases = s.phase_times()
    s.synchronize()
    s.close()
    # the compute roof's denominators: measured FP64 rates of this GPU
    fp64 = {k: v / 1e9 for k, v in lare.fp64_rates(local).items()} if rank == 0 else None

    # ---------------- end to end through the C ABI ----------------
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(fields[f]).pin_memory() for f in range(lare.NFIELDS)]
        state = [f for f in range(lare.NFIELDS) if lare.FIELD_NAMES[f] in
                 ("rho", "energy_electron", "energy_ion", "vx", "vy", "vz", "bx", "by", "bz")]
        outs = [torch.empty_like(pinned[f]).pin_memory() for f in state]
        s2 = lare.LARE3D(p, b, device=local)
        s2.set_stream(stream.cuda_stream)
        s2.upload_all(fields)              # the solve's scratch/aux fields
        s2.step(1, graph=True)             # graph recorded outside the timed region
        s2.synchronize()
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()
        L = lare.lib()
        h = s2.handle
        e0.record(stream)
        for f in state:
            lare._check(L.sams_lare_upload_field(h, f, ctypes_addr(pinned[f])))
        dts = []
        for _ in range(args.steps):
            lare._check(L.sams_lare_step_graph(h, 1))
            dts.append(s2.dt)
        for f, o in zip(state, outs):
            lare._check(L.sams_lare_download_field(h, f, ctypes_addr(o)))
        e1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(pg, e0.elapsed_time(e1), "cuda")
        box_bytes = int(np.prod(lare.box_shape(*w.grid))) * 8
        e2e = {"value": replica_throughput(world, cells, args.steps, ems), "unit": UNIT,
               "h2d_bytes_per_step": len(state) * box_bytes / args.steps,
               "d2h_bytes_per_step": (len(state) * box_bytes + 8 * args.steps) / args.steps,
               "what": "state upload from pinned host memory, K steps each reading dt back, state download"}
        s2.close()

    # the batched and served workloads are single-GPU configurations
    batched = None
    if not args.no_batched and world == 1:
        batched = run_batched(args, local, stream)
    served = None
    if args.serve_seconds > 0 and world == 1:
        served = run_served(args, local)

    if rank != 0:
        return
    peak, peak_kind = measured_peak()
    achieved = w.algo_bytes * cells / (ms_per_step / 1e3) / 1e9
    traffic = ncu_traffic(w)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind,
                "kernel": "one LARE3D timestep (a CUDA graph of %d kernels)" % launches,
                "algorithmic_bytes_per_launch": w.algo_bytes * cells}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            csteps = max(4, min(50, int(6.7e7 / cells)))  # about 10 s of host time
            secs, kind, threads, isa = cpu_reference(w, csteps)
            cpu = {"value": cells * len(secs) / sum(secs), "unit": UNIT, "cores": threads, "kind": kind,
                   "isa": isa, "sample": f"{csteps} steps of the {w.name} workload (all steps timed)"}
        except Exception as ex:  # report, do not fail the GPU line
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {ex}"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w.text, "case": w.case, "grid": list(w.grid),
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": l2_note(w)},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": launches * args.steps,
        "batched": batched,
        "served": served,
        "phases_ms": dict(zip(["lagrangian", "corrector", "remap_x", "remap_y", "remap_z"], phases)),
        "fp64_rates_gops": fp64,
        "fp64_roof": fp64_roof(w, ms_per_step, fp64),
    }
    print(json.dumps(line), flush=True)


def run_batched(args, local, stream, sequential=True):
    """Config 3: 64 independent Orszag-Tang solves, n x n x 4 with n drawn
    log-uniformly from 64..512 and B0 uniformly from [0.5, 1.5]/sqrt(4 pi)
    (seeded).  Throughput of the batch (one persistent launch per phase over
    all solves, autotuned tiling, one graph per step) against the same solves
    run one after another with the plain single-solve path."""
    import math
    import torch
    from sams_b200 import lare

    rng = np.random.default_rng(2024)
    ns = [int(round(64 * 8 ** u)) for u in rng.random(64)]
    b0s = rng.uniform(0.5, 1.5, 64) / math.sqrt(4 * math.pi)
    K = args.batch_steps
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    cells = [n * n * 4 for n in ns]

    # plain, one solve after another
    seq_ms = 0.0
    for n, b0 in zip(ns, b0s) if sequential else []:
        p, b = lare.case_setup("ot", n, n, 4, b0)
        s = lare.LARE3D(p, b, device=local)
        s.set_stream(stream.cuda_stream)
        s.upload_all(lare.case_fields("ot", p, seed=1, b0=b0))
        s.step(1, graph=True)
        s.synchronize()
        e0.record(stream)
        for _ in range(K):
            s.step(1, graph=True)
        e1.record(stream)
        torch.cuda.synchronize()
        seq_ms += e0.elapsed_time(e1)
        s.close()

    # batched
    bt = lare.Batch(device=local)
    bt.set_stream(stream.cuda_stream)
    for n, b0 in zip(ns, b0s):
        p, b = lare.case_setup("ot", n, n, 4, b0)
        bt.add(p, b, lare.case_fields("ot", p, seed=1, b0=b0))
    if sequential:
        tile, bps, _ = bt.autotune(trial_steps=2)
    else:  # the tiling the autotuner picks on B200 for this batch
        tile, bps = 8, 8
        bt.set_tuning(tile, bps)
    for _ in range(args.warmup):
        bt.step(1, graph=True)
    bt.synchronize()
    e0.record(stream)
    for _ in range(K):
        bt.step(1, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    bat_ms = e0.elapsed_time(e1)
    dev_bytes = bt.device_bytes
    bt.close()
    total = float(sum(cells)) * K
    seq = total / (seq_ms / 1e3) if sequential else None
    bat = total / (bat_ms / 1e3)
    return {"workload": "64 Orszag-Tang solves n x n x 4, n log-uniform in [64,512] (seeded), "
                        "B0 uniform in [0.5,1.5]/sqrt(4 pi), per-solve dt",
            "steps_each": K, "cells_total": int(sum(cells)), "value": bat, "unit": UNIT,
            "plain_sequential": seq, "speedup_vs_plain_sequential": bat / seq if seq else None,
            "ms_per_batched_step": bat_ms / K, "tile_planes": tile, "blocks_per_sm": bps,
            "device_bytes": dev_bytes}


def run_served(args, local):
    """Config 4: Poisson arrivals (rate args.rate over args.serve_seconds) of
    random-field cube solves (edge drawn from {32,64,96,128,192}, 100..2000
    steps, resistive), each with its own seed, admitted in arrival order by
    an HBM budget into one continuously batched server.  A background thread
    generates each request's initial state on the host once the request has
    arrived, keeping a few generated requests queued ahead of admission (the
    rest wait as arrivals, in order).  Latency is measured from ARRIVAL to
    the result on the host, so it includes waiting for generation and for
    admission.  Reports p50/p99 over the requests completed in the window and
    the delivered cell-updates/s."""
    import random
    from sams_b200 import lare

    rng = random.Random(7)
    edges = [32, 64, 96, 128, 192]
    window = args.serve_seconds
    arrivals, t = [], rng.expovariate(args.rate)
    while t < window:  # (arrival time, edge, steps, seed)
        arrivals.append((t, rng.choice(edges), rng.randint(100, 2000), 1000 + len(arrivals)))
        t += rng.expovariate(args.rate)
    setups = {e: lare.case_setup("rf", e, e, e) for e in edges}
    srv = lare.Server(int(args.budget_gb * (1 << 30)), device=local, max_cells=args.serve_max_cells)
    lock = threading.Lock()
    stop = threading.Event()
    open_tickets = {}  # ticket -> (arrival time, submit time)
    gen = {"submitted": 0, "gen_s": 0.0}
    t0 = time.perf_counter()

    def generator():
        for ta, e, steps, seed in arrivals:
            while not stop.is_set() and time.perf_counter() - t0 < ta:
                time.sleep(min(0.01, max(0.0, ta - (time.perf_counter() - t0))))
            while not stop.is_set() and srv.stats()["queued"] >= args.serve_lookahead:
                time.sleep(0.005)
            if stop.is_set():
                return
            p, b = setups[e]
            g0 = time.perf_counter()
            ic = lare.case_fields("rf", p, seed=seed)
            gen["gen_s"] += time.perf_counter() - g0
            tk = srv.submit(p, b, ic, steps)
            with lock:
                open_tickets[tk] = (ta, time.perf_counter() - t0)
                gen["submitted"] += 1

    th = threading.Thread(target=generator, daemon=True)
    th.start()
    lat = []
    while time.perf_counter() - t0 < window:
        with lock:
            items = list(open_tickets.items())
        for tk, (ta, ts) in items:
            st, lib_lat = srv.poll(tk)
            if st in ("done", "failed"):
                if st == "done":
                    lat.append(ts - ta + lib_lat)  # arrival -> submit, then submit -> result on the host
                srv.release(tk)
                with lock:
                    del open_tickets[tk]
        time.sleep(0.005)
    stop.set()
    th.join()
    stats = srv.stats()
    srv.close()
    offered = sum(float(e) ** 3 * steps for _, e, steps, _ in arrivals)
    lat.sort()

    def pct(q):
        return lat[min(len(lat) - 1, int(q * len(lat)))] if lat else None
    return {"workload": "Poisson %g req/s, rf cubes edge U{32,64,96,128,192}, steps U[100,2000], seed per "
                        "request, eta=1e-4, %g GB HBM budget, %g s window" % (args.rate, args.budget_gb, window),
            "arrived": len(arrivals), "submitted": gen["submitted"], "completed": len(lat),
            "failed": stats["failed"], "queued_at_end": stats["queued"], "running_at_end": stats["running"],
            "p50_latency_s": pct(0.50), "p99_latency_s": pct(0.99),
            "mean_latency_s": sum(lat) / len(lat) if lat else None,
            "latency_from": "arrival (includes waiting for initial-state generation and admission)",
            "value": stats["cell_updates_per_s"], "unit": UNIT,
            "offered_cell_updates_per_s": offered / window,
            "host_ic_generation_s": gen["gen_s"],
            "admission": "arrival order; HBM budget %g GB; at most %d interior cells running at once"
                         % (args.budget_gb, args.serve_max_cells),
            "note": "offered load exceeds one B200's capacity, so latency includes growing queueing"}


def ctypes_addr(t):
    import ctypes
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), ctypes.POINTER(ctypes.c_double))


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        elif args.only_served:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps({"served": run_served(args, local)}), flush=True)
        elif args.only_batched:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps({"batched": run_batched(args, local, torch.cuda.Stream(device=local), sequential=False)}))
        else:
            run_sams(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
