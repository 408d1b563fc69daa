"""Build the B200 LARE3D library (libsams_lare.so) in-tree.

The library is compiled for sm_100a only, with --fmad=false so that no
multiply-add is contracted (the timestep must reproduce the reference's
rounding term by term).  Output: sams_b200/_lib/libsams_lare.so.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libsams_lare.so")

CU_SOURCES = ["lare_solver.cu", "lare_batch.cu", "lare_serve.cu", "lare_capi.cu", "lare_noalloc.cu", "lare_dump.cu",
              "lare_router.cu", "lare_dist.cu", "lare_fp64_roof.cu"]
C_SOURCES = ["lare_ic.c"]
HEADERS = ["lare_device.cuh", "lare_ops.cuh", "lare_solver.cuh", "lare_batch.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(LIBDIR, exist_ok=True)
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    deps = [os.path.join(CSRC, s) for s in CU_SOURCES + C_SOURCES + HEADERS]
    deps += [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include")) if h.endswith(".h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objs, cmds = [], []
    for src in CU_SOURCES:
        obj = os.path.join(LIBDIR, src + ".o")
        cmds.append([nvcc()] + NVCC_FLAGS + inc + ["-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    for src in C_SOURCES:
        obj = os.path.join(LIBDIR, src + ".o")
        cmds.append(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fPIC", "-fopenmp"] + inc +
                    ["-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(8, len(cmds))) as ex:
        list(ex.map(lambda c: _run(c, verbose), cmds))
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + \
          ["-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
    _run(cmd, verbose)
    return LIB


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]))
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
