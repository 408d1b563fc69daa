"""Reader for SAMSDUMP1 state dumps written by oracle/ref_harness.cpp.

Test infrastructure only.  A dump is the text line ``SAMSDUMP1``, one JSON
header line (grid size, step, dt history and an array directory with each
array's own index bounds), then the arrays as little-endian float64 in the
order of the directory, each laid out row-major (last index fastest) over its
bounds.
"""
import json

import numpy as np


def write(path, header, arrays):
    """Write a SAMSDUMP1 file: `header` (dict without "arrays") plus the
    named arrays as (array, lower_bounds) pairs, each over its own bounds."""
    entries, blobs, off = [], [], 0
    for name, (arr, lb) in arrays.items():
        arr = np.ascontiguousarray(arr, dtype="<f8")
        ub = [l + s - 1 for l, s in zip(lb, arr.shape)]
        entries.append({"name": name, "rank": arr.ndim, "lb": list(lb) + [0] * (3 - arr.ndim),
                        "ub": ub + [0] * (3 - arr.ndim), "offset": off})
        blobs.append(arr.tobytes())
        off += arr.nbytes
    h = dict(header)
    h["arrays"] = entries
    with open(path, "wb") as f:
        f.write(b"SAMSDUMP1\n")
        f.write(json.dumps(h, separators=(",", ":")).encode() + b"\n")
        for b in blobs:
            f.write(b)


class Dump:
    def __init__(self, path):
        with open(path, "rb") as f:
            magic = f.readline()
            if magic.strip() != b"SAMSDUMP1":
                raise ValueError(f"{path}: not a SAMSDUMP1 file")
            self.header = json.loads(f.readline())
            self._data = f.read()
        self.nx = self.header["nx"]
        self.ny = self.header["ny"]
        self.nz = self.header["nz"]
        self.arrays = {a["name"]: a for a in self.header["arrays"]}

    def names(self):
        return list(self.arrays)

    def bounds(self, name):
        a = self.arrays[name]
        r = a["rank"]
        return a["lb"][:r], a["ub"][:r]

    def get(self, name):
        """Return (array, lower_bounds) for a named array."""
        a = self.arrays[name]
        r = a["rank"]
        lb, ub = a["lb"][:r], a["ub"][:r]
        shape = tuple(u - l + 1 for l, u in zip(lb, ub))
        n = int(np.prod(shape))
        arr = np.frombuffer(self._data, dtype="<f8", count=n, offset=a["offset"]).reshape(shape)
        return arr, lb

    def box(self, name):
        """Return a 3-D array over the -2..n+2 box; entries outside the
        array's own bounds are NaN."""
        arr, lb = self.get(name)
        out = np.full((self.nx + 5, self.ny + 5, self.nz + 5), np.nan)
        sl = tuple(slice(l + 2, l + 2 + s) for l, s in zip(lb, arr.shape))
        out[sl] = arr
        return out
