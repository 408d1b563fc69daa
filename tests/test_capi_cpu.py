"""The C-ABI library loads and exports every function include/*.h declares
(no GPU needed: nothing here launches a kernel)."""
import ctypes
import os
import re

import numpy as np
import pytest

from sams_b200 import lare

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_functions():
    names = set()
    for h in os.listdir(INCLUDE):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ \*]*?\b(sams_[a-z0-9_]+)\s*\(", text, flags=re.M):
            if "static inline" in text[max(0, m.start() - 40):m.start() + 40]:
                continue
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_functions():
    names = declared_functions()
    assert "sams_lare_create" in names and "sams_lare_step" in names
    assert "sams_ic_orszag_tang" in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    L = lare.lib()
    assert hasattr(L, name), f"{name} declared in include/ but not exported by {lare.LIB_PATH}"


def test_abi_version_and_error_string():
    L = lare.lib()
    assert L.sams_lare_abi_version() == 100
    assert isinstance(L.sams_lare_last_error(), bytes)


def test_create_rejects_bad_params_without_gpu():
    p, b = lare.case_setup("ot", 8, 8, 4)
    p.geometry = 3               # no such geometry (0, 1, 2 are built)
    with pytest.raises(lare.LareError) as e:
        lare.LARE3D(p, b)
    assert e.value.status == -4
    p.geometry = 0
    p.nx = 0
    with pytest.raises(lare.LareError):
        lare.LARE3D(p, b)


def test_product_ic_matches_checker_ic():
    """Both builds of the IC generator give identical states."""
    from oracle import lare_oracle as lo
    for case in ["ot", "rf", "harris"]:
        p, _ = lare.case_setup(case, 10, 8, 6)
        a = lare.case_fields(case, p, seed=5)
        p2, _ = lo.case_setup(case, 10, 8, 6)
        b = lo.case_fields(case, p2, seed=5)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_random_field_is_divergence_free_and_normalised():
    p, _ = lare.case_setup("rf", 16, 16, 16)
    f = lare.case_fields("rf", p, seed=3)
    bx, by, bz = f[9], f[10], f[11]
    d = 1.0 / 16
    # div B at cells 1..n: (bx(i)-bx(i-1))/dx + ... ; box index = i + 2
    s = slice(3, 19)
    sm = slice(2, 18)
    div = (bx[s, s, s] - bx[sm, s, s]) / d + (by[s, s, s] - by[s, sm, s]) / d + (bz[s, s, s] - bz[s, s, sm]) / d
    bmag = np.sqrt((bx[s, s, s] ** 2 + by[s, s, s] ** 2 + bz[s, s, s] ** 2).mean())
    assert abs(bmag - 0.1) < 1e-12
    assert np.abs(div).max() < 1e-12 * 16 * 0.1 * 100
    v = np.sqrt((f[3][s, s, s] ** 2 + f[4][s, s, s] ** 2 + f[5][s, s, s] ** 2).mean())
    assert abs(v - 0.05) < 1e-12


def test_harris_pressure_balance():
    p, _ = lare.case_setup("harris", 16, 16, 4)
    f = lare.case_fields("harris", p, seed=1)
    g = 5.0 / 3.0
    rho, ee, ei, bx = f[0][2:-2, 2:-2, 2:-2], f[1][2:-2, 2:-2, 2:-2], f[2][2:-2, 2:-2, 2:-2], f[9][2:-2, 2:-2, 2:-2]
    ptot = (g - 1) * rho * (ee + ei) + 0.5 * bx ** 2
    assert np.allclose(ptot, 0.55, rtol=0, atol=1e-14)


@pytest.mark.parametrize("n,own_stream", [((32, 32, 32), False), ((64, 64, 64), False), ((96, 96, 96), True),
                                          ((192, 192, 192), True), ((256, 256, 4), False), ((20, 16, 24), True)])
def test_serve_footprint_follows_the_path_a_solve_takes(n, own_stream):
    """The server charges a solve the device bytes of the path it runs on:
    its own solver (padded rows, 32 arrays, host-transfer staging) when its
    z lines fill the fused kernels' tiles (nz >= 23 with full tiles), else a
    batch slot (dense rows).  Host arithmetic only, no GPU."""
    p, _ = lare.case_setup("rf", *n)
    got = lare.solve_bytes(p)
    nx, ny, nz = n
    zrow = (nz + 6 + 7) // 8 * 8
    solver = (32 * (nx + 5) * (ny + 5) * zrow + (nx + 5) * (ny + 5) * (nz + 5) + 6 * (nx + ny + nz + 18)) * 8
    batch_arrays = 32 * (nx + 5) * (ny + 5) * (nz + 5) * 8
    if own_stream:
        assert solver <= got <= solver + 8192
    else:
        assert batch_arrays <= got < solver
