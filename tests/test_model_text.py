"""The text model readers of the drop-in programs (sm_read_model_a, _e and
_ecyl, host/sm_io.c) on the CPU: the values after the header, parsed on host
threads, equal a correctly rounded parse of the same text bit for bit, and
the reference's rules hold (io_utils.c:892-1094): one column (a row for the
cylindrical models) followed by nothing that reads as a number is a profile
replicated over the grid; fewer numbers than needed, or a token that is not a
number, is an error."""
import ctypes as C
import os

import numpy as np
import pytest

from seismod_b200 import _lib as L


class Grid(C.Structure):
    _fields_ = [("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double)]


def _read(path):
    lib = L.load()
    f = lib.sm_read_model_a
    f.argtypes = [C.c_char_p, C.POINTER(Grid), C.POINTER(C.POINTER(C.c_double)),
                  C.POINTER(C.POINTER(C.c_double))]
    f.restype = C.c_int
    g = Grid()
    vp, rho = C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
    rc = f(path.encode(), C.byref(g), C.byref(vp), C.byref(rho))
    if rc:
        return rc, None, None, g
    n = g.nx * g.ny * g.nz
    a = np.ctypeslib.as_array(vp, shape=(n,)).copy()
    b = np.ctypeslib.as_array(rho, shape=(n,)).copy()
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    libc.free(C.cast(vp, C.c_void_p))
    libc.free(C.cast(rho, C.c_void_p))
    return rc, a, b, g


def _header(shape):
    nx, ny, nz = shape
    return f"{nx} {ny} {nz}\n5.0 5.0 5.0\n0.0 0.0 0.0\nisotropic_acoustic_3d\n"


def _body(vp, rho, rng, fmts=("%.17g", "%g", "%.6e", "%.3f")):
    seps = [" ", "\t", "  ", " \t "]
    ends = ["\n", "\r\n", " \n", "\n\n"]
    lines = []
    for k, (a, b) in enumerate(zip(vp, rho)):
        fa = fmts[k % len(fmts)]
        fb = fmts[(k // 3) % len(fmts)]
        lines.append((fa % a) + seps[k % len(seps)] + (fb % b) + ends[(k // 7) % len(ends)])
    return "".join(lines)


def _expect(text_body, count):
    toks = text_body.split()[: 2 * count]
    v = np.array([float(t) for t in toks])   # correctly rounded, as strtod
    return v[0::2], v[1::2]


@pytest.mark.timeout(120)
def test_full_model_equals_a_correctly_rounded_parse(tmp_path):
    rng = np.random.default_rng(11)
    shape = (23, 37, 61)   # 51,911 cells, a few MB of text: parsed on several threads
    n = int(np.prod(shape))
    vp = 1500 + 3000 * rng.random(n)
    rho = 1800 + 500 * rng.random(n)
    body = _body(vp, rho, rng)
    path = os.path.join(tmp_path, "m.txt")
    with open(path, "w", newline="") as f:
        f.write(_header(shape) + body + "trailing words are ignored\n")
    assert os.path.getsize(path) > 1 << 20
    rc, a, b, g = _read(path)
    assert rc == 0 and (g.nx, g.ny, g.nz) == shape
    ea, eb = _expect(body, n)
    np.testing.assert_array_equal(a, ea)
    np.testing.assert_array_equal(b, eb)


@pytest.mark.parametrize("tail", ["", "end of profile\n", "\n\n  \n"])
def test_one_column_is_a_replicated_profile(tmp_path, tail):
    rng = np.random.default_rng(12)
    shape = (4, 3, 9)
    vp = 1500 + 3000 * rng.random(shape[2])
    rho = 1800 + 500 * rng.random(shape[2])
    body = _body(vp, rho, rng)
    path = os.path.join(tmp_path, "p.txt")
    with open(path, "w", newline="") as f:
        f.write(_header(shape) + body + tail)
    rc, a, b, _ = _read(path)
    assert rc == 0
    ea, eb = _expect(body, shape[2])
    np.testing.assert_array_equal(a, np.tile(ea, shape[0] * shape[1]))
    np.testing.assert_array_equal(b, np.tile(eb, shape[0] * shape[1]))


def test_short_or_malformed_models_are_errors(tmp_path):
    rng = np.random.default_rng(13)
    shape = (3, 4, 5)
    n = int(np.prod(shape))
    vp = 1500 + 3000 * rng.random(n)
    rho = 1800 + 500 * rng.random(n)
    body = _body(vp, rho, rng)
    toks = body.split()
    cases = {
        "short": " ".join(toks[:-3]),                       # more than a column, fewer than all
        "half_column": " ".join(toks[: shape[2]]),          # not even one column
        "bad_token": " ".join(toks[:40] + ["12abc"] + toks[41:]),
        "odd_after_column": " ".join(toks[: 2 * shape[2]] + ["7.5"]),
    }
    for name, text in cases.items():
        path = os.path.join(tmp_path, f"{name}.txt")
        with open(path, "w") as f:
            f.write(_header(shape) + text + "\n")
        rc, _, _, _ = _read(path)
        assert rc == L.SM_EIO, name


def _read3(fn, path):
    lib = L.load()
    f = getattr(lib, fn)
    P = C.POINTER(C.c_double)
    f.argtypes = [C.c_char_p, C.POINTER(Grid), C.POINTER(P), C.POINTER(P), C.POINTER(P)]
    f.restype = C.c_int
    g = Grid()
    ptrs = [P(), P(), P()]
    rc = f(path.encode(), C.byref(g), *[C.byref(p) for p in ptrs])
    if rc:
        return rc, None, g
    n = g.nx * g.nz
    out = [np.ctypeslib.as_array(p, shape=(n,)).copy().reshape(g.nx, g.nz) for p in ptrs]
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    for p in ptrs:
        libc.free(C.cast(p, C.c_void_p))
    return rc, out, g


@pytest.mark.timeout(120)
@pytest.mark.parametrize("fn,kw,rows_are_z", [("sm_read_model_e", "isotropic_elastic", False),
                                              ("sm_read_model_ecyl", "isotropic_elastic_cyl", True)])
@pytest.mark.parametrize("profile", [False, True])
def test_2d_models_equal_a_correctly_rounded_parse(tmp_path, fn, kw, rows_are_z, profile):
    # e_iso files list x columns (z fast, io_utils.c:892-947); e_cyl_iso files
    # list z rows (r fast, io_utils.c:949-991); both store [x][z].  A profile
    # is the first column (e_iso) or row (e_cyl_iso), copied over the grid.
    rng = np.random.default_rng(14)
    nx, nz = (301, 211) if not profile else (37, 23)   # the full case: several MB, threads
    fields = [1500 + 3000 * rng.random((nx, nz)), 900 + 1500 * rng.random((nx, nz)),
              1800 + 500 * rng.random((nx, nz))]
    order = [f.T.reshape(-1) if rows_are_z else f.reshape(-1) for f in fields]
    ncells = (nx if rows_are_z else nz) if profile else nx * nz
    fmts = ("%.17g", "%g", "%.6e", "%.3f")
    seps = [" ", "\t", "  "]
    lines = []
    for k in range(ncells):
        lines.append(seps[k % 3].join(fmts[(k + f) % 4] % order[f][k] for f in range(3)) + "\n")
    body = "".join(lines)
    path = os.path.join(tmp_path, "m.txt")
    with open(path, "w") as f:
        f.write(f"{nx} {nz}\n1.0 1.0\n0.0 0.0\n{kw}\n" + body)
    rc, out, g = _read3(fn, path)
    assert rc == 0 and (g.nx, g.nz) == (nx, nz)
    v = np.array([float(t) for t in body.split()])
    for f in range(3):
        got = v[f::3]
        if profile and rows_are_z:
            want = np.repeat(got[:, None], nz, axis=1)            # row 0 down every row
        elif profile:
            want = np.repeat(got[None, :], nx, axis=0)            # column 0 over every x
        elif rows_are_z:
            want = got.reshape(nz, nx).T
        else:
            want = got.reshape(nx, nz)
        np.testing.assert_array_equal(out[f], want)
    # one value short of the whole grid is an error (unless it is a profile)
    if not profile:
        with open(path, "w") as f:
            f.write(f"{nx} {nz}\n1.0 1.0\n0.0 0.0\n{kw}\n" + " ".join(body.split()[:-1]) + "\n")
        rc, _, _ = _read3(fn, path)
        assert rc == L.SM_EIO

