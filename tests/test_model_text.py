"""The a_iso_3d text model reader of the drop-in program (sm_read_model_a,
host/sm_io.c) on the CPU: the values after the header, parsed on host
threads, equal a correctly rounded parse of the same text bit for bit, and
the reference's rules hold (io_utils.c:1029-1094): one column followed by
nothing that reads as a number is a 1-D profile replicated over (x, y); fewer
numbers than needed, or a token that is not a number, is an error."""
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
