"""Text snapshots of the drop-in programs on the CPU: sm_write_snapshot and
sm_write_snapshot_cyl (columns formatted on host threads) write the bytes of
write_snapshot (io_utils.c:1775-1820): "x  z  1e3*v" per node in "%le", the
interior, or with plstr the padded grid, x slow."""
import ctypes as C
import os

import numpy as np
import pytest

from seismod_b200 import _lib as L


def _fn(name):
    f = getattr(L.load(), name)
    f.argtypes = [C.c_char_p, C.c_size_t, C.c_double, C.POINTER(C.c_double), C.c_size_t,
                  C.c_size_t, C.c_size_t, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
    f.restype = C.c_int
    return f


def _expected(data, npl, npr, np_, dx, dz, x0, z0, strips):
    nx2, nz2 = data.shape
    out = []
    if strips:
        for i in range(nx2):
            x = x0 + (float(i) - float(npl)) * dx
            for k in range(nz2):
                out.append("%e  %e  %e\n" % (x, z0 + (float(k) - float(np_)) * dz, 1e3 * data[i, k]))
    else:
        for i in range(nx2 - npl - npr):
            x = x0 + i * dx
            for k in range(nz2 - 2 * np_):
                out.append("%e  %e  %e\n" % (x, z0 + k * dz, 1e3 * data[i + npl, k + np_]))
    return "".join(out).encode()


@pytest.mark.timeout(120)
@pytest.mark.parametrize("fn,cyl", [("sm_write_snapshot", False), ("sm_write_snapshot_cyl", True)])
@pytest.mark.parametrize("strips", [0, 1])
def test_snapshot_bytes(tmp_path, monkeypatch, fn, cyl, strips):
    monkeypatch.chdir(tmp_path)
    rng = np.random.default_rng(31)
    nx2, nz2, np_ = 403, 257, 9           # 103,571 nodes with the frame: several threads
    data = np.ascontiguousarray(rng.standard_normal((nx2, nz2)) * 10.0 ** rng.integers(-12, 2, (nx2, nz2)))
    dx, dz, x0, z0, t = 2.5, 1.25, -10.0, 3.0, 0.0123
    f = _fn(fn)
    assert f(b"snap", 3, t, data.ctypes.data_as(C.POINTER(C.c_double)), nx2, nz2, np_,
             dx, dz, x0, z0, strips) == 0
    path = os.path.join("ssh", "snap", "snap_3_%f.ssh" % t)
    got = open(path, "rb").read()
    npl = 0 if cyl else np_
    assert got == _expected(data, npl, np_, np_, dx, dz, x0, z0, strips)
