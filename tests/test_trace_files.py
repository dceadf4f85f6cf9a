"""Trace files of the drop-in programs on the CPU: sm_write_trace_set (host
threads, one file per receiver) writes the same bytes as the single-file
writer of the reference's format (io_utils.c:1744-1768) called receiver by
receiver, with each trace's times taken by the sampling test."""
import ctypes as C
import os

import numpy as np
import pytest

from seismod_b200 import _lib as L


def _fns():
    lib = L.load()
    ws = lib.sm_write_trace_set
    ws.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_double),
                   C.POINTER(C.c_double), C.c_double, C.c_size_t, C.POINTER(C.c_double),
                   C.c_size_t, C.POINTER(C.c_size_t)]
    ws.restype = C.c_int
    wf = lib.sm_write_trace_file
    wf.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_double),
                   C.c_size_t]
    wf.restype = C.c_int
    pred = lib.sm_sample_predicate
    pred.argtypes = [C.c_size_t, C.c_double, C.c_double, C.c_double]
    pred.restype = C.c_int
    return lib, ws, wf, pred


def _sz(a):
    return a.ctypes.data_as(C.POINTER(C.c_size_t))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@pytest.mark.timeout(120)
def test_threaded_trace_files_equal_the_single_file_writer(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    lib, ws, wf, pred = _fns()
    rng = np.random.default_rng(21)
    nrec, nsteps, dt = 300, 400, 1e-4
    recno = np.ascontiguousarray(rng.permutation(nrec).astype(np.uintp))
    t0 = np.ascontiguousarray(rng.choice([0.0, 5e-4, 2.5e-3], nrec))
    rdt = np.ascontiguousarray(rng.choice([dt, 2 * dt, 3 * dt], nrec))
    times = []
    for r in range(nrec):
        times.append([dt * (it + 1) for it in range(nsteps) if pred(it, dt, t0[r], rdt[r])])
    counts = np.ascontiguousarray([len(t) for t in times], dtype=np.uintp)
    ld = int(counts.max())
    vals = np.ascontiguousarray(rng.standard_normal((nrec, ld)) * 10.0 ** rng.integers(-9, 3, (nrec, 1)))
    assert ws(b"thr", nrec, _sz(recno), _dp(t0), _dp(rdt), dt, nsteps, _dp(vals), ld, _sz(counts)) == 0
    for r in range(nrec):
        t = np.ascontiguousarray(times[r], dtype=np.float64)
        v = np.ascontiguousarray(vals[r, :counts[r]])
        assert wf(b"seq", int(recno[r]) + 1, _dp(t), _dp(v), int(counts[r])) == 0
    for r in range(nrec):
        n = int(recno[r]) + 1
        a = open(os.path.join("trc", "thr", f"thr_{n}.trc"), "rb").read()
        b = open(os.path.join("trc", "seq", f"seq_{n}.trc"), "rb").read()
        assert a == b, n
        assert a.count(b"\n") == counts[r]
    assert len(os.listdir(os.path.join("trc", "thr"))) == nrec


def test_trace_set_reports_an_unwritable_directory(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    lib, ws, _, _ = _fns()
    os.makedirs("trc")
    open(os.path.join("trc", "blocked"), "w").close()   # a file where the directory goes
    one = np.ones(1, dtype=np.uintp)
    zero = np.zeros(1)
    vals = np.ones(1)
    rc = ws(b"blocked", 1, _sz(np.zeros(1, dtype=np.uintp)), _dp(zero), _dp(np.full(1, 1e-4)),
            1e-4, 1, _dp(vals), 1, _sz(one))
    assert rc == L.SM_EIO
    assert b"not a directory" in lib.sm_last_error()
