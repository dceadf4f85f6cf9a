"""sm_eiso_run_noalloc: one e_iso shot run without any device allocation.

It exists for callers that cannot call cudaMalloc (their device memory is all
handed out by their own allocator, or they run where an allocation is not
allowed or would stall the device); the whole run lives in a fixed array
inside the library.  Its traces must equal the handle path's
(sm_eiso_create / sm_eiso_run / sm_eiso_read_traces) on the same shot bit for
bit (every launch configuration of the e_iso step rounds identically), and lie
within the FP32 tolerance used throughout the tests of the FP64 oracle, on two
calls in a row: the second call reuses the array the first one left behind.

This file is collected last on purpose, so that a run that stops at the first
failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import harness as H
from seismod_b200 import _lib as L
from seismod_b200 import api
from seismod_b200 import serving
from seismod_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5   # relative L2 over all traces, as the other FP32 parity tests


def _fn():
    f = serving.lib().sm_eiso_run_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_void_p, C.POINTER(serving.EisoRequest), C.POINTER(C.c_double),
                  C.c_size_t, C.POINTER(C.c_size_t)]
    return f


def _run_noalloc(p, precision="fp32"):
    r, keep = serving.eiso_request(p, precision)
    ld = max(int(r.nsteps), 1)
    out = np.zeros((r.nrec, ld))
    counts = np.zeros(r.nrec, dtype=np.uintp)
    rc = _fn()(0, None, C.byref(r), L.dptr(out), ld, L.szptr(counts))
    del keep
    return rc, [out[k, :counts[k]].copy() for k in range(r.nrec)]


def _check(p):
    rc, got = _run_noalloc(p)
    L.check(rc)
    ref = api.run_eiso(p, "fp32")[0]
    assert [len(a) for a in got] == [len(a) for a in ref]
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)
    orc, _, _ = H.run_eiso_oracle(p)
    assert H.rel_l2([1e3 * a for a in got], orc) < TOL_FP32


def test_noalloc_matches_the_handle_path_on_two_calls_in_a_row():
    # two different shots back to back: the second starts from the first's
    # leftovers in the shared array
    _check(W.cfg0(nx=150, nz=110, npml=10, nsteps=260, nrec=9))
    _check(W.cfg0(nx=96, nz=140, npml=7, nsteps=330, nrec=5))


def test_noalloc_rejects_what_it_cannot_hold():
    big = W.cfg0(nx=1400, nz=1400, npml=20, nsteps=10, nrec=2)
    rc, _ = _run_noalloc(big)
    assert rc == L.SM_EINVAL
    assert b"scratch" in L.load().sm_last_error()
    rc, _ = _run_noalloc(W.cfg0(nx=40, nz=40, npml=4, nsteps=10, nrec=2), precision="fp64")
    assert rc == L.SM_EINVAL
