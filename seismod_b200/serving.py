"""Python side of the request loop (sm_server_*, include/seismod_gpu.h).

A Server takes e_iso and a_iso_3d problems (seismod_b200.workloads), copies
their inputs into the library's request structs and hands them to the C++
worker; wait(), traces() and stats() read back.  The structs below mirror
sm_eiso_request, sm_a3d_request and sm_server_stats field for field; their
sizes are checked against sm_server_struct_sizes().
"""
import ctypes as C

import numpy as np

from . import _lib as L
from . import api

_sz = C.c_size_t
_d = C.c_double
_dp = C.POINTER(C.c_double)
_szp = C.POINTER(C.c_size_t)
_ip = C.POINTER(C.c_int)


class EisoRequest(C.Structure):
    _fields_ = [("nx", _sz), ("nz", _sz), ("npml", _sz), ("h", _d), ("dt", _d),
                ("la", _dp), ("mu", _dp), ("l2m", _dp), ("b", _dp), ("bm", _dp),
                ("d", _dp), ("dh", _dp), ("dH", _dp), ("precision", C.c_int),
                ("nsrc", _sz), ("src_index", _szp), ("src_type", _ip), ("src_fct", _dp),
                ("src_length", _szp), ("src_stride", _sz), ("src_scale", _d),
                ("nrec", _sz), ("rec_index", _szp), ("rec_comp", _ip), ("rec_t0", _dp),
                ("rec_dt", _dp), ("nsteps", _sz)]


class A3dRequest(C.Structure):
    _fields_ = [("nx2", _sz), ("ny2", _sz), ("nz2", _sz), ("np", _sz),
                ("dx", _d), ("dy", _d), ("dz", _d), ("dt", _d),
                ("vp", _dp), ("rho", _dp), ("coef", C.POINTER(_dp)), ("precision", C.c_int),
                ("nsrc", _sz), ("src_index", _szp), ("src_fct", _dp), ("src_length", _szp),
                ("src_stride", _sz), ("src_scale", _d),
                ("nrec", _sz), ("rec_index", _szp), ("rec_comp", _ip), ("rec_t0", _dp),
                ("rec_dt", _dp), ("nsteps", _sz)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", _sz), ("completed", _sz), ("failed", _sz), ("running", _sz),
                ("queued", _sz), ("latency_p50", _d), ("latency_p99", _d),
                ("latency_mean", _d), ("latency_max", _d), ("wait_p50", _d), ("wait_p99", _d),
                ("busy_s", _d), ("shots_per_s", _d), ("gcell_per_s", _d),
                ("hbm_budget", _sz), ("hbm_peak", _sz), ("max_running", _sz)]


_SIGS = {
    "sm_server_create": (C.c_int, [C.c_int, _sz, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.c_void_p)]),
    "sm_server_submit_eiso": (C.c_int, [C.c_void_p, C.POINTER(EisoRequest),
                                        C.POINTER(C.c_uint64)]),
    "sm_server_submit_a3d": (C.c_int, [C.c_void_p, C.POINTER(A3dRequest),
                                       C.POINTER(C.c_uint64)]),
    "sm_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, _d]),
    "sm_server_drain": (C.c_int, [C.c_void_p, _d]),
    "sm_server_status": (C.c_int, [C.c_void_p, C.c_uint64, _ip, _dp]),
    "sm_server_traces": (C.c_int, [C.c_void_p, C.c_uint64, _sz, _sz, _dp, _sz, _szp]),
    "sm_server_release": (C.c_int, [C.c_void_p, C.c_uint64]),
    "sm_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "sm_server_destroy": (C.c_int, [C.c_void_p]),
    "sm_server_set_group": (C.c_int, [C.c_void_p, C.c_int]),
    "sm_server_struct_sizes": (C.c_int, [_szp, _szp, _szp]),
    "sm_eiso_device_bytes": (C.c_int, [_sz, _sz, _sz, C.c_int, _sz, _sz, _sz, _szp]),
    "sm_a3d_device_bytes": (C.c_int, [_sz, _sz, _sz, _sz, C.c_int, _sz, _sz, _szp]),
}


def lib():
    lb = L.load()
    if not getattr(lb, "_server_sigs", False):
        for name, (res, args) in _SIGS.items():
            f = getattr(lb, name)
            f.restype, f.argtypes = res, args
        lb._server_sigs = True
    return lb


def struct_sizes():
    e, a, s = _sz(), _sz(), _sz()
    L.check(lib().sm_server_struct_sizes(C.byref(e), C.byref(a), C.byref(s)))
    return e.value, a.value, s.value


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u(a):
    return np.ascontiguousarray(a, dtype=np.uintp)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def eiso_request(p, precision="fp32", shot=0):
    """(EisoRequest, keep-alive list) for shot `shot` of e_iso problem p."""
    q = api.eiso_inputs(p, [shot])
    idx, typ, fct, ln = q["src"][0]
    keep = [_f64(q[k]) for k in ("la", "mu", "l2m", "b", "bm", "d", "dh", "dH")]
    fct = _f64(fct)
    fct = fct.reshape(len(idx), -1)
    sidx, styp, sln = _u(idx), _i32(typ), _u(ln)
    ridx, comps, t0, rdt = q["rec"]
    ridx, comps, t0, rdt = _u(ridx), _i32(comps), _f64(t0), _f64(rdt)
    keep += [fct, sidx, styp, sln, ridx, comps, t0, rdt]
    r = EisoRequest(q["nx"], q["nz"], q["npml"], q["h"], q["dt"],
                    *[L.dptr(a) for a in keep[:8]], L.PRECISIONS[precision],
                    len(sidx), L.szptr(sidx), L.iptr(styp), L.dptr(fct), L.szptr(sln),
                    fct.shape[1], q["src_scale"],
                    len(ridx), L.szptr(ridx), L.iptr(comps), L.dptr(t0), L.dptr(rdt),
                    q["nsteps"])
    return r, keep


def a3d_request(p, precision="fp32"):
    """(A3dRequest, keep-alive list) for a_iso_3d problem p."""
    q = api.a3d_inputs(p)
    vp, rho = _f64(q["vp"]), _f64(q["rho"])
    cf = [_f64(c) for c in q["coef"]]
    P = (_dp * 18)(*[L.dptr(c) for c in cf])
    idx, fct, ln = q["src"]
    fct = _f64(fct).reshape(len(idx), -1)
    sidx, sln = _u(idx), _u(ln)
    ridx, comps, t0, rdt = q["rec"]
    ridx, comps, t0, rdt = _u(ridx), _i32(comps), _f64(t0), _f64(rdt)
    keep = [vp, rho, cf, P, fct, sidx, sln, ridx, comps, t0, rdt]
    n = vp.shape
    d = q["d"]
    r = A3dRequest(n[0], n[1], n[2], q["npml"], d[0], d[1], d[2], q["dt"],
                   L.dptr(vp), L.dptr(rho), C.cast(P, C.POINTER(_dp)), L.PRECISIONS[precision],
                   len(sidx), L.szptr(sidx), L.dptr(fct), L.szptr(sln), fct.shape[1],
                   q["src_scale"],
                   len(ridx), L.szptr(ridx), L.iptr(comps), L.dptr(t0), L.dptr(rdt),
                   q["nsteps"])
    return r, keep


class Server:
    """A request loop on one GPU (sm_server_*)."""

    def __init__(self, device=0, hbm_budget=0, max_active=0, slice_steps=0, graph_steps=0,
                 group=False):
        h = C.c_void_p()
        L.check(lib().sm_server_create(device, hbm_budget, max_active, slice_steps, graph_steps,
                                       C.byref(h)))
        self._h = h
        self._nrec = {}
        if group:
            L.check(lib().sm_server_set_group(h, 1))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().sm_server_destroy(self._h)
            self._h = None

    __del__ = close

    def submit(self, kind, problem, precision="fp32", shot=0):
        """Queue one shot; returns its ticket."""
        t = C.c_uint64()
        if kind == "eiso":
            r, keep = eiso_request(problem, precision, shot)
            L.check(lib().sm_server_submit_eiso(self._h, C.byref(r), C.byref(t)))
        elif kind == "a3d":
            r, keep = a3d_request(problem, precision)
            L.check(lib().sm_server_submit_a3d(self._h, C.byref(r), C.byref(t)))
        else:
            raise ValueError(kind)
        del keep   # the library copied the arrays
        self._nrec[t.value] = r.nrec
        return t.value

    def wait(self, ticket, timeout=-1.0):
        L.check(lib().sm_server_wait(self._h, ticket, float(timeout)))

    def drain(self, timeout=-1.0):
        L.check(lib().sm_server_drain(self._h, float(timeout)))

    def status(self, ticket):
        st, lat = C.c_int(), C.c_double()
        L.check(lib().sm_server_status(self._h, ticket, C.byref(st), C.byref(lat)))
        return st.value, lat.value

    def traces(self, ticket):
        n = self._nrec[ticket]
        counts = np.zeros(n, dtype=np.uintp)
        L.check(lib().sm_server_traces(self._h, ticket, 0, n, None, 0, L.szptr(counts)))
        ld = max(int(counts.max()) if n else 1, 1)
        out = np.zeros((n, ld))
        L.check(lib().sm_server_traces(self._h, ticket, 0, n, L.dptr(out), ld, None))
        return [out[k, :counts[k]].copy() for k in range(n)]

    def release(self, ticket):
        L.check(lib().sm_server_release(self._h, ticket))
        self._nrec.pop(ticket, None)

    def stats(self):
        st = ServerStats()
        L.check(lib().sm_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}


def device_bytes(kind, problem, precision="fp32"):
    """Device memory one shot of `problem` takes (the admission estimate)."""
    b = _sz()
    if kind == "eiso":
        p = problem
        L.check(lib().sm_eiso_device_bytes(p.nx, p.nz, p.npml, L.PRECISIONS[precision], 1,
                                           len(p.receivers), api.nsteps(p.duration, p.dt),
                                           C.byref(b)))
    else:
        p = problem
        n = [s + 2 * p.npml for s in p.shape]
        L.check(lib().sm_a3d_device_bytes(n[0], n[1], n[2], p.npml, L.PRECISIONS[precision],
                                          len(p.receivers), api.nsteps(p.duration, p.dt),
                                          C.byref(b)))
    return b.value
