"""Python front end of the C ABI: device handles for e_iso, a_iso_3d and
e_cyl_iso and
helpers that take a whole shot from a workload description to traces.

Everything here calls libseismod_gpu.so; the arithmetic of the set-up
(materials, PML/CPML profiles, Ricker wavelets, sampling predicate) is the
library's C host code, identical to the reference's, and the time loop runs
on the GPU.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L


def c_round(v):
    """C round() / lround(): half away from zero (io_utils.c:1488, 1650)."""
    return int(math.copysign(math.floor(abs(v) + 0.5), v))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ----------------------------------------------------------------------------
# host set-up helpers (C, FP64)
# ----------------------------------------------------------------------------

def ricker(A, f, dt, fac=1.0):
    """src.c:43-65 -> (fct [n, stride], lengths)."""
    lib = L.load()
    A, f = _f64(np.atleast_1d(A)), _f64(np.atleast_1d(f))
    stride = max(int(lib.sm_ricker_length(float(x), dt, fac)) for x in f)
    fct = np.zeros((len(A), stride))
    ln = np.zeros(len(A), dtype=np.uintp)
    L.check(lib.sm_ricker(len(A), L.dptr(A), L.dptr(f), dt, fac, stride, L.dptr(fct),
                          L.szptr(ln)))
    return fct, ln.astype(np.int64)


def nsteps(duration, dt):
    return int(L.load().sm_nsteps(duration, dt))


def sample_predicate(it, dt, t0, rdt):
    return bool(L.load().sm_sample_predicate(it, dt, t0, rdt))


def eiso_materials(vp, vs, rho):
    lib = L.load()
    nx, nz = vp.shape
    vp, vs, rho = _f64(vp), _f64(vs), _f64(rho)
    out = [np.zeros((nx, nz)) for _ in range(5)]
    vmax = C.c_double()
    L.check(lib.sm_eiso_materials(nx, nz, L.dptr(vp), L.dptr(vs), L.dptr(rho),
                                  *[L.dptr(a) for a in out], C.byref(vmax)))
    return (*out, vmax.value)


def eiso_profiles(npml, h, vp):
    vp = _f64(vp)
    d, dh, dH = np.zeros(npml), np.zeros(npml), np.zeros(npml + 1)
    L.check(L.load().sm_eiso_profiles(npml, h, vp.size, L.dptr(vp), L.dptr(d), L.dptr(dh),
                                      L.dptr(dH)))
    return d, dh, dH


def a3d_pad_model(vp, rho, npml):
    nx, ny, nz = vp.shape
    vp, rho = _f64(vp), _f64(rho)
    shp = (nx + 2 * npml, ny + 2 * npml, nz + 2 * npml)
    vpp, rhop = np.empty(shp), np.empty(shp)   # every cell is written
    L.check(L.load().sm_a3d_pad_model(nx, ny, nz, npml, L.dptr(vp), L.dptr(rho), L.dptr(vpp),
                                      L.dptr(rhop)))
    return vpp, rhop


def a3d_cfl_vpmax(nx, nz, vp_pad):
    return L.load().sm_a3d_cfl_vpmax(nx, nz, L.dptr(_f64(vp_pad)))


def a3d_cfl_vpmax_unpadded(vp, npml):
    """a3d_cfl_vpmax of the padded model, read from the unpadded one."""
    nx, ny, nz = vp.shape
    return L.load().sm_a3d_cfl_vpmax_unpadded(nx, ny, nz, npml, L.dptr(_f64(vp)))


def a3d_cpml(npml, shape2, d, dt, pml_order=2.0, vmax=5000.0, Rc=1e-5, kappa_max=1.0,
             alpha_max_flag=1, f0=0.0):
    n2 = list(shape2)
    arrs = [np.zeros(n2[c // 3]) for c in range(9)] + \
           [np.zeros(n2[(c - 9) // 3] - 1) for c in range(9, 18)]
    P = (L._dp * 18)(*[L.dptr(a) for a in arrs])
    L.check(L.load().sm_a3d_cpml(npml, n2[0], n2[1], n2[2], d[0], d[1], d[2], dt, pml_order,
                                 vmax, Rc, kappa_max, alpha_max_flag, f0, P))
    return arrs


# ----------------------------------------------------------------------------
# device handles
# ----------------------------------------------------------------------------

class EIsoDevice:
    """An e_iso state on the GPU: nshots shots over one model."""

    def __init__(self, nx, nz, npml, h, dt, la, mu, l2m, b, bm, d, dh, dH,
                 precision="fp32", nshots=1, device=0):
        lib = L.load()
        self.nx, self.nz, self.npml, self.h, self.dt = nx, nz, npml, h, dt
        self.NX, self.NZ = nx + 2 * npml, nz + 2 * npml
        self.nshots = nshots
        self.precision = precision
        arrs = [_f64(a) for a in (la, mu, l2m, b, bm, d, dh, dH)]
        hnd = C.c_void_p()
        L.check(lib.sm_eiso_create(device, nx, nz, npml, h, dt, *[L.dptr(a) for a in arrs],
                                   L.PRECISIONS[precision], nshots, C.byref(hnd)))
        self._h = hnd
        self.nrec = [0] * nshots

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.load().sm_eiso_destroy(self._h)
            self._h = None

    __del__ = close

    def set_sources(self, shot, index, types, fct, lengths, scale):
        index = np.ascontiguousarray(index, dtype=np.uintp)
        types = np.ascontiguousarray(types, dtype=np.int32)
        fct = _f64(fct)
        lengths = np.ascontiguousarray(lengths, dtype=np.uintp)
        shot = L.SM_ALL_SHOTS if shot is None else shot
        L.check(L.load().sm_eiso_set_sources(self._h, shot, len(index), L.szptr(index),
                                             L.iptr(types), L.dptr(fct), L.szptr(lengths),
                                             fct.shape[1] if fct.ndim == 2 else fct.size, scale))

    def set_receivers(self, shot, index, comps, t0, rdt, nsteps_max):
        index = np.ascontiguousarray(index, dtype=np.uintp)
        comps = np.ascontiguousarray(comps, dtype=np.int32)
        t0, rdt = _f64(t0), _f64(rdt)
        L.check(L.load().sm_eiso_set_receivers(
            self._h, L.SM_ALL_SHOTS if shot is None else shot, len(index), L.szptr(index),
            L.iptr(comps), L.dptr(t0), L.dptr(rdt), nsteps_max))
        for s in (range(self.nshots) if shot is None else [shot]):
            self.nrec[s] = len(index)

    def run(self, n):
        L.check(L.load().sm_eiso_run(self._h, n))

    def sync(self):
        L.check(L.load().sm_eiso_sync(self._h))

    def step_count(self):
        n = C.c_size_t()
        L.check(L.load().sm_eiso_step_count(self._h, C.byref(n)))
        return n.value

    def traces(self, shot=0, max_samples=None):
        n = self.nrec[shot]
        counts = np.zeros(n, dtype=np.uintp)
        L.check(L.load().sm_eiso_read_traces(self._h, shot, 0, n, None, 0, L.szptr(counts)))
        ld = int(counts.max()) if n else 0
        out = np.zeros((n, max(ld, 1)))
        if n and ld:
            L.check(L.load().sm_eiso_read_traces(self._h, shot, 0, n, L.dptr(out), ld,
                                                 L.szptr(counts)))
        return [out[r, :int(counts[r])].copy() for r in range(n)]

    def traces_array(self, shot=0):
        """Traces of one shot as one [nrec, nsamples] array, one copy from
        the device (receivers with fewer samples are zero-padded)."""
        n = self.nrec[shot]
        counts = np.zeros(n, dtype=np.uintp)
        L.check(L.load().sm_eiso_read_traces(self._h, shot, 0, n, None, 0, L.szptr(counts)))
        ld = int(counts.max()) if n else 0
        out = np.zeros((n, max(ld, 1)))
        if n and ld:
            L.check(L.load().sm_eiso_read_traces(self._h, shot, 0, n, L.dptr(out), ld,
                                                 L.szptr(counts)))
        return out

    def get_field(self, comp, shot=0, part="total"):
        out = np.zeros((self.NX, self.NZ))
        L.check(L.load().sm_eiso_get_field(self._h, shot, L.SM_COMP[comp], L.SM_PART[part],
                                           L.dptr(out)))
        return out

    def set_field(self, comp, arr, shot=0, part="total"):
        a = _f64(arr).reshape(self.NX, self.NZ)
        L.check(L.load().sm_eiso_set_field(self._h, shot, L.SM_COMP[comp], L.SM_PART[part],
                                           L.dptr(a)))

    def reset(self):
        L.check(L.load().sm_eiso_reset(self._h))

    def stream(self):
        p = C.c_void_p()
        L.check(L.load().sm_eiso_stream(self._h, C.byref(p)))
        return p.value

    def set_timing(self, on=True):
        L.check(L.load().sm_eiso_set_timing(self._h, 1 if on else 0))

    def set_config(self, config):
        L.check(L.load().sm_eiso_set_config(self._h, int(config)))

    def autotune(self, trial_steps=32):
        """Pick the fastest launch configuration (the handle is left reset).
        Returns (config, ms per step)."""
        c, ms = C.c_int(), C.c_double()
        L.check(L.load().sm_eiso_autotune(self._h, int(trial_steps), C.byref(c), C.byref(ms)))
        return c.value, ms.value

    def set_graph(self, steps):
        L.check(L.load().sm_eiso_set_graph(self._h, int(steps)))

    def get_config(self):
        """(current config, number of configs)."""
        c, n = C.c_int(), C.c_int()
        L.check(L.load().sm_eiso_get_config(self._h, C.byref(c), C.byref(n)))
        return c.value, n.value

    def kernel_stats(self, reset=False):
        """(summed update-kernel ms, timed launches, all kernel launches)."""
        ms = C.c_double()
        n = C.c_size_t()
        a = C.c_size_t()
        L.check(L.load().sm_eiso_kernel_stats(self._h, 1 if reset else 0, C.byref(ms),
                                              C.byref(n), C.byref(a)))
        return ms.value, n.value, a.value


class A3DDevice:
    """An a_iso_3d state on the GPU."""

    def __init__(self, vp_pad, rho_pad, npml, d, dt, coef, precision="fp32", device=0,
                 padded=True):
        """vp_pad, rho_pad: the padded model (sm_a3d_create), or with
        padded=False the unpadded one, edge-replicated as it is staged
        (sm_a3d_create_unpadded)."""
        lib = L.load()
        n = vp_pad.shape
        self.shape = n if padded else tuple(x + 2 * npml for x in n)
        self.npml, self.d, self.dt, self.precision = npml, d, dt, precision
        vp_pad, rho_pad = _f64(vp_pad), _f64(rho_pad)
        cf = [_f64(c) for c in coef]
        P = (L._dp * 18)(*[L.dptr(c) for c in cf])
        hnd = C.c_void_p()
        create = lib.sm_a3d_create if padded else lib.sm_a3d_create_unpadded
        L.check(create(device, n[0], n[1], n[2], npml, d[0], d[1], d[2], dt,
                       L.dptr(vp_pad), L.dptr(rho_pad), P, L.PRECISIONS[precision],
                       C.byref(hnd)))
        self._h = hnd
        self.nrec = 0

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.load().sm_a3d_destroy(self._h)
            self._h = None

    __del__ = close

    def set_sources(self, index, fct, lengths, scale):
        index = np.ascontiguousarray(index, dtype=np.uintp)
        fct = _f64(fct)
        lengths = np.ascontiguousarray(lengths, dtype=np.uintp)
        L.check(L.load().sm_a3d_set_sources(self._h, len(index), L.szptr(index), L.dptr(fct),
                                            L.szptr(lengths), fct.shape[1], scale))

    def set_receivers(self, index, comps, t0, rdt, nsteps_max):
        index = np.ascontiguousarray(index, dtype=np.uintp)
        comps = np.ascontiguousarray(comps, dtype=np.int32)
        t0, rdt = _f64(t0), _f64(rdt)
        L.check(L.load().sm_a3d_set_receivers(self._h, len(index), L.szptr(index),
                                              L.iptr(comps), L.dptr(t0), L.dptr(rdt),
                                              nsteps_max))
        self.nrec = len(index)

    def run(self, n):
        L.check(L.load().sm_a3d_run(self._h, n))

    def sync(self):
        L.check(L.load().sm_a3d_sync(self._h))

    def step_count(self):
        n = C.c_size_t()
        L.check(L.load().sm_a3d_step_count(self._h, C.byref(n)))
        return n.value

    def traces(self):
        n = self.nrec
        counts = np.zeros(n, dtype=np.uintp)
        L.check(L.load().sm_a3d_read_traces(self._h, 0, n, None, 0, L.szptr(counts)))
        ld = int(counts.max()) if n else 0
        out = np.zeros((n, max(ld, 1)))
        if n and ld:
            L.check(L.load().sm_a3d_read_traces(self._h, 0, n, L.dptr(out), ld, L.szptr(counts)))
        return [out[r, :int(counts[r])].copy() for r in range(n)]

    def traces_array(self):
        """Traces as one [nrec, nsamples] array (all receivers equally sampled)."""
        n = self.nrec
        counts = np.zeros(n, dtype=np.uintp)
        L.check(L.load().sm_a3d_read_traces(self._h, 0, n, None, 0, L.szptr(counts)))
        ld = int(counts.max()) if n else 0
        out = np.zeros((n, max(ld, 1)))
        if n and ld:
            L.check(L.load().sm_a3d_read_traces(self._h, 0, n, L.dptr(out), ld, L.szptr(counts)))
        return out

    def set_config(self, config):
        L.check(L.load().sm_a3d_set_config(self._h, int(config)))

    def set_chunk(self, chunk):
        L.check(L.load().sm_a3d_set_chunk(self._h, int(chunk)))

    def autotune(self, trial_steps=32):
        """Pick the fastest launch configuration (the handle is left reset);
        with graphs set (set_graph) the trials replay them.  Returns (config,
        chunk, ms per step)."""
        c, k, ms = C.c_int(), C.c_int(), C.c_double()
        L.check(L.load().sm_a3d_autotune(self._h, int(trial_steps), C.byref(c), C.byref(k),
                                         C.byref(ms)))
        return c.value, k.value, ms.value

    def set_graph(self, steps):
        L.check(L.load().sm_a3d_set_graph(self._h, int(steps)))

    def get_config(self):
        c, n = C.c_int(), C.c_int()
        L.check(L.load().sm_a3d_get_config(self._h, C.byref(c), C.byref(n)))
        return c.value, n.value

    def get_field(self, comp):
        out = np.zeros(self.shape)
        L.check(L.load().sm_a3d_get_field(self._h, L.SM_COMP[comp], L.dptr(out)))
        return out

    def set_field(self, comp, arr):
        L.check(L.load().sm_a3d_set_field(self._h, L.SM_COMP[comp], L.dptr(_f64(arr))))

    def reset(self):
        L.check(L.load().sm_a3d_reset(self._h))

    def stream(self):
        p = C.c_void_p()
        L.check(L.load().sm_a3d_stream(self._h, C.byref(p)))
        return p.value

    def set_timing(self, on=True):
        L.check(L.load().sm_a3d_set_timing(self._h, 1 if on else 0))

    def kernel_stats(self, reset=False):
        """(summed update-kernel ms, timed launches, all kernel launches)."""
        ms = C.c_double()
        n = C.c_size_t()
        a = C.c_size_t()
        L.check(L.load().sm_a3d_kernel_stats(self._h, 1 if reset else 0, C.byref(ms),
                                              C.byref(n), C.byref(a)))
        return ms.value, n.value, a.value


# ----------------------------------------------------------------------------
# whole shots from workload descriptions (seismod_b200.workloads)
# ----------------------------------------------------------------------------

def eiso_inputs(p, shots=None):
    """Everything sm_eiso_create and the source / receiver set-up take for
    problem p (host arrays), as e_iso.c:379-557 prepares it: averaged
    materials, PML profiles, Ricker series of each shot, node indices."""
    la, mu, l2m, b, bm, vpmax = eiso_materials(p.vp, p.vs, p.rho)
    dt = p.dt
    if dt > p.h / (math.sqrt(2.0) * vpmax):
        raise L.SeismodError(L.SM_ECFL, "time step too large (e_iso.c:476)")
    d, dh, dH = eiso_profiles(p.npml, p.h, p.vp)
    shots = list(range(len(p.shots))) if shots is None else list(shots)
    src = []
    for s in shots:
        srcs = p.shots[s]
        fct, ln = ricker([q[1] for q in srcs], [q[2] for q in srcs], dt)
        idx = [c_round((q[3] - p.x0) / p.h) * p.nz + c_round((q[4] - p.z0) / p.h) for q in srcs]
        typ = [L.SM_SRC[q[0].lower()] for q in srcs]
        src.append((idx, typ, fct, ln))
    ridx = [c_round((x - p.x0) / p.h) * p.nz + c_round((z - p.z0) / p.h)
            for (_, x, z, _, _) in p.receivers]
    comps = [L.SM_COMP[c.lower()] for (c, _, _, _, _) in p.receivers]
    t0 = [r[3] for r in p.receivers]
    rdt = [r[4] * 1e-3 for r in p.receivers]
    return dict(nx=p.nx, nz=p.nz, npml=p.npml, h=p.h, dt=dt, la=la, mu=mu, l2m=l2m, b=b, bm=bm,
                d=d, dh=dh, dH=dH, src=src, src_scale=dt, rec=(ridx, comps, t0, rdt),
                nsteps=nsteps(p.duration, dt))


def eiso_device(p, precision="fp32", shots=None, device=0):
    """Build an EIsoDevice for problem p with sources of `shots` (default:
    all shots of p) and p's receivers.  Returns (dev, nsteps)."""
    q = eiso_inputs(p, shots)
    dev = EIsoDevice(q["nx"], q["nz"], q["npml"], q["h"], q["dt"], q["la"], q["mu"], q["l2m"],
                     q["b"], q["bm"], q["d"], q["dh"], q["dH"], precision, len(q["src"]), device)
    for k, (idx, typ, fct, ln) in enumerate(q["src"]):
        dev.set_sources(k, idx, typ, fct, ln, q["src_scale"])
    n = q["nsteps"]
    dev.set_receivers(None, *q["rec"], n)
    return dev, n


def run_eiso(p, precision="fp32", shots=None, device=0, nsteps_override=None):
    """Whole shots on the GPU -> list (per shot) of lists of trace arrays
    (raw velocities; the reference's .trc files hold 1e3 * v)."""
    dev, n = eiso_device(p, precision, shots, device)
    dev.run(n if nsteps_override is None else nsteps_override)
    out = [dev.traces(s) for s in range(dev.nshots)]
    dev.close()
    return out


def group_run(devs, n):
    """Advance several EIsoDevice objects (any grid sizes, same precision) by
    n steps together: one launch per step for all of them."""
    arr = (C.c_void_p * len(devs))(*[d._h.value for d in devs])
    L.check(L.load().sm_eiso_group_run(arr, len(devs), n))


def a3d_group_run(devs, n):
    """Advance several A3dDevice objects (any grid sizes, same precision) by
    n steps together: one launch per step for all of them."""
    arr = (C.c_void_p * len(devs))(*[d._h.value for d in devs])
    L.check(L.load().sm_a3d_group_run(arr, len(devs), n))


def a3d_index(p, x, y, z):
    nx2, ny2, nz2 = (n + 2 * p.npml for n in p.shape)
    i = c_round((x - p.origin[0]) / p.d[0]) + p.npml
    j = c_round((y - p.origin[1]) / p.d[1]) + p.npml
    k = c_round((z - p.origin[2]) / p.d[2]) + p.npml
    return (i * ny2 + j) * nz2 + k


def _c_round_many(v):
    """c_round over an array: half away from zero."""
    return (np.sign(v) * np.floor(np.abs(v) + 0.5)).astype(np.int64)


def _a3d_index_many(p, xyz):
    nx2, ny2, nz2 = (n + 2 * p.npml for n in p.shape)
    i = _c_round_many((xyz[:, 0] - p.origin[0]) / p.d[0]) + p.npml
    j = _c_round_many((xyz[:, 1] - p.origin[1]) / p.d[1]) + p.npml
    k = _c_round_many((xyz[:, 2] - p.origin[2]) / p.d[2]) + p.npml
    return ((i * ny2 + j) * nz2 + k).tolist()


def a3d_inputs(p, pad=True):
    """Everything sm_a3d_create and the source / receiver set-up take for
    problem p (host arrays), as a_iso_3d.c:317-590 prepares it.  pad=False
    leaves the model unpadded, for A3DDevice(..., padded=False)."""
    nx, ny, nz = p.shape
    dt = p.dt
    if pad:
        vpp, rhop = a3d_pad_model(p.vp, p.rho, p.npml)
        vpmax = a3d_cfl_vpmax(nx, nz, vpp)
    else:
        vpp, rhop = _f64(p.vp), _f64(p.rho)
        vpmax = a3d_cfl_vpmax_unpadded(vpp, p.npml)
    shape2 = tuple(n + 2 * p.npml for n in p.shape)
    dx, dy, dz = p.d
    if dt * vpmax * math.sqrt(1. / dx ** 2 + 1. / dy ** 2 + 1. / dz ** 2) > 1.:
        raise L.SeismodError(L.SM_ECFL, "time step too large (a_iso_3d.c:411-417)")
    coef = a3d_cpml(p.npml, shape2, p.d, dt, 2.0, 5000.0, p.Rc, p.kappa_max, p.alpha_max,
                    p.sources[0][2])
    fct, ln = ricker([q[1] for q in p.sources], [q[2] for q in p.sources], dt)
    idx = [a3d_index(p, q[3], q[4], q[5]) for q in p.sources]
    # receivers (component, x, y, z, t0, dt) transposed once: a large grid
    # of receivers is tens of thousands of tuples
    cols = list(zip(*p.receivers)) if p.receivers else [()] * 6
    rxyz = np.array(cols[1:4], dtype=np.float64).reshape(3, -1).T
    ridx = _a3d_index_many(p, rxyz)
    code = {c: L.SM_COMP[c.lower()] for c in set(cols[0])}
    comps = [code[c] for c in cols[0]]
    return dict(vp=vpp, rho=rhop, padded=pad, npml=p.npml, d=p.d, dt=dt, coef=coef,
                src=(idx, fct, ln), src_scale=dt * 1e6,
                rec=(ridx, comps, list(cols[4]), (np.array(cols[5], dtype=np.float64) * 1e-3).tolist()),
                nsteps=nsteps(p.duration, dt))


def a3d_device(p, precision="fp32", device=0, pad_on_host=False):
    """A handle for problem p; the model is padded as it is staged unless
    pad_on_host (the padded model through sm_a3d_create, the same bits)."""
    q = a3d_inputs(p, pad=pad_on_host)
    dev = A3DDevice(q["vp"], q["rho"], q["npml"], q["d"], q["dt"], q["coef"], precision, device,
                    padded=pad_on_host)
    n = q["nsteps"]
    dev.set_sources(*q["src"], q["src_scale"])
    dev.set_receivers(*q["rec"], n)
    return dev, n


def run_a3d(p, precision="fp32", device=0, nsteps_override=None):
    dev, n = a3d_device(p, precision, device)
    dev.run(n if nsteps_override is None else nsteps_override)
    out = dev.traces()
    dev.close()
    return out


# ----------------------------------------------------------------------------
# e_cyl_iso
# ----------------------------------------------------------------------------

ECYL_COMP = {"vr": L.SM_VR, "vtheta": L.SM_VT, "vz": L.SM_VZ, "trr": L.SM_TRR,
             "trtheta": L.SM_TRT, "trz": L.SM_TRZ, "tthetatheta": L.SM_TTT,
             "tthetaz": L.SM_TTZ, "tzz": L.SM_TZZ, "div": L.SM_DIV, "curl": L.SM_CURL}
ECYL_FIELD = {"vr": L.SM_VR, "vt": L.SM_VT, "vz": L.SM_VZ, "trr": L.SM_TRR, "ttt": L.SM_TTT,
              "tzz": L.SM_TZZ, "trz": L.SM_TRZ, "trt": L.SM_TRT, "ttz": L.SM_TTZ}
ECYL_SRC = {"fr": 9, "ftheta": 10, "fz": 11, "bulk": 6, "kurkjian": 12}


def ecyl_inputs(p):
    """Everything sm_ecyl_create and the source / receiver set-up take for an
    ECylProblem, as e_cyl_iso.c:277-600 prepares it (library host code)."""
    lib = L.load()
    npml = p.np_used
    nx2, nz2 = p.nx + npml, p.nz + 2 * npml
    pads = [np.zeros((nx2, nz2)) for _ in range(3)]
    vp, vs, rho = _f64(p.vp), _f64(p.vs), _f64(p.rho)
    L.check(lib.sm_ecyl_pad_model(p.nx, p.nz, npml, L.dptr(vp), L.dptr(vs), L.dptr(rho),
                                  *[L.dptr(a) for a in pads]))
    mats = [np.zeros((nx2, nz2)) for _ in range(8)]
    vmax = C.c_double()
    mp = (L._dp * 8)(*[L.dptr(a) for a in mats])
    L.check(lib.sm_ecyl_materials(nx2, nz2, *[L.dptr(a) for a in pads], mp, C.byref(vmax)))
    dt = p.dt
    if dt > 0.5 * (p.dx + p.dz) / (math.sqrt(2.0) * vmax.value):
        raise L.SeismodError(L.SM_ECFL, "time step too large (e_cyl_iso.c:484-488)")
    alpha = math.pi * p.sources[0][2] if p.alpha_max else 0.0
    coef = [np.zeros(npml if k < 9 else npml + 1) for k in range(15)]
    cp = (L._dp * 15)(*[L.dptr(a) for a in coef])
    L.check(lib.sm_ecyl_cpml(npml, p.dx, p.dz, dt, 2.0, 5000.0, p.Rc, p.kappa_max, alpha,
                             int(p.absorb), cp))

    def index(x, z):
        return c_round((x - p.x0) / p.dx) * nz2 + c_round((z - p.z0) / p.dz) + npml

    sidx = [index(q[3], q[4]) for q in p.sources]
    if p.sources[0][0].lower() == "kurkjian":
        q = p.sources[0]
        n = int(lib.sm_ecyl_kurkjian(q[1], q[2], dt, 0.0, q[3], p.dx, p.dz, p.n, 0, None))
        fct = np.zeros((1, max(n, 1)))
        lij = mats[0].reshape(-1)[sidx[0]]
        n = int(lib.sm_ecyl_kurkjian(q[1], q[2], dt, lij, q[3], p.dx, p.dz, p.n, n,
                                     L.dptr(fct)))
        src = ([sidx[0]], [ECYL_SRC["kurkjian"]], fct, [n])
    else:
        fct, ln = ricker([q[1] for q in p.sources], [q[2] for q in p.sources], dt)
        src = (sidx, [ECYL_SRC[q[0].lower()] for q in p.sources], fct, ln)
    rec = ([index(x, z) for (_, x, z, _, _) in p.receivers],
           [ECYL_COMP[c.lower()] for (c, _, _, _, _) in p.receivers],
           [t0 for (_, _, _, t0, _) in p.receivers],
           [r * 1e-3 for (_, _, _, _, r) in p.receivers])
    return dict(npml=npml, mats=mats, coef=coef, dt=dt, src=src, rec=rec,
                nsteps=nsteps(p.duration, dt))


class ECylDevice:
    """An e_cyl_iso state on the GPU."""

    def __init__(self, nx, nz, npml, n, dx, dz, dt, mats, coef, precision="fp32", device=0):
        lib = L.load()
        self.shape = (nx + npml, nz + 2 * npml)
        self._keep = [_f64(a) for a in mats] + [_f64(c) for c in coef]
        mp = (L._dp * 8)(*[L.dptr(a) for a in self._keep[:8]])
        cp = (L._dp * 15)(*[L.dptr(a) for a in self._keep[8:]])
        hnd = C.c_void_p()
        L.check(lib.sm_ecyl_create(device, nx, nz, npml, int(n), dx, dz, dt, mp, cp,
                                   L.PRECISIONS[precision], C.byref(hnd)))
        self._h = hnd
        self.nrec = 0

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.load().sm_ecyl_destroy(self._h)
            self._h = None

    __del__ = close

    def set_sources(self, index, types, fct, lengths):
        index = np.ascontiguousarray(index, dtype=np.uintp)
        types = np.ascontiguousarray(types, dtype=np.int32)
        fct = _f64(np.atleast_2d(fct))
        lengths = np.ascontiguousarray(lengths, dtype=np.uintp)
        L.check(L.load().sm_ecyl_set_sources(self._h, len(index), L.szptr(index),
                                             types.ctypes.data_as(L._ip), L.dptr(fct),
                                             L.szptr(lengths), fct.shape[1]))

    def set_receivers(self, index, comp, t0, rdt, nsteps_max):
        index = np.ascontiguousarray(index, dtype=np.uintp)
        comp = np.ascontiguousarray(comp, dtype=np.int32)
        t0, rdt = _f64(t0), _f64(rdt)
        L.check(L.load().sm_ecyl_set_receivers(self._h, len(index), L.szptr(index),
                                               comp.ctypes.data_as(L._ip), L.dptr(t0),
                                               L.dptr(rdt), nsteps_max))
        self.nrec = len(index)

    def run(self, n):
        L.check(L.load().sm_ecyl_run(self._h, n))

    def sync(self):
        L.check(L.load().sm_ecyl_sync(self._h))

    def reset(self):
        L.check(L.load().sm_ecyl_reset(self._h))

    def stream(self):
        s = C.c_void_p()
        L.check(L.load().sm_ecyl_stream(self._h, C.byref(s)))
        return s.value

    def traces(self):
        n = self.nrec
        counts = np.zeros(n, dtype=np.uintp)
        L.check(L.load().sm_ecyl_read_traces(self._h, 0, n, None, 0, L.szptr(counts)))
        ld = int(counts.max()) if n else 0
        out = np.zeros((n, max(ld, 1)))
        if n and ld:
            L.check(L.load().sm_ecyl_read_traces(self._h, 0, n, L.dptr(out), ld,
                                                 L.szptr(counts)))
        return [out[k, :counts[k]].copy() for k in range(n)]

    def set_timing(self, on=True):
        L.check(L.load().sm_ecyl_set_timing(self._h, 1 if on else 0))

    def kernel_stats(self, reset=False):
        """(summed velocity + source + stress ms, timed steps, all kernel launches)."""
        ms = C.c_double()
        n = C.c_size_t()
        a = C.c_size_t()
        L.check(L.load().sm_ecyl_kernel_stats(self._h, 1 if reset else 0, C.byref(ms),
                                              C.byref(n), C.byref(a)))
        return ms.value, n.value, a.value

    def get_field(self, name):
        out = np.zeros(self.shape)
        L.check(L.load().sm_ecyl_get_field(self._h, ECYL_FIELD[name], L.dptr(out)))
        return out

    def set_field(self, name, arr):
        a = _f64(arr)
        L.check(L.load().sm_ecyl_set_field(self._h, ECYL_FIELD[name], L.dptr(a)))


def ecyl_device(p, precision="fp32", device=0):
    q = ecyl_inputs(p)
    dev = ECylDevice(p.nx, p.nz, q["npml"], p.n, p.dx, p.dz, q["dt"], q["mats"], q["coef"],
                     precision, device)
    dev.set_sources(*q["src"])
    dev.set_receivers(*q["rec"], q["nsteps"])
    return dev, q["nsteps"]


def run_ecyl(p, precision="fp32", device=0, nsteps_override=None):
    """A whole e_cyl_iso shot -> list of trace arrays (raw values; the
    reference's .trc files hold 1e3 * value)."""
    dev, n = ecyl_device(p, precision, device)
    dev.run(n if nsteps_override is None else nsteps_override)
    out = dev.traces()
    dev.close()
    return out
