"""Test harness: run a whole shot through the FP64 oracle the way the
reference drivers do (e_iso.c:342-670, a_iso_3d/a_iso_3d.c:224-741), and
small shared helpers.  Test infrastructure only."""
from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

SRC_TYPES = {"sx": 0, "sz": 2, "sxz": 4, "bulk": 6}
COMPS = {"vx": 0, "vy": 1, "vz": 2, "p": 8}


def c_round(v):
    """C round()/lround(): half away from zero."""
    return int(math.copysign(math.floor(abs(v) + 0.5), v))


def sample_schedule(nsteps, dt, t0, rdt):
    return [it for it in range(nsteps) if O.sample(it, dt, t0, rdt)]


def eiso_setup(p):
    """Host set-up of e_iso.c:361-536 for an EIsoProblem -> dict."""
    la, mu, l2m, b, bm, vpmax = O.eiso_materials(p.vp, p.vs, p.rho)
    dt = p.dt
    if dt > p.h / (math.sqrt(2.0) * vpmax):
        raise ValueError("CFL")
    d, dh, dH = O.eiso_profiles(p.npml, p.h, p.vp)
    return dict(la=la, mu=mu, l2m=l2m, b=b, bm=bm, d=d, dh=dh, dH=dH, dt=dt,
                nsteps=O.nsteps(p.duration, dt))


def eiso_sources(p, shot=0):
    srcs = p.shots[shot]
    A = [s[1] for s in srcs]
    f = [s[2] for s in srcs]
    fct = O.src_fct(A, f, p.dt, 1.0)
    out = []
    for s, w in zip(srcs, fct):
        i = c_round((s[3] - p.x0) / p.h)
        j = c_round((s[4] - p.z0) / p.h)
        out.append((i * p.nz + j, SRC_TYPES[s[0].lower()], w))
    return out


def eiso_receivers(p):
    out = []
    for (comp, x, z, t0, rdt_ms) in p.receivers:
        i = c_round((x - p.x0) / p.h)
        j = c_round((z - p.z0) / p.h)
        out.append((i * p.nz + j, comp.lower(), t0, rdt_ms * 1e-3))
    return out


# the source patches of e_iso block storage: EISO_PR rows (whole blocks of
# 4, two blocks on each side of the source's) by EISO_PC columns centred on
# each source, in source order, a patch only where it keeps clear of the
# shot's earlier ones (by 18 rows when their columns meet)
EISO_PR, EISO_PC = 20, 9


def eiso_source_patches(p, srcs):
    out = []
    for (idx, _, _) in srcs:
        X, Z = idx // p.nz + p.npml, idx % p.nz + p.npml
        px, pz = 4 * (X // 4 - 2), Z - 4
        clear = all(not (pz < qz + EISO_PC and qz < pz + EISO_PC and
                         px - 18 < qx + EISO_PR and qx - 18 < px + EISO_PR)
                    for (qx, qz) in out)
        if clear:
            out.append((px, pz))
    return out


def run_eiso_oracle(p, shot=0, nsteps=None, fields_at=None, bfp_block=0, bfp_axis="x"):
    """FP64 oracle run.  Returns (traces list of np arrays, times list,
    optional dict of padded fields after the last step).  bfp_block > 0
    rounds the stored state to 16-bit block floating point (checker mode)."""
    s = eiso_setup(p)
    n = s["nsteps"] if nsteps is None else nsteps
    o = O.EIso(p.nx, p.nz, p.npml, p.h, s["dt"], s["la"], s["mu"], s["l2m"], s["b"],
               s["bm"], s["d"], s["dh"], s["dH"])
    if bfp_block:
        o.set_bfp(bfp_block, bfp_axis)
    srcs = eiso_sources(p, shot)
    if bfp_block:
        for (px, pz) in eiso_source_patches(p, srcs):
            o.add_patch(px, pz, EISO_PR, EISO_PC)
    recs = eiso_receivers(p)
    tr = [[] for _ in recs]
    tt = [[] for _ in recs]
    dt = s["dt"]
    for it in range(n):
        o.velocity()
        o.stress()
        for (idx, typ, w) in srcs:
            if it < len(w):
                o.add_source(idx, typ, dt * w[it])
        t = dt * (it + 1)
        for r, (idx, comp, t0, rdt) in enumerate(recs):
            if O.sample(it, dt, t0, rdt):
                tr[r].append(1e3 * o.probe(comp, idx))
                tt[r].append(t)
    fields = None
    if fields_at:
        fields = {f: o.get(f) for f in fields_at}
    return [np.array(a) for a in tr], [np.array(a) for a in tt], fields


def a3d_setup(p):
    nx, ny, nz = p.shape
    vpp, rhop = O.a3d_pad_model(p.vp, p.rho, p.npml)
    dt = p.dt
    vpmax = O.a3d_cfl_vpmax(nx, nz, vpp)
    dx, dy, dz = p.d
    if dt * vpmax * math.sqrt(1. / (dx * dx) + 1. / (dy * dy) + 1. / (dz * dz)) > 1.:
        raise ValueError("CFL")
    f0 = p.sources[0][2]
    coef = O.a3d_cpml(p.npml, vpp.shape, dx, dy, dz, dt, 2.0, 5000.0, p.Rc, p.kappa_max,
                      p.alpha_max, f0)
    return dict(vpp=vpp, rhop=rhop, coef=coef, dt=dt, nsteps=O.nsteps(p.duration, dt))


def a3d_index(p, x, y, z):
    nx2, ny2, nz2 = (n + 2 * p.npml for n in p.shape)
    i = c_round((x - p.origin[0]) / p.d[0]) + p.npml
    j = c_round((y - p.origin[1]) / p.d[1]) + p.npml
    k = c_round((z - p.origin[2]) / p.d[2]) + p.npml
    return (i * ny2 + j) * nz2 + k


def run_a3d_oracle(p, nsteps=None, fields_at=None, bfp_block=0, bfp_axis="y"):
    """FP64 oracle run of an a_iso_3d shot; bfp_block > 0 rounds every stored
    value to 16-bit block floating point with blocks of that many cells along
    bfp_axis ("y" or "z"; the storage-rounding checker mode)."""
    s = a3d_setup(p)
    n = s["nsteps"] if nsteps is None else nsteps
    o = O.A3D(s["vpp"], s["rhop"], *p.d, s["dt"], s["coef"])
    if bfp_block:
        o.set_bfp(bfp_block, bfp_axis)
    A = [q[1] for q in p.sources]
    f = [q[2] for q in p.sources]
    fct = O.src_fct(A, f, p.dt, 1.0)
    srcs = [(a3d_index(p, q[3], q[4], q[5]), w) for q, w in zip(p.sources, fct)]
    recs = [(a3d_index(p, x, y, z), c.lower(), t0, r * 1e-3)
            for (c, x, y, z, t0, r) in p.receivers]
    tr = [[] for _ in recs]
    tt = [[] for _ in recs]
    dt = s["dt"]
    # receivers sharing (t0, rdt) are sampled on the same steps: one gather
    # per group and step
    groups = {}
    for r, (idx, comp, t0, rdt) in enumerate(recs):
        groups.setdefault((t0, rdt), []).append(r)
    gsel = {key: (np.array(rs), np.array([O.FIELDS_A[recs[r][1]] for r in rs]),
                  np.array([recs[r][0] for r in rs])) for key, rs in groups.items()}
    for it in range(n):
        o.velocity()
        o.pressure()
        for (idx, w) in srcs:
            if it < len(w):
                o.add_source(idx, dt * w[it] * 1.e6)
        t = dt * (it + 1)
        for (t0, rdt), (rs, fl, qs) in gsel.items():
            if O.sample(it, dt, t0, rdt):
                vals = o.gather(fl, qs)
                for r, v in zip(rs, vals):
                    tr[r].append(1e3 * v)
                    tt[r].append(t)
    fields = None
    if fields_at:
        fields = {f: o.get(f) for f in fields_at}
    return [np.array(a) for a in tr], [np.array(a) for a in tt], fields


def rel_l2(a, b):
    return O.rel_l2(np.concatenate([np.ravel(x) for x in a]),
                    np.concatenate([np.ravel(x) for x in b]))


# ----------------------------------------------------------------------------
# e_cyl_iso (e_cyl_iso.c:277-790)
# ----------------------------------------------------------------------------

ECYL_COMPS = {"vr": "vr", "vtheta": "vt", "vz": "vz", "trr": "trr", "trtheta": "trt",
              "trz": "trz", "tthetatheta": "ttt", "tthetaz": "ttz", "tzz": "tzz",
              "div": "div", "curl": "curl"}


def ecyl_pad(p, a):
    """read_model_e_cyl's padding (io_utils.c:993-1026): z rows copied into
    the top and bottom PML, the last radial column into the outer PML."""
    n = p.np_used
    out = np.zeros((p.nx + n, p.nz + 2 * n))
    out[:p.nx, n:n + p.nz] = a
    out[:p.nx, :n] = a[:, :1]
    out[:p.nx, n + p.nz:] = a[:, -1:]
    out[p.nx:, :] = out[p.nx - 1:p.nx, :]
    return out


def ecyl_setup(p):
    vp, vs, rho = (ecyl_pad(p, a) for a in (p.vp, p.vs, p.rho))
    mats, vpmax = O.ecyl_materials(vp, vs, rho)
    dt = p.dt
    if dt > 0.5 * (p.dx + p.dz) / (math.sqrt(2.0) * vpmax):
        raise ValueError("CFL")
    f0 = p.sources[0][2]
    alpha = math.pi * f0 if p.alpha_max else 0.0
    coef = O.ecyl_cpml(p.np_used, p.dx, p.dz, dt, 2.0, 5000.0, p.Rc, p.kappa_max, alpha,
                       p.absorb)
    return dict(mats=mats, coef=coef, dt=dt, nsteps=O.nsteps(p.duration, dt), vp=vp)


def ecyl_index(p, x, z):
    i = c_round((x - p.x0) / p.dx)          # no PML before r = 0
    j = c_round((z - p.z0) / p.dz) + p.np_used
    return i * (p.nz + 2 * p.np_used) + j


def ecyl_sources(p, s):
    """[(index, type id, samples)], Kurkjian wavelet for a Kurkjian first
    source (e_cyl_iso.c:497-502), Ricker otherwise."""
    idx = [ecyl_index(p, q[3], q[4]) for q in p.sources]
    if p.sources[0][0] == "Kurkjian":
        q = p.sources[0]
        w = O.ecyl_kurkjian(q[1], q[2], p.dt, s["mats"]["lij"].reshape(-1)[idx[0]], q[3],
                            p.dx, p.dz, p.n)
        return [(idx[0], O.ECYL_SRC["Kurkjian"], w)]
    fct = O.src_fct([q[1] for q in p.sources], [q[2] for q in p.sources], p.dt, 1.0)
    return [(k, O.ECYL_SRC[q[0]], w) for k, q, w in zip(idx, p.sources, fct)]


def run_ecyl_oracle(p, nsteps=None, fields_at=None):
    """FP64 oracle run of a whole e_cyl_iso shot: traces (1e3 * value, as
    write_trace writes them), times, optional final fields."""
    s = ecyl_setup(p)
    n = s["nsteps"] if nsteps is None else nsteps
    o = O.ECyl(p.nx, p.nz, p.np_used, p.n, p.dx, p.dz, s["dt"], s["mats"], s["coef"])
    srcs = ecyl_sources(p, s)
    recs = [(ecyl_index(p, x, z), ECYL_COMPS[c.lower()], t0, r * 1e-3)
            for (c, x, z, t0, r) in p.receivers]
    dt = s["dt"]
    tr = [[] for _ in recs]
    tt = [[] for _ in recs]
    kurk = srcs[0][1] == O.ECYL_SRC["Kurkjian"]
    for it in range(n):
        o.velocity()
        if not kurk:
            for (idx, typ, w) in srcs:
                if it < len(w):
                    o.force(idx, typ, w[it])
        o.stress()
        if kurk and it < len(srcs[0][2]):
            o.kurkjian(srcs[0][0], srcs[0][2][it])
        t = dt * (it + 1)
        for r, (idx, comp, t0, rdt) in enumerate(recs):
            if O.sample(it, dt, t0, rdt):
                tr[r].append(1e3 * o.probe(comp, idx))
                tt[r].append(t)
    fields = {f: o.get(f) for f in fields_at} if fields_at else None
    return [np.array(a) for a in tr], [np.array(a) for a in tt], fields
