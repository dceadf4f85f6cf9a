"""Generate the golden trace fixtures from the reference programs.

Run in a container where the reference sources are present, after
``make -C oracle REF=<reference source tree>`` has built oracle/_ref/:

    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py ecyl     # the e_cyl_iso ones only

Each case is a small seeded problem.  The reference program (e_iso,
e_iso_lrfix for nx > nz, a_iso_3d, or e_cyl_iso_serial) runs it from its own input files and
the traces it writes are stored, together with the complete problem, in
tests/golden/<case>.npz.  The tests rebuild the problem from the fixture, so
nothing at test time needs the reference.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from seismod_b200 import formats as F  # noqa: E402
from seismod_b200 import workloads as W  # noqa: E402


def eiso_cases():
    cases = {}
    # cfg0 family, square grid
    p = W.cfg0(nx=60, nz=60, npml=8, nsteps=400, nrec=8)
    p.receivers = [("Vz" if k % 2 else "Vx", x, z, t0, r) for k, (_, x, z, t0, r) in
                   enumerate(p.receivers)]
    p.name = "eiso_square"
    cases[p.name] = (p, "e_iso")
    # nx < nz, heterogeneous model, several source types, subsampled records
    rng = np.random.default_rng(11)
    nx, nz = 40, 64
    vp = 2500 + 1500 * rng.random((nx, nz))
    vs = vp / (1.6 + 0.3 * rng.random((nx, nz)))
    rho = 1800 + 700 * rng.random((nx, nz))
    dt_ms = 0.45 / (np.sqrt(2) * vp.max()) * 1e3
    srcs = [("Sx", 2.0, 60.0, 12.0, 20.0), ("Sz", 1.0, 60.0, 25.0, 30.0),
            ("Sxz", 0.5, 60.0, 18.0, 44.0)]
    recs = [("Vx", 5.0, 5.0, 0.0, dt_ms), ("Vz", 33.0, 60.0, 0.002, 2 * dt_ms),
            ("Vz", 20.0, 10.0, 0.0, 3 * dt_ms), ("Vx", 39.0, 0.0, 0.0, dt_ms)]
    q = W.EIsoProblem(vp, vs, rho, 1.0, 6, dt_ms, W.steps_duration(350, dt_ms), [srcs],
                      recs, name="eiso_tall")
    cases[q.name] = (q, "e_iso")
    # nx > nz (the reference reads past its arrays there; the corrected build is used)
    r = W.cfg2(nx=64, nz=40, npml=7, nsteps=300, nshots=2, nrec=6, seed=5)
    r.name = "eiso_wide"
    cases[r.name] = (r, "e_iso_lrfix")
    return cases


def a3d_cases():
    cases = {}
    p = W.cfg1(n=24, npml=6, nsteps=200, seed=9)
    p.sources = [("Bulk", 1.0, 40.0, 60.0, 55.0, 50.0)]
    p.receivers = [("Vz", 5.0, 10.0, 0.0, 0.0, p.dt_ms), ("Vx", 80.0, 35.0, 15.0, 0.0, p.dt_ms),
                   ("Vy", 60.0, 15.0, 70.0, 0.0, 2 * p.dt_ms),
                   ("Vz", 55.0, 60.0, 45.0, 0.0, p.dt_ms)]
    p.name = "a3d_cube"
    cases[p.name] = (p, "a_iso_3d")
    # rectangular box, kappa_max > 1, alpha off, two sources, 1-D model file
    nx, ny, nz = 18, 22, 26
    vp1 = np.linspace(1800.0, 3200.0, nz)
    vp = np.broadcast_to(vp1, (nx, ny, nz)).copy()
    rho = np.broadcast_to(np.linspace(1900.0, 2300.0, nz), (nx, ny, nz)).copy()
    dx = 4.0
    dt_ms = 0.45 * dx / (np.sqrt(3) * 3200.0) * 1e3
    srcs = [("Bulk", 1.0, 50.0, 36.0, 40.0, 48.0), ("Sz", 0.5, 50.0, 20.0, 60.0, 30.0)]
    recs = [("Vx", 4.0, 8.0, 0.0, 0.0, dt_ms), ("Vz", 68.0, 84.0, 100.0, 0.0, dt_ms),
            ("Vy", 36.0, 40.0, 60.0, 0.001, dt_ms)]
    q = W.A3DProblem(vp, rho, (dx, dx, dx), 5, dt_ms, W.steps_duration(180, dt_ms), srcs, recs,
                     Rc=1e-4, kappa_max=2.0, alpha_max=0, name="a3d_box")
    cases[q.name] = (q, "a_iso_3d_1d")
    return cases


ECYL_COMPS = ("Vr", "Vz", "Vtheta", "trr", "tzz", "trz", "trtheta", "tthetatheta", "tthetaz",
              "div", "curl")


def ecyl_cases():
    """e_cyl_iso, run by the reference built without OpenMP (its force
    sources are added once per thread under OpenMP, see oracle/Makefile)."""
    cases = {}
    p = W.ecyl_case(nx=48, nz=56, npml=8, nsteps=220, n=0, src="Fz", nrec=22, comps=ECYL_COMPS,
                    seed=21)
    p.name = "ecyl_m0"
    cases[p.name] = p
    q = W.ecyl_case(nx=44, nz=60, npml=7, nsteps=200, n=1, src="Kurkjian", nrec=22,
                    comps=ECYL_COMPS, seed=22)
    q.name = "ecyl_m1_kurkjian"
    cases[q.name] = q
    r = W.ecyl_case(nx=40, nz=50, npml=6, nsteps=200, n=2, src="Bulk", nrec=11,
                    comps=ECYL_COMPS, seed=23, dx=1.5, dz=1.0)
    r.alpha_max, r.kappa_max, r.Rc = 0, 1.5, 1e-4
    r.receivers = [(c, x, z, 0.002 if k % 3 == 0 else 0.0, (2 if k % 2 else 1) * rdt)
                   for k, (c, x, z, t0, rdt) in enumerate(r.receivers)]
    r.name = "ecyl_m2_bulk"
    cases[r.name] = r
    u = W.ecyl_case(nx=36, nz=40, npml=6, nsteps=160, n=0, src="Fr", nrec=11, comps=ECYL_COMPS,
                    seed=24, absorb=0)
    u.name = "ecyl_noabs"
    cases[u.name] = u
    return cases


def _save(path, p, kind, program, t, v):
    meta = dict(kind=kind, program=program, name=p.name, npml=p.npml, dt_ms=p.dt_ms,
                duration=p.duration)
    arrays = dict(ref_t=np.concatenate(t), ref_v=np.concatenate(v),
                  ref_n=np.array([len(a) for a in v], dtype=np.int64))
    if kind == "eiso":
        meta.update(h=p.h, x0=p.x0, z0=p.z0, shots=p.shots[:1], receivers=p.receivers)
        arrays.update(vp=p.vp, vs=p.vs, rho=p.rho)
    elif kind == "ecyl":
        meta.update(dx=p.dx, dz=p.dz, x0=p.x0, z0=p.z0, sources=p.sources,
                    receivers=p.receivers, n=p.n, absorb=p.absorb, Rc=p.Rc,
                    kappa_max=p.kappa_max, alpha_max=p.alpha_max)
        arrays.update(vp=p.vp, vs=p.vs, rho=p.rho)
    else:
        meta.update(d=list(p.d), origin=list(p.origin), sources=p.sources,
                    receivers=p.receivers, Rc=p.Rc, kappa_max=p.kappa_max,
                    alpha_max=p.alpha_max)
        arrays.update(vp=p.vp, rho=p.rho)
    np.savez_compressed(path, meta=json.dumps(meta), **arrays)


def segy_case():
    """a_iso_3d with SEG-Y output (segy 1): the reference's .sgy bytes."""
    p = W.cfg1(n=20, npml=5, nsteps=120, seed=13)
    p.sources = [("Bulk", 1.0, 40.0, 50.0, 45.0, 40.0)]
    p.receivers = [("Vz", 5.0, 10.0, 0.0, 0.0, p.dt_ms), ("Vx", 70.0, 35.0, 15.0, 0.0, p.dt_ms),
                   ("Vy", 60.0, 15.0, 50.0, 0.0, p.dt_ms), ("Vz", 45.0, 60.0, 35.0, 0.0, p.dt_ms)]
    p.name = "a3d_segy"
    return p


def make_segy_fixture():
    p = segy_case()
    d = tempfile.mkdtemp(prefix="golden_")
    par = p.write(d, segy=1, shotpoint=7)
    O.run_reference("a_iso_3d", par, d)
    with open(os.path.join(d, "segy", f"{p.name}.sgy"), "rb") as f:
        sgy = np.frombuffer(f.read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "segy_a3d.npz"), sgy=sgy)
    print(f"{p.name}: a_iso_3d segy -> {sgy.size} bytes")


def make_ecyl_fixtures():
    for name, p in ecyl_cases().items():
        d = tempfile.mkdtemp(prefix="golden_")
        par = p.write(d)
        O.run_reference("e_cyl_iso_serial", par, d)
        t, v = F.read_traces(d, p.name, len(p.receivers))
        _save(os.path.join(HERE, f"{name}.npz"), p, "ecyl", "e_cyl_iso_serial", t, v)
        print(f"{name}: e_cyl_iso_serial -> {[len(a) for a in v]}")


def main():
    if not O.ref_available():
        O.build()
    if sys.argv[1:] == ["ecyl"]:   # only the e_cyl_iso fixtures
        make_ecyl_fixtures()
        return
    make_segy_fixture()
    make_ecyl_fixtures()
    for name, (p, prog) in {**eiso_cases(), **a3d_cases()}.items():
        d = tempfile.mkdtemp(prefix="golden_")
        if prog.startswith("a_iso_3d"):
            par = p.write(d, profile_1d=prog.endswith("_1d"))
            O.run_reference("a_iso_3d", par, d)
            t, v = F.read_traces(d, p.name, len(p.receivers))
            kind, base = "a3d", p.name
        else:
            par = p.write(d, shot=0, basename=p.name)
            O.run_reference(prog, par, d)
            t, v = F.read_traces(d, p.name, len(p.receivers))
            kind, base = "eiso", p.name
        _save(os.path.join(HERE, f"{base}.npz"), p, kind, prog, t, v)
        print(f"{name}: {prog} -> {[len(a) for a in v]}")


def load(path):
    """Rebuild (problem, kind, program, ref_t list, ref_v list) from a fixture."""
    z = np.load(path, allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    if meta["kind"] == "eiso":
        p = W.EIsoProblem(z["vp"], z["vs"], z["rho"], meta["h"], meta["npml"], meta["dt_ms"],
                          meta["duration"], [[tuple(s) for s in meta["shots"][0]]],
                          [tuple(r) for r in meta["receivers"]], meta["x0"], meta["z0"],
                          name=meta["name"])
    elif meta["kind"] == "ecyl":
        p = W.ECylProblem(z["vp"], z["vs"], z["rho"], meta["dx"], meta["dz"], meta["npml"],
                          meta["dt_ms"], meta["duration"], [tuple(s) for s in meta["sources"]],
                          [tuple(r) for r in meta["receivers"]], n=meta["n"],
                          absorb=meta["absorb"], Rc=meta["Rc"], kappa_max=meta["kappa_max"],
                          alpha_max=meta["alpha_max"], x0=meta["x0"], z0=meta["z0"],
                          name=meta["name"])
    else:
        p = W.A3DProblem(z["vp"], z["rho"], tuple(meta["d"]), meta["npml"], meta["dt_ms"],
                         meta["duration"], [tuple(s) for s in meta["sources"]],
                         [tuple(r) for r in meta["receivers"]], meta["Rc"], meta["kappa_max"],
                         meta["alpha_max"], tuple(meta["origin"]), name=meta["name"])
    cut = np.cumsum(z["ref_n"])[:-1]
    return (p, meta["kind"], meta["program"], np.split(z["ref_t"], cut),
            np.split(z["ref_v"], cut))


if __name__ == "__main__":
    main()
