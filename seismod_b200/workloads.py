"""Seeded synthetic workloads for the e_iso and a_iso_3d paths.

The reference ships no benchmark inputs and names no public dataset, so every
workload here is generated from a seed with the shapes, spacings, velocity
ranges and source/receiver geometry the five benchmark configurations name:

  cfg0  e_iso 400 x 400, dx 1 m, two flat layers, 20-cell PML, 50 Hz Bulk
        source at (200, 50), dt at CFL 0.5, 1500 steps, 64 Vz receivers z=10
  cfg1  a_iso_3d 256^3, dx 5 m, 6 flat layers 1500..4500 m/s times (1 + d),
        d a Gaussian-smoothed random field (sigma 8 cells, std 3 %),
        rho 2000, 16-cell CPML, 15 Hz Bulk source, 1000 steps,
        128 x 128 surface Vz receivers (every 2nd node)
  cfg2  e_iso 1000 x 500, seeded random layers (Vp 2000..5000, Vs=Vp/1.73,
        Gardner rho), 64 Bulk shots at z=5, 256 Vz receivers, 2000 steps
  cfg3  a_iso_3d 512^3, cfg1's model family with a new seed, 2000 steps
  cfg4  a Poisson stream of mixed e_iso / a_iso_3d requests

Every generator takes a size override so tests can run the same family small.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

from . import formats


@dataclasses.dataclass
class EIsoProblem:
    vp: np.ndarray                 # (nx, nz) m/s
    vs: np.ndarray
    rho: np.ndarray
    h: float                       # dx = dz, m
    npml: int
    dt_ms: float                   # as written in the parameter file
    duration: float                # s
    shots: list                    # per shot: list of (type, A, f, x, z)
    receivers: list                # (comp, x, z, t0_s, rdt_ms)
    x0: float = 0.0
    z0: float = 0.0
    name: str = "eiso"

    @property
    def nx(self):
        return self.vp.shape[0]

    @property
    def nz(self):
        return self.vp.shape[1]

    @property
    def dt(self):
        return self.dt_ms * 0.001

    @property
    def cells(self):
        return (self.nx + 2 * self.npml) * (self.nz + 2 * self.npml)

    def write(self, workdir, shot=0, basename=None, profile_1d=False, **par_extra):
        """Write the reference's input files for one shot; returns the .par path.
        par_extra adds .par keywords (e.g. plstr=1)."""
        os.makedirs(workdir, exist_ok=True)
        base = basename or f"{self.name}_s{shot}"
        if profile_1d:
            formats.write_model_e_1d(os.path.join(workdir, "model.dat"), self.nx, self.vp[0],
                                     self.vs[0], self.rho[0], self.h, self.x0, self.z0)
        else:
            formats.write_model_e(os.path.join(workdir, "model.dat"), self.vp, self.vs,
                                  self.rho, self.h, self.x0, self.z0)
        formats.write_src(os.path.join(workdir, "src.dat"), self.shots[shot])
        formats.write_rcv(os.path.join(workdir, "rcv.dat"),
                          [(c, (x, z), t0, r) for (c, x, z, t0, r) in self.receivers])
        par = os.path.join(workdir, "run.par")
        formats.write_par(par, "model.dat", "src.dat", "rcv.dat", base, self.duration,
                          self.dt_ms, abs_=1 if self.npml > 0 else 0, nl=self.npml, **par_extra)
        return par


@dataclasses.dataclass
class ECylProblem:
    """One e_cyl_iso run: radial (r) by vertical (z) model, azimuthal mode n."""
    vp: np.ndarray                 # (nx, nz) m/s, r slow, z fast
    vs: np.ndarray
    rho: np.ndarray
    dx: float                      # radial step, m
    dz: float
    npml: int
    dt_ms: float
    duration: float
    sources: list                  # (type, A, f, r, z); type Fr Fz Ftheta Bulk Kurkjian
    receivers: list                # (comp, r, z, t0_s, rdt_ms)
    n: int = 0                     # azimuthal mode
    absorb: int = 1                # the .par "abs" flag
    Rc: float = 1e-5
    kappa_max: float = 1.0
    alpha_max: int = 1
    x0: float = 0.0
    z0: float = 0.0
    name: str = "ecyl"

    @property
    def nx(self):
        return self.vp.shape[0]

    @property
    def nz(self):
        return self.vp.shape[1]

    @property
    def dt(self):
        return self.dt_ms * 0.001

    @property
    def np_used(self):
        """PML width the programs use: abs 0 sets it to zero (io_utils.c:293)."""
        return self.npml if self.absorb else 0

    @property
    def cells(self):
        return (self.nx + self.np_used) * (self.nz + 2 * self.np_used)

    def write(self, workdir, basename=None, profile_1d=False, **par_extra):
        """The reference's input files; returns the .par path."""
        os.makedirs(workdir, exist_ok=True)
        base = basename or self.name
        formats.write_model_ecyl(os.path.join(workdir, "model.dat"), self.vp, self.vs, self.rho,
                                 self.dx, self.dz, self.x0, self.z0, profile_1d=profile_1d)
        formats.write_src(os.path.join(workdir, "src.dat"), self.sources)
        formats.write_rcv(os.path.join(workdir, "rcv.dat"),
                          [(c, (x, z), t0, r) for (c, x, z, t0, r) in self.receivers])
        par = os.path.join(workdir, "run.par")
        extra = dict(Rc=self.Rc, kappa_max=self.kappa_max, alpha_max=self.alpha_max,
                     azimuthal_mode=self.n)
        extra.update(par_extra)
        formats.write_par(par, "model.dat", "src.dat", "rcv.dat", base, self.duration,
                          self.dt_ms, abs_=self.absorb, nl=self.npml, **extra)
        return par


def ecyl_case(nx=120, nz=160, npml=12, nsteps=300, n=0, src="Fz", seed=5, nrec=12,
              dx=1.0, dz=1.0, comps=("Vr", "Vz"), absorb=1):
    """A seeded layered cylindrical model (vp per layer, vs = vp/1.73,
    Gardner density), one source at r = 0.3 nx dr, z = 0.45 nz dz, receivers
    along the radius three cells below the source, components cycling
    through `comps`."""
    vp1 = random_layers_1d(nz, seed, vmin=1800.0, vmax=4200.0, min_thick=8)
    vp = vp1[None, :].repeat(nx, 0)
    vs = vp / 1.73
    rho = gardner(vp)
    dt_ms = 0.5 * 0.5 * (dx + dz) / (math.sqrt(2.0) * float(vp.max())) * 1e3
    A = 1.0e-6 if src == "Kurkjian" else 1.0
    sources = [(src, A, 60.0, round(0.3 * nx) * dx, round(0.45 * nz) * dz)]
    recs = []
    for k in range(nrec):
        comp = comps[k % len(comps)]
        recs.append((comp, (2 + k * (nx - 4) // max(nrec - 1, 1)) * dx,
                     (round(0.45 * nz) + 3) * dz, 0.0, dt_ms))
    return ECylProblem(vp, vs, rho, dx, dz, npml, dt_ms, steps_duration(nsteps, dt_ms),
                       sources, recs, n=n, absorb=absorb, name="ecyl")


@dataclasses.dataclass
class A3DProblem:
    vp: np.ndarray                 # (nx, ny, nz) m/s
    rho: np.ndarray
    d: tuple                       # (dx, dy, dz)
    npml: int
    dt_ms: float
    duration: float
    sources: list                  # (type, A, f, x, y, z)
    receivers: list                # (comp, x, y, z, t0_s, rdt_ms)
    Rc: float = 1e-5
    kappa_max: float = 1.0
    alpha_max: int = 1
    origin: tuple = (0.0, 0.0, 0.0)
    name: str = "a3d"

    @property
    def shape(self):
        return self.vp.shape

    @property
    def dt(self):
        return self.dt_ms * 0.001

    @property
    def cells(self):
        return int(np.prod([n + 2 * self.npml for n in self.shape]))

    def write(self, workdir, basename=None, profile_1d=False, **par_extra):
        """Write run.par, model.dat, src.dat, rcv.dat; par_extra adds .par
        keywords (e.g. segy=1)."""
        os.makedirs(workdir, exist_ok=True)
        base = basename or self.name
        if profile_1d:
            formats.write_model_a_1d(os.path.join(workdir, "model.dat"), self.shape,
                                     self.vp[0, 0], self.rho[0, 0], self.d, self.origin)
        else:
            formats.write_model_a(os.path.join(workdir, "model.dat"), self.vp, self.rho,
                                  self.d, self.origin)
        formats.write_src(os.path.join(workdir, "src.dat"), self.sources)
        formats.write_rcv(os.path.join(workdir, "rcv.dat"),
                          [(c, (x, y, z), t0, r) for (c, x, y, z, t0, r) in self.receivers])
        par = os.path.join(workdir, "run.par")
        formats.write_par(par, "model.dat", "src.dat", "rcv.dat", base, self.duration,
                          self.dt_ms, abs_=1 if self.npml > 0 else 0, nl=self.npml,
                          Rc=repr(self.Rc), kappa_max=repr(self.kappa_max),
                          alpha_max=int(self.alpha_max), **par_extra)
        return par


def steps_duration(nsteps, dt_ms):
    """A time window that the reference turns into exactly nsteps steps
    (e_iso.c:575-576 computes floor(duration/dt), plus one if short)."""
    dt = dt_ms * 0.001
    dur = nsteps * dt
    n = int(dur / dt)
    if n * dt < dur:
        n += 1
    if n != nsteps:
        dur = math.nextafter(dur, 0.0) if n > nsteps else math.nextafter(dur, 1.0)
    return dur


# ----------------------------------------------------------------------------
# cfg0: e_iso two-layer model
# ----------------------------------------------------------------------------

def cfg0(nx=400, nz=400, npml=20, nsteps=1500, nrec=64):
    h = 1.0
    z = np.arange(nz) * h
    top = z < 250.0 * (nz / 400.0)
    vp = np.where(top, 3000.0, 4000.0)[None, :].repeat(nx, 0)
    vs = np.where(top, 1700.0, 2300.0)[None, :].repeat(nx, 0)
    rho = np.where(top, 2200.0, 2500.0)[None, :].repeat(nx, 0)
    dt_ms = 0.5 * h / (math.sqrt(2.0) * 4000.0) * 1e3
    src = [("Bulk", 1.0, 50.0, 200.0 * nx / 400.0, 50.0 * nz / 400.0)]
    xr = [k * (nx - 1) / (nrec - 1) for k in range(nrec)]
    rec = [("Vz", x, 10.0 * nz / 400.0, 0.0, dt_ms) for x in xr]
    return EIsoProblem(vp, vs, rho, h, npml, dt_ms, steps_duration(nsteps, dt_ms), [src], rec,
                       name="cfg0")


# ----------------------------------------------------------------------------
# cfg1 / cfg3: a_iso_3d layered + smoothed random perturbation
# ----------------------------------------------------------------------------

def layered_perturbed_3d(n, seed, sigma=8.0, std=0.03, layers=(1500, 2100, 2700, 3300, 3900, 4500)):
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    nl = len(layers)
    k = np.arange(n)
    base = np.asarray(layers, dtype=np.float64)[np.minimum(k * nl // n, nl - 1)]
    delta = rng.standard_normal((n, n, n), dtype=np.float32)
    delta = gaussian_filter(delta, sigma=sigma, mode="wrap")
    delta *= std / float(delta.std())
    vp = base[None, None, :] * (1.0 + delta.astype(np.float64))
    return vp


def cfg1(n=256, npml=16, nsteps=1000, seed=1, rec_stride=2, nrec_side=None, dx=5.0):
    vp = layered_perturbed_3d(n, seed)
    rho = np.full_like(vp, 2000.0)
    vmax = float(vp.max())
    dt_ms = 0.5 * dx / (math.sqrt(3.0) * vmax) * 1e3
    c = (n // 2) * dx
    src = [("Bulk", 1.0, 15.0, c, c, 10 * dx)]
    nside = nrec_side or n // rec_stride
    rec = [("Vz", i * rec_stride * dx, j * rec_stride * dx, 0.0, 0.0, dt_ms)
           for i in range(nside) for j in range(nside)]
    return A3DProblem(vp, rho, (dx, dx, dx), npml, dt_ms, steps_duration(nsteps, dt_ms), src,
                      rec, Rc=1e-3, kappa_max=1.0, alpha_max=1, name="cfg1")


def cfg3(n=512, npml=16, nsteps=2000, seed=3):
    p = cfg1(n=n, npml=npml, nsteps=nsteps, seed=seed)
    p.name = "cfg3"
    return p


# ----------------------------------------------------------------------------
# cfg2: e_iso batched shots over a random-layered model
# ----------------------------------------------------------------------------

def random_layers_1d(nz, seed, vmin=2000.0, vmax=5000.0, min_thick=10, max_layers=12):
    rng = np.random.default_rng(seed)
    nlay = int(rng.integers(4, max_layers + 1))
    cuts = np.sort(rng.choice(np.arange(min_thick, max(nz - min_thick, min_thick + 1)),
                              size=min(nlay - 1, max(nz // min_thick - 2, 1)), replace=False))
    vps = rng.uniform(vmin, vmax, size=len(cuts) + 1)
    idx = np.searchsorted(cuts, np.arange(nz), side="right")
    return vps[idx]


def gardner(vp):
    return 310.0 * vp ** 0.25


def cfg2(nx=1000, nz=500, npml=20, nsteps=2000, nshots=64, nrec=256, seed=2):
    h = 1.0
    vp1 = random_layers_1d(nz, seed)
    vp = vp1[None, :].repeat(nx, 0)
    vs = vp / 1.73
    rho = gardner(vp)
    dt_ms = 0.5 * h / (math.sqrt(2.0) * float(vp.max())) * 1e3
    zs = 5.0
    shots = [[("Bulk", 1.0, 50.0, (k + 0.5) * nx / nshots * h, zs)] for k in range(nshots)]
    rec = [("Vz", k * (nx - 1) / max(nrec - 1, 1) * h, zs, 0.0, dt_ms) for k in range(nrec)]
    return EIsoProblem(vp, vs, rho, h, npml, dt_ms, steps_duration(nsteps, dt_ms), shots, rec,
                       name="cfg2")


# ----------------------------------------------------------------------------
# cfg4: serving stream
# ----------------------------------------------------------------------------

@dataclasses.dataclass
class Request:
    arrival: float                 # s after stream start
    kind: str                      # "eiso" | "a3d"
    problem: object


def eiso_request(side, nsteps, seed, npml=20, nrec=32):
    h = 1.0
    vp1 = random_layers_1d(side, seed)
    vp = vp1[None, :].repeat(side, 0)
    vs = vp / 1.73
    rho = gardner(vp)
    dt_ms = 0.5 * h / (math.sqrt(2.0) * float(vp.max())) * 1e3
    src = [("Bulk", 1.0, 50.0, side / 2 * h, 5.0)]
    rec = [("Vz", k * (side - 1) / (nrec - 1), 5.0, 0.0, dt_ms) for k in range(nrec)]
    return EIsoProblem(vp, vs, rho, h, npml, dt_ms, steps_duration(nsteps, dt_ms), [src], rec,
                       name=f"req{seed}")


def a3d_request(side, nsteps, seed, npml=16, nrec_side=16, dx=5.0):
    vp1 = random_layers_1d(side, seed, vmin=1500.0, vmax=4500.0, min_thick=4)
    vp = np.broadcast_to(vp1[None, None, :], (side, side, side)).copy()
    rho = gardner(vp)
    dt_ms = 0.5 * dx / (math.sqrt(3.0) * float(vp.max())) * 1e3
    c = side // 2 * dx
    src = [("Bulk", 1.0, 15.0, c, c, 10 * dx)]
    st = max(side // nrec_side, 1)
    rec = [("Vz", i * st * dx, j * st * dx, 0.0, 0.0, dt_ms)
           for i in range(nrec_side) for j in range(nrec_side)]
    return A3DProblem(vp, rho, (dx, dx, dx), npml, dt_ms, steps_duration(nsteps, dt_ms), src, rec,
                      Rc=1e-3, name=f"req{seed}")


def cfg4(nreq=64, rate_hz=4.0, seed=4, e_side=(200, 2000), a_side=(128, 384),
         steps=(500, 3000)):
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for r in range(nreq):
        t += float(rng.exponential(1.0 / rate_hz))
        ns = int(rng.integers(steps[0], steps[1] + 1))
        if rng.random() < 0.7:
            side = int(rng.integers(e_side[0], e_side[1] + 1))
            out.append(Request(t, "eiso", eiso_request(side, ns, seed * 1000 + r)))
        else:
            side = int(rng.integers(a_side[0], a_side[1] + 1))
            out.append(Request(t, "a3d", a3d_request(side, ns, seed * 1000 + r)))
    return out
