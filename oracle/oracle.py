"""ctypes front end of the FP64 CPU oracle (test infrastructure only).

Only the test suite, the smoke check and the CPU-baseline leg of the
benchmark import this module.  It wraps

* ``liboracle.so``            our FP64 C restatement (seismod_oracle.c), and
* ``_ref/libref_eiso.so``     the reference's own update_vx / update_vz /
                              update_txxzz / update_txz / pml_v / pml_t
                              (propagate.c:2511-2670, pml.c:39-1403),
                              compiled from its sources by oracle/Makefile,
* ``_ref/e_iso``, ``_ref/a_iso_3d``  the reference programs.

plus small pure-Python helpers for the reference's 8-region PML layout
(pml.c:54,98,133,177,213,248,290,325) used by the function-level pin.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)
_sz = C.c_size_t


def _ptr(a):
    return a.ctypes.data_as(_dp)


def build():
    """Compile the restatement (and the reference when its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    lib.orc_src_len.restype = _sz
    lib.orc_src_len.argtypes = [C.c_double, C.c_double, C.c_double]
    lib.orc_src_fct.argtypes = [_sz, _dp, _dp, C.c_double, C.c_double, _sz, _dp,
                                C.POINTER(_sz)]
    lib.orc_nsteps.restype = _sz
    lib.orc_nsteps.argtypes = [C.c_double, C.c_double]
    lib.orc_sample.restype = C.c_int
    lib.orc_sample.argtypes = [_sz, C.c_double, C.c_double, C.c_double]
    lib.orc_eiso_materials.restype = C.c_double
    lib.orc_eiso_materials.argtypes = [_sz, _sz, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
    lib.orc_eiso_profiles.argtypes = [_sz, C.c_double, _sz, _dp, _dp, _dp, _dp]
    lib.orc_eiso_new.restype = C.c_void_p
    lib.orc_eiso_new.argtypes = [_sz, _sz, _sz, C.c_double, C.c_double] + [_dp] * 8
    lib.orc_eiso_free.argtypes = [C.c_void_p]
    lib.orc_eiso_velocity.argtypes = [C.c_void_p]
    lib.orc_eiso_stress.argtypes = [C.c_void_p]
    lib.orc_eiso_add_source.argtypes = [C.c_void_p, _sz, C.c_int, C.c_double]
    lib.orc_eiso_get.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
    lib.orc_eiso_set.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
    lib.orc_eiso_set_bfp.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.orc_eiso_add_patch.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_long, C.c_long]
    lib.orc_eiso_probe.restype = C.c_double
    lib.orc_eiso_probe.argtypes = [C.c_void_p, C.c_int, _sz]
    lib.orc_a3d_pad_model.argtypes = [_sz, _sz, _sz, _sz, _dp, _dp, _dp, _dp]
    lib.orc_a3d_cfl_vpmax.restype = C.c_double
    lib.orc_a3d_cfl_vpmax.argtypes = [_sz, _sz, _dp]
    lib.orc_a3d_cpml.argtypes = [_sz, _sz, _sz, _sz, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.c_int, C.c_double, C.POINTER(_dp)]
    lib.orc_a3d_new.restype = C.c_void_p
    lib.orc_a3d_new.argtypes = [_sz, _sz, _sz, C.c_double, C.c_double, C.c_double,
                                C.c_double, _dp, _dp, C.POINTER(_dp)]
    lib.orc_a3d_free.argtypes = [C.c_void_p]
    lib.orc_a3d_velocity.argtypes = [C.c_void_p]
    lib.orc_a3d_pressure.argtypes = [C.c_void_p]
    lib.orc_a3d_add_source.argtypes = [C.c_void_p, _sz, C.c_double]
    lib.orc_a3d_get.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.orc_a3d_gather.argtypes = [C.c_void_p, _sz, C.POINTER(C.c_int), C.POINTER(_sz), _dp]
    lib.orc_a3d_set_bfp.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.orc_a3d_set.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.orc_a3d_probe.restype = C.c_double
    lib.orc_a3d_probe.argtypes = [C.c_void_p, C.c_int, _sz]
    return lib


def _load_ecyl(lib):
    lib.orc_ecyl_materials.restype = C.c_double
    lib.orc_ecyl_materials.argtypes = [_sz, _sz] + [_dp] * 11
    lib.orc_ecyl_cpml.argtypes = [_sz] + [C.c_double] * 8 + [C.c_int, C.POINTER(_dp)]
    lib.orc_ecyl_kurkjian.restype = _sz
    lib.orc_ecyl_kurkjian.argtypes = [C.c_double] * 7 + [C.c_int, _sz, _dp]
    lib.orc_ecyl_new.restype = C.c_void_p
    lib.orc_ecyl_new.argtypes = [_sz, _sz, _sz, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.POINTER(_dp), C.POINTER(_dp)]
    lib.orc_ecyl_free.argtypes = [C.c_void_p]
    lib.orc_ecyl_velocity.argtypes = [C.c_void_p]
    lib.orc_ecyl_stress.argtypes = [C.c_void_p]
    lib.orc_ecyl_force.argtypes = [C.c_void_p, _sz, C.c_int, C.c_double]
    lib.orc_ecyl_kurkjian_add.argtypes = [C.c_void_p, _sz, C.c_double]
    lib.orc_ecyl_get.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.orc_ecyl_set.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.orc_ecyl_probe.restype = C.c_double
    lib.orc_ecyl_probe.argtypes = [C.c_void_p, C.c_int, _sz]


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _load()
        _load_ecyl(_LIB)
    return _LIB


# ----------------------------------------------------------------------------
# shared set-up
# ----------------------------------------------------------------------------

def src_fct(A, f, dt, fac=1.0):
    """Ricker wavelets exactly as src.c:43-65 computes them -> list of arrays."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    n = len(A)
    maxlen = max(lib().orc_src_len(float(fi), dt, fac) for fi in f)
    fct = np.zeros(n * maxlen)
    ln = (_sz * n)()
    lib().orc_src_fct(n, _ptr(A), _ptr(f), dt, fac, maxlen, _ptr(fct), ln)
    return [fct[s * maxlen: s * maxlen + ln[s]].copy() for s in range(n)]


def nsteps(duration, dt):
    return int(lib().orc_nsteps(duration, dt))


def sample(it, dt, t0, rdt):
    return bool(lib().orc_sample(it, dt, t0, rdt))


# ----------------------------------------------------------------------------
# e_iso
# ----------------------------------------------------------------------------

def eiso_materials(vp, vs, rho):
    """(la, mu, l2m, b, bm, vpmax) from nx x nz arrays, e_iso.c:423-462."""
    nx, nz = vp.shape
    vp, vs, rho = (np.ascontiguousarray(a, dtype=np.float64) for a in (vp, vs, rho))
    out = [np.zeros((nx, nz)) for _ in range(5)]
    vpmax = lib().orc_eiso_materials(nx, nz, _ptr(vp), _ptr(vs), _ptr(rho),
                                     *[_ptr(a) for a in out])
    return (*out, vpmax)


def eiso_profiles(npml, h, vp):
    vp = np.ascontiguousarray(vp, dtype=np.float64)
    d, dh, dH = np.zeros(npml), np.zeros(npml), np.zeros(npml + 1)
    lib().orc_eiso_profiles(npml, h, vp.size, _ptr(vp), _ptr(d), _ptr(dh), _ptr(dH))
    return d, dh, dH


FIELDS_E = {"vx": 0, "vz": 1, "txx": 2, "tzz": 3, "txz": 4}
PARTS = {"total": 0, "x": 1, "z": 2}


class EIso:
    """FP64 e_iso state on the padded grid (oracle)."""

    def __init__(self, nx, nz, npml, h, dt, la, mu, l2m, b, bm, d, dh, dH):
        self.nx, self.nz, self.np, self.h, self.dt = nx, nz, npml, h, dt
        self.NX, self.NZ = nx + 2 * npml, nz + 2 * npml
        self._keep = [np.ascontiguousarray(a, dtype=np.float64)
                      for a in (la, mu, l2m, b, bm, d, dh, dH)]
        self.h_ = lib().orc_eiso_new(nx, nz, npml, h, dt, *[_ptr(a) for a in self._keep])

    def __del__(self):
        if getattr(self, "h_", None):
            lib().orc_eiso_free(self.h_)
            self.h_ = None

    def velocity(self):
        lib().orc_eiso_velocity(self.h_)

    def stress(self):
        lib().orc_eiso_stress(self.h_)

    def add_source(self, index, typ, value):
        lib().orc_eiso_add_source(self.h_, int(index), int(typ), float(value))

    def get(self, field, part="total"):
        out = np.zeros((self.NX, self.NZ))
        lib().orc_eiso_get(self.h_, FIELDS_E[field], PARTS[part], _ptr(out))
        return out

    def set(self, field, part, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.NX, self.NZ)
        lib().orc_eiso_set(self.h_, FIELDS_E[field], PARTS[part], _ptr(a))

    def set_bfp(self, block, axis="x"):
        """checker mode: the state a step stores is rounded to 16-bit block
        floating point with blocks of `block` cells along x or z (0: FP64)"""
        lib().orc_eiso_set_bfp(self.h_, int(block), 0 if axis == "x" else 1)

    def add_patch(self, X0, Z0, rows, cols):
        """checker mode: padded cells the block storage keeps exact"""
        lib().orc_eiso_add_patch(self.h_, int(X0), int(Z0), int(rows), int(cols))

    def probe(self, field, index):
        return lib().orc_eiso_probe(self.h_, FIELDS_E[field], int(index))


# ----------------------------------------------------------------------------
# a_iso_3d
# ----------------------------------------------------------------------------

def a3d_pad_model(vp, rho, npml):
    nx, ny, nz = vp.shape
    vp, rho = (np.ascontiguousarray(a, dtype=np.float64) for a in (vp, rho))
    shp = (nx + 2 * npml, ny + 2 * npml, nz + 2 * npml)
    vpp, rhop = np.zeros(shp), np.zeros(shp)
    lib().orc_a3d_pad_model(nx, ny, nz, npml, _ptr(vp), _ptr(rho), _ptr(vpp), _ptr(rhop))
    return vpp, rhop


def a3d_cfl_vpmax(nx, nz, vp_pad):
    v = np.ascontiguousarray(vp_pad, dtype=np.float64)
    return lib().orc_a3d_cfl_vpmax(nx, nz, _ptr(v))


def a3d_cpml(npml, shape2, dx, dy, dz, dt, pml_order=2.0, vmax=5000.0, Rc=1e-5,
             kappa_max=1.0, alpha_max_flag=1, f0=0.0):
    """18 coefficient arrays in the order ax bx kx ay by ky az bz kz + _h."""
    n2 = list(shape2)
    arrs = [np.zeros(n2[c // 3]) for c in range(9)] + \
           [np.zeros(n2[(c - 9) // 3] - 1) for c in range(9, 18)]
    P = (_dp * 18)(*[_ptr(a) for a in arrs])
    lib().orc_a3d_cpml(npml, n2[0], n2[1], n2[2], dx, dy, dz, dt, pml_order, vmax, Rc,
                       kappa_max, alpha_max_flag, f0, P)
    return arrs


FIELDS_A = {"vx": 0, "vy": 1, "vz": 2, "p": 3}


class A3D:
    """FP64 a_iso_3d state (oracle), reference padded layout."""

    def __init__(self, vp_pad, rho_pad, dx, dy, dz, dt, coef):
        self.shape = vp_pad.shape
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (vp_pad, rho_pad)]
        self._coef = [np.ascontiguousarray(a, dtype=np.float64) for a in coef]
        P = (_dp * 18)(*[_ptr(a) for a in self._coef])
        n = self.shape
        self.h_ = lib().orc_a3d_new(n[0], n[1], n[2], dx, dy, dz, dt,
                                    _ptr(self._keep[0]), _ptr(self._keep[1]), P)

    def __del__(self):
        if getattr(self, "h_", None):
            lib().orc_a3d_free(self.h_)
            self.h_ = None

    def velocity(self):
        lib().orc_a3d_velocity(self.h_)

    def pressure(self):
        lib().orc_a3d_pressure(self.h_)

    def add_source(self, index, value):
        lib().orc_a3d_add_source(self.h_, int(index), float(value))

    def get(self, field):
        out = np.zeros(self.shape)
        lib().orc_a3d_get(self.h_, FIELDS_A[field], _ptr(out))
        return out

    def set(self, field, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        lib().orc_a3d_set(self.h_, FIELDS_A[field], _ptr(a))

    def probe(self, field, index):
        return lib().orc_a3d_probe(self.h_, FIELDS_A[field], int(index))

    def gather(self, fields, index):
        """values of fields[r] at index[r] (arrays of field ids and indices)"""
        f = np.ascontiguousarray(fields, dtype=np.int32)
        q = np.ascontiguousarray(index, dtype=np.uintp)
        out = np.zeros(len(q))
        lib().orc_a3d_gather(self.h_, len(q), f.ctypes.data_as(C.POINTER(C.c_int)),
                             q.ctypes.data_as(C.POINTER(_sz)), _ptr(out))
        return out

    def set_bfp(self, block, axis="y"):
        """checker mode: round the stored state to 16-bit block floating
        point with blocks of `block` cells along y or z (0: FP64 storage)"""
        lib().orc_a3d_set_bfp(self.h_, int(block), 1 if axis == "y" else 2)


# ----------------------------------------------------------------------------
# e_cyl_iso
# ----------------------------------------------------------------------------

FIELDS_C = {"vr": 0, "vt": 1, "vz": 2, "trr": 3, "ttt": 4, "tzz": 5, "trz": 6, "trt": 7,
            "ttz": 8, "div": 9, "curl": 10}
ECYL_MATS = ("lij", "l2mij", "mu", "mui", "muj", "bi", "bj", "bij")
ECYL_SRC = {"Bulk": 6, "Fr": 9, "Ftheta": 10, "Fz": 11, "Kurkjian": 12}


def ecyl_materials(vp, vs, rho):
    """Padded (nx2, nz2) models -> (dict of the 8 averaged materials, vpmax)."""
    vp, vs, rho = (np.ascontiguousarray(a, dtype=np.float64) for a in (vp, vs, rho))
    out = {k: np.zeros(vp.shape) for k in ECYL_MATS}
    vmax = lib().orc_ecyl_materials(vp.shape[0], vp.shape[1], _ptr(vp), _ptr(vs), _ptr(rho),
                                    *[_ptr(out[k]) for k in ECYL_MATS])
    return out, vmax


def ecyl_cpml(npml, dx, dz, dt, order=2.0, vmax=5000.0, Rc=1e-5, kappa_max=1.0,
              alpha_max=0.0, absorb=1):
    """The 15 coefficient arrays of pml.c:2107-2185 (9 of npml, 6 of npml+1)."""
    arrs = [np.zeros(npml if k < 9 else npml + 1) for k in range(15)]
    ptrs = (_dp * 15)(*[_ptr(a) for a in arrs])
    lib().orc_ecyl_cpml(npml, dx, dz, dt, order, vmax, Rc, kappa_max, alpha_max, int(absorb),
                        ptrs)
    return arrs


def ecyl_kurkjian(A, f, dt, lij_at_src, x_src, dx, dz, n):
    maxlen = int(np.ceil(2.0 / f / dt)) + 2
    out = np.zeros(maxlen)
    k = lib().orc_ecyl_kurkjian(A, f, dt, lij_at_src, x_src, dx, dz, int(n), maxlen, _ptr(out))
    return out[:k].copy()


class ECyl:
    """FP64 e_cyl_iso state: padded nx2 = nx + npml by nz2 = nz + 2 npml."""

    def __init__(self, nx, nz, npml, n, dx, dz, dt, mats, coef):
        self.shape = (nx + npml, nz + 2 * npml)
        self._mats = [np.ascontiguousarray(mats[k], dtype=np.float64) for k in ECYL_MATS]
        self._coef = [np.ascontiguousarray(c, dtype=np.float64) for c in coef]
        mp = (_dp * 8)(*[_ptr(a) for a in self._mats])
        cp = (_dp * 15)(*[_ptr(a) for a in self._coef])
        self.h_ = lib().orc_ecyl_new(nx, nz, npml, int(n), dx, dz, dt, mp, cp)

    def __del__(self):
        if getattr(self, "h_", None):
            lib().orc_ecyl_free(self.h_)
            self.h_ = None

    def velocity(self):
        lib().orc_ecyl_velocity(self.h_)

    def stress(self):
        lib().orc_ecyl_stress(self.h_)

    def force(self, index, typ, value):
        lib().orc_ecyl_force(self.h_, int(index), int(typ), float(value))

    def kurkjian(self, index, value):
        lib().orc_ecyl_kurkjian_add(self.h_, int(index), float(value))

    def get(self, field):
        out = np.zeros(self.shape)
        lib().orc_ecyl_get(self.h_, FIELDS_C[field], _ptr(out))
        return out

    def set(self, field, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        lib().orc_ecyl_set(self.h_, FIELDS_C[field], _ptr(a))

    def probe(self, comp, index):
        return lib().orc_ecyl_probe(self.h_, FIELDS_C[comp], int(index))


# ----------------------------------------------------------------------------
# the reference itself
# ----------------------------------------------------------------------------

def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, f))
               for f in ("e_iso", "a_iso_3d", "libref_eiso.so"))


def pml_regions(nx, nz, npml):
    """The reference's 8 PML regions as (offset, x0, nxr, z0, nzr) in padded
    coordinates, in storage order (pml.c:54-325): UL corner, left strip, LL
    corner, upper strip, lower strip, UR corner, right strip, LR corner.
    Within a region the index is i*nzr + j."""
    P = npml
    regs = [
        (0, P, 0, P),               # UL
        (0, P, P, nz),              # left
        (0, P, P + nz, P),          # LL
        (P, nx, 0, P),              # upper
        (P, nx, P + nz, P),         # lower
        (P + nx, P, 0, P),          # UR
        (P + nx, P, P, nz),         # right
        (P + nx, P, P + nz, P),     # LR
    ]
    out, off = [], 0
    for (x0, nxr, z0, nzr) in regs:
        out.append((off, x0, nxr, z0, nzr))
        off += nxr * nzr
    return out, off


def padded_to_regions(a, nx, nz, npml):
    regs, total = pml_regions(nx, nz, npml)
    out = np.zeros(total)
    for (off, x0, nxr, z0, nzr) in regs:
        out[off:off + nxr * nzr] = a[x0:x0 + nxr, z0:z0 + nzr].reshape(-1)
    return out


def regions_to_padded(r, nx, nz, npml, into):
    regs, _ = pml_regions(nx, nz, npml)
    for (off, x0, nxr, z0, nzr) in regs:
        into[x0:x0 + nxr, z0:z0 + nzr] = r[off:off + nxr * nzr].reshape(nxr, nzr)
    return into


class _Grid(C.Structure):
    # struct grid, structs.h:62-70 (with struct abs_params, :49-60)
    _fields_ = [("coord", C.c_int), ("nx", _sz), ("nz", _sz), ("nx2", _sz), ("nz2", _sz),
                ("Qdamping", C.c_short), ("x0", C.c_double), ("z0", C.c_double),
                ("dx", C.c_double), ("dz", C.c_double),
                ("np", _sz), ("median", C.c_short), ("alpha_max", C.c_short),
                ("alfa", C.c_double), ("vmax", C.c_double), ("pmlOrder", C.c_double),
                ("Rc", C.c_double), ("kappa_max", C.c_double),
                ("gobx", C.c_void_p), ("gobz", C.c_void_p)]


class RefEIso:
    """The reference's own e_iso update functions on reference-layout arrays."""

    def __init__(self, nx, nz, npml, h, dt, la, mu, l2m, b, bm, d, dh, dH, lrfix=False):
        # lrfix: the build whose lower-right corner reads [nx*nz-1] (pml.c:1044-1084)
        name = "libref_eiso_lrfix.so" if lrfix else "libref_eiso.so"
        self.L = C.CDLL(os.path.join(REF_DIR, name))
        self.nx, self.nz, self.np, self.h, self.dt = nx, nz, npml, h, dt
        self.g = _Grid(coord=0, nx=nx, nz=nz, nx2=nx, nz2=nz, dx=h, dz=h, np=0)
        self.mat = {k: np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
                    for k, v in dict(la=la, mu=mu, l2m=l2m, b=b, bm=bm).items()}
        self.prof = [np.ascontiguousarray(a, dtype=np.float64) for a in (d, dh, dH)]
        _, self.npml_cells = pml_regions(nx, nz, npml)
        self.f = {k: np.zeros(nx * nz) for k in ("vx", "vz", "txx", "tzz", "txz")}
        self.s = {k: np.zeros(self.npml_cells) for k in
                  ("vx_x", "vx_z", "vz_x", "vz_z", "txx_x", "txx_z", "tzz_x", "tzz_z",
                   "txz_x", "txz_z")}

    def velocity(self):
        L, g, f, s, m = self.L, C.byref(self.g), self.f, self.s, self.mat
        dt, h, P = C.c_double(self.dt), C.c_double(self.h), _sz(self.np)
        L.update_vx(_ptr(f["vx"]), _ptr(f["txx"]), _ptr(f["txz"]), _ptr(m["b"]),
                    _ptr(s["txx_x"]), _ptr(s["txx_z"]), _ptr(s["txz_x"]), _ptr(s["txz_z"]),
                    g, dt, h, P)
        L.update_vz(_ptr(f["vz"]), _ptr(f["txz"]), _ptr(f["tzz"]), _ptr(m["bm"]),
                    _ptr(s["txz_x"]), _ptr(s["txz_z"]), _ptr(s["tzz_x"]), _ptr(s["tzz_z"]),
                    g, dt, h, P)
        L.pml_v(*[_ptr(s[k]) for k in ("vx_x", "vx_z", "vz_x", "vz_z", "txx_x", "txx_z",
                                       "tzz_x", "tzz_z", "txz_x", "txz_z")],
                *[_ptr(a) for a in self.prof], _ptr(f["txx"]), _ptr(f["tzz"]),
                _ptr(f["txz"]), _ptr(m["b"]), _ptr(m["bm"]), _sz(self.nx), _sz(self.nz),
                P, dt, h)

    def stress(self):
        L, g, f, s, m = self.L, C.byref(self.g), self.f, self.s, self.mat
        dt, h, P = C.c_double(self.dt), C.c_double(self.h), _sz(self.np)
        L.update_txxzz(_ptr(f["txx"]), _ptr(f["tzz"]), _ptr(f["vx"]), _ptr(f["vz"]),
                       _ptr(m["la"]), _ptr(m["l2m"]), _ptr(s["vx_x"]), _ptr(s["vx_z"]),
                       _ptr(s["vz_x"]), _ptr(s["vz_z"]), g, dt, h, P)
        L.update_txz(_ptr(f["txz"]), _ptr(f["vx"]), _ptr(f["vz"]), _ptr(m["mu"]),
                     _ptr(s["vx_x"]), _ptr(s["vx_z"]), _ptr(s["vz_x"]), _ptr(s["vz_z"]),
                     g, dt, h, P)
        L.pml_t(*[_ptr(s[k]) for k in ("vx_x", "vx_z", "vz_x", "vz_z", "txx_x", "txx_z",
                                       "tzz_x", "tzz_z", "txz_x", "txz_z")],
                *[_ptr(a) for a in self.prof], _ptr(f["vx"]), _ptr(f["vz"]),
                _ptr(m["la"]), _ptr(m["l2m"]), _ptr(m["mu"]), _sz(self.nx), _sz(self.nz),
                P, dt, h)

    def padded(self, field, part="total"):
        """Field in our padded layout: totals inside, parts summed outside."""
        NX, NZ, P = self.nx + 2 * self.np, self.nz + 2 * self.np, self.np
        out = np.zeros((NX, NZ))
        if part in ("total", "x"):
            regions_to_padded(self.s[field + "_x"], self.nx, self.nz, P, out)
        if part in ("total", "z"):
            tmp = regions_to_padded(self.s[field + "_z"], self.nx, self.nz, P, np.zeros((NX, NZ)))
            out += tmp
        if part == "total":
            out[P:P + self.nx, P:P + self.nz] = self.f[field].reshape(self.nx, self.nz)
        return out


def run_reference(program, parfile, cwd, timeout=3600):
    """Run oracle/_ref/<program> -p parfile in cwd; returns wall seconds."""
    import time
    exe = os.path.join(REF_DIR, program)
    t0 = time.perf_counter()
    subprocess.run([exe, "-p", parfile], cwd=cwd, check=True, timeout=timeout,
                   stdout=subprocess.DEVNULL)
    return time.perf_counter() - t0


def read_trc(path):
    """A reference .trc file (write_trace, io_utils.c:1744-1768) -> (t, v)."""
    a = np.loadtxt(path, ndmin=2)
    return a[:, 0], a[:, 1]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)


