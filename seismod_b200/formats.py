"""Writers and readers for the reference's input and output file formats.

The formats are the ones the reference programs read and write:

* parameter file   ``value  # keyword, comment`` lines (io_utils.c:214-292);
                   the comma is required by the reference parser.
* e_iso model      ``nx nz / dx dz / x0 z0 / isotropic_elastic`` then one
                   ``vp vs rho`` line per node, x slow, z fast; a single
                   column (nz lines) is a 1-D profile (io_utils.c:892-947).
* a_iso_3d model   ``nx ny nz / dx dy dz / x0 y0 z0 / isotropic_acoustic_3d``
                   then ``vp rho`` per node, x slowest, z fastest; a single
                   column is a 1-D profile (io_utils.c:1029-1153).
* source file      ``nsrc / ntemplate`` then per source ``type / A / f /
                   coordinates`` (io_utils.c:1432-1589).
* output file      ``nrec`` then per record ``comp / Trace / coordinates /
                   t0 (s) / dt (ms)`` (io_utils.c:1592-1741).
* e_cyl_iso model  ``nr nz / dr dz / r0 z0 / isotropic_elastic_cyl`` then
                   ``vp vs rho`` per node, r fast within each z row; a single
                   row is a radial profile (io_utils.c:949-1027).
* trace file       ``trc/<base>/<base>_<n>.trc``: ``"%le    %le"`` of time
                   and 1e3 * velocity (io_utils.c:1744-1768).
* binary model     this package's own: the same model values without text
                   parsing (write_model_bin); the drop-in programs read either.
"""
from __future__ import annotations

import os

import numpy as np


def _num(x):
    """Shortest text that parses back to the same double."""
    return repr(float(x))


def write_par(path, model, source, output, basename, duration, dt_ms, abs_=1, nl=20,
              **extra):
    lines = [
        f"{model}    # model, model file",
        f"{source}    # source, source file",
        f"{output}    # output, description of output records",
        f"{basename}    # basename, common for all output files",
        f"{_num(duration)}    # time, length of time window in s",
        f"{_num(dt_ms)}    # dt, time step in ms",
        f"{int(abs_)}    # abs, apply absorbing boundary",
        f"{int(nl)}    # nl, number of absorbing layers",
    ]
    for k, v in extra.items():
        lines.append(f"{v}    # {k}, extra")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def _write_rows(f, cols):
    data = np.column_stack([np.asarray(c, dtype=np.float64).reshape(-1) for c in cols])
    np.savetxt(f, data, fmt="%.17g")


def write_model_e(path, vp, vs, rho, dx, x0=0.0, z0=0.0):
    """vp, vs, rho: (nx, nz) arrays, or (nz,) 1-D profiles with nx given by
    passing a tuple (nx, profile) is not supported: use write_model_e_1d."""
    nx, nz = vp.shape
    with open(path, "w") as f:
        f.write(f"{nx} {nz}\n{_num(dx)} {_num(dx)}\n{_num(x0)} {_num(z0)}\nisotropic_elastic\n")
        _write_rows(f, (vp, vs, rho))


def write_model_e_1d(path, nx, vp, vs, rho, dx, x0=0.0, z0=0.0):
    nz = len(vp)
    with open(path, "w") as f:
        f.write(f"{nx} {nz}\n{_num(dx)} {_num(dx)}\n{_num(x0)} {_num(z0)}\nisotropic_elastic\n")
        _write_rows(f, (vp, vs, rho))


def write_model_ecyl(path, vp, vs, rho, dx, dz, x0=0.0, z0=0.0, profile_1d=False):
    """e_cyl_iso model (io_utils.c:949-1027): ``nr nz / dr dz / r0 z0 /
    isotropic_elastic_cyl`` then ``vp vs rho`` per node, r fastest within
    each z row; with profile_1d only the first row (a radial profile, copied
    down every row by the reader)."""
    nx, nz = vp.shape
    with open(path, "w") as f:
        f.write(f"{nx} {nz}\n{_num(dx)} {_num(dz)}\n{_num(x0)} {_num(z0)}\nisotropic_elastic_cyl\n")
        rows = 1 if profile_1d else nz
        for j in range(rows):
            _write_rows(f, (vp[:, j], vs[:, j], rho[:, j]))


def write_model_a(path, vp, rho, d, origin=(0.0, 0.0, 0.0)):
    """vp, rho: (nx, ny, nz); d = (dx, dy, dz)."""
    nx, ny, nz = vp.shape
    with open(path, "w") as f:
        f.write(f"{nx} {ny} {nz}\n{_num(d[0])} {_num(d[1])} {_num(d[2])}\n"
                f"{_num(origin[0])} {_num(origin[1])} {_num(origin[2])}\nisotropic_acoustic_3d\n")
        # chunked so very large models do not need one giant text buffer
        v = vp.reshape(nx, -1)
        r = rho.reshape(nx, -1)
        for i in range(nx):
            _write_rows(f, (v[i], r[i]))


def write_model_a_1d(path, shape, vp, rho, d, origin=(0.0, 0.0, 0.0)):
    nx, ny, nz = shape
    assert len(vp) == nz
    with open(path, "w") as f:
        f.write(f"{nx} {ny} {nz}\n{_num(d[0])} {_num(d[1])} {_num(d[2])}\n"
                f"{_num(origin[0])} {_num(origin[1])} {_num(origin[2])}\nisotropic_acoustic_3d\n")
        _write_rows(f, (vp, rho))


def write_src(path, sources, ntemplate=1):
    """sources: list of (type, A, f, coords...) with 2 (x, z) or 3 (x, y, z) coords."""
    with open(path, "w") as f:
        f.write(f"{len(sources)}\n{ntemplate}\n")
        for s in sources:
            typ, A, fr, *xyz = s
            f.write(f"\n{typ}\n{_num(A)}\n{_num(fr)}\n{' '.join(_num(c) for c in xyz)}\n")


def write_rcv(path, records):
    """records: list of (comp, coords tuple, t0_s, dt_ms[, "Trace" | "Snapshot"]).
    A Snapshot record has no coordinates in the file (io_utils.c:1668-1672):
    its coords entry is ignored."""
    with open(path, "w") as f:
        f.write(f"{len(records)}\n")
        for comp, xyz, t0, dtms, *kind in records:
            typ = kind[0] if kind else "Trace"
            where = "" if typ.lower() == "snapshot" else " ".join(_num(c) for c in xyz) + "\n"
            f.write(f"\n{comp}\n{typ}\n{where}{_num(t0)}\n{_num(dtms)}\n")


def read_snapshot(path):
    """(x, z, value) columns of a text snapshot (write_snapshot layout)."""
    a = np.loadtxt(path, ndmin=2)
    return a[:, 0], a[:, 1], a[:, 2]


def trace_path(workdir, basename, n):
    """Path of record n (1-based) as write_trace names it (io_utils.c:1759)."""
    return os.path.join(workdir, "trc", basename, f"{basename}_{n}.trc")


def read_trc(path):
    a = np.loadtxt(path, ndmin=2)
    return a[:, 0], a[:, 1]


def read_traces(workdir, basename, nrec):
    """All .trc records -> (list of time arrays, list of value arrays); the
    records may have different sample counts."""
    ts, vs = [], []
    for n in range(1, nrec + 1):
        t, v = read_trc(trace_path(workdir, basename, n))
        ts.append(t)
        vs.append(v)
    return ts, vs


def write_model_bin(path, fields, d, origin):
    """Binary model file read by the drop-in programs in place of the ASCII
    model: "SEISMODB", uint32 version 1, ndim, nfields, 0; uint64 nx ny nz;
    float64 dx dy dz x0 y0 z0; the fields' float64 values, index
    (i*ny + j)*nz + k (host byte order).  fields: [vp, vs, rho] of shape
    (nx, nz) for e_iso, [vp, rho] of shape (nx, ny, nz) for a_iso_3d; d and
    origin have 2 or 3 entries to match."""
    arrs = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
    shape = arrs[0].shape
    ndim = len(shape)
    n3 = (shape[0], 1, shape[1]) if ndim == 2 else shape
    d3 = (d[0], 1.0, d[1]) if ndim == 2 else tuple(d)
    o3 = (origin[0], 0.0, origin[1]) if ndim == 2 else tuple(origin)
    with open(path, "wb") as f:
        f.write(b"SEISMODB")
        f.write(np.array([1, ndim, len(arrs), 0], dtype=np.uint32).tobytes())
        f.write(np.array(n3, dtype=np.uint64).tobytes())
        f.write(np.array(d3 + o3, dtype=np.float64).tobytes())
        for a in arrs:
            f.write(a.tobytes())
