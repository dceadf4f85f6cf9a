"""The drop-in programs e_iso_gpu / a_iso_3d_gpu / e_cyl_iso_gpu: argument and input errors
come back as a non-zero exit with the reference's message (CPU: these paths
return before the device is used); on the GPU the trace files they write
match the reference's (golden fixtures) in format and values."""
import glob
import os
import subprocess

import numpy as np
import pytest

import harness as H
from golden import make_golden as G
from seismod_b200 import formats as F
from seismod_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "seismod_b200", "bin")
GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith("segy_"))


def run(prog, args, cwd):
    return subprocess.run([os.path.join(BIN, prog)] + args, cwd=cwd, capture_output=True,
                          text=True, timeout=600)


def test_usage_and_missing_files(tmp_path):
    r = run("e_iso_gpu", [], tmp_path)
    assert r.returncode != 0 and "usage" in r.stderr
    r = run("a_iso_3d_gpu", ["-p", "nope.par"], tmp_path)
    assert r.returncode != 0 and "cannot open parameter file" in r.stderr
    r = run("e_iso_gpu", ["-P", "fp8", "-p", "x.par"], tmp_path)
    assert r.returncode != 0 and "-P takes" in r.stderr


def test_parameter_file_without_comma_is_an_error(tmp_path):
    (tmp_path / "run.par").write_text("model.dat # model\n")
    r = run("e_iso_gpu", ["-p", "run.par"], tmp_path)
    assert r.returncode != 0 and "keyword" in r.stderr


def test_cfl_violation_is_refused_like_the_reference(tmp_path):
    p = W.cfg0(nx=30, nz=30, npml=5, nsteps=10, nrec=2)
    p.dt_ms *= 2.5   # beyond h / (sqrt(2) vpmax)
    par = p.write(str(tmp_path), basename="cfl")
    r = run("e_iso_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode != 0 and "Time step too large" in r.stderr
    q = W.cfg1(n=12, npml=3, nsteps=5, seed=1, rec_stride=6, nrec_side=2)
    q.dt_ms *= 2.5
    par = q.write(str(tmp_path / "a3d"))
    r = run("a_iso_3d_gpu", ["-p", "run.par"], tmp_path / "a3d")
    assert r.returncode != 0 and "Time step too large" in r.stderr


def test_unequal_spacing_is_refused(tmp_path):
    (tmp_path / "model.dat").write_text("4 4\n1.0 2.0\n0 0\nisotropic_elastic\n" +
                                        "3000 1700 2000\n" * 16)
    (tmp_path / "run.par").write_text("model.dat # model, m\nsrc.dat # source, s\n"
                                      "rcv.dat # output, o\n1 # abs, a\n")
    r = run("e_iso_gpu", ["-p", "run.par"], tmp_path)
    assert r.returncode != 0 and "equal in X and Z" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_drop_in_programs_write_the_reference_traces(path, tmp_path):
    p, kind, program, ref_t, ref_v = G.load(path)
    if kind == "ecyl":
        _check_ecyl_drop_in(p, ref_t, ref_v, tmp_path, "fp32")
        return
    if kind == "eiso":
        par = p.write(str(tmp_path), shot=0, basename=p.name)
        r = run("e_iso_gpu", ["-p", os.path.basename(par)], tmp_path)
    else:
        par = p.write(str(tmp_path), profile_1d=program.endswith("_1d"))
        r = run("a_iso_3d_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode == 0, r.stderr
    t, v = F.read_traces(str(tmp_path), p.name, len(p.receivers))
    assert [len(a) for a in v] == [len(a) for a in ref_v]
    for a, b in zip(t, ref_t):
        np.testing.assert_allclose(a, b, rtol=1e-6)
    assert H.rel_l2(v, ref_v) < 1e-5
    # the same "%le    %le" text layout
    line = open(F.trace_path(str(tmp_path), p.name, 1)).readline()
    assert len(line.split("    ")) == 2 and "e" in line.split()[0]


SEGY = os.path.join(os.path.dirname(__file__), "golden", "segy_a3d.npz")


def _segy_traces(b, ns_key=114):
    """(headers, samples) of each trace of a SEG-Y byte string laid out as
    save_segy writes it (host byte order)."""
    out, pos = [], 3600
    while pos < len(b):
        hdr = b[pos:pos + 240]
        ns = int(np.frombuffer(hdr[ns_key:ns_key + 2].tobytes(), dtype=np.int16)[0])
        out.append((hdr, np.frombuffer(b[pos + 240:pos + 240 + 4 * ns].tobytes(), dtype=np.float32)))
        pos += 240 + 4 * ns
    return out


@pytest.mark.gpu
def test_segy_output_matches_the_reference_layout(tmp_path):
    """segy 1: same file, headers field for field (clock fields and sample
    counts aside), the reference's samples.  Sample i is the value at
    i * dt; the reference keeps one sample too few (its last recorded one is
    written past its array) and leaves sample 0 (t = 0) uninitialised, so
    samples 1 .. n-1 are compared and ours holds one more, and zero at t = 0."""
    ref = np.load(SEGY)["sgy"]
    p = G.segy_case()
    par = p.write(str(tmp_path), segy=1, shotpoint=7)
    r = run("a_iso_3d_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(os.path.join(str(tmp_path), "segy", f"{p.name}.sgy"), dtype=np.uint8)
    # textual and binary file headers: equal except the sample counts (bytes 3221-3224)
    keep = np.ones(3600, bool)
    keep[3220:3224] = False
    np.testing.assert_array_equal(got[:3600][keep], ref[:3600][keep])
    rt, gt = _segy_traces(ref), _segy_traces(got)
    assert len(rt) == len(gt) == len(p.receivers)
    hkeep = np.ones(240, bool)
    hkeep[114:116] = False      # samples in this trace
    hkeep[156:166] = False      # year, day, hour, minute, second of writing
    a, b = [], []
    for (rh, rs), (gh, gs) in zip(rt, gt):
        np.testing.assert_array_equal(gh[hkeep], rh[hkeep])
        assert len(gs) == len(rs) + 1 and gs[0] == 0.0
        a.append(gs[1:len(rs)].astype(np.float64))
        b.append(rs[1:].astype(np.float64))
    assert H.rel_l2(a, b) < 1e-5
    # the samples are the raw velocities the trace files would hold (x 1e-3)
    r = run("a_iso_3d_gpu", ["-p", os.path.basename(p.write(str(tmp_path / "trc")))], tmp_path / "trc")
    assert r.returncode == 0, r.stderr
    t, v = F.read_traces(str(tmp_path / "trc"), p.name, len(p.receivers))
    assert H.rel_l2([1e-3 * x for x in v], [g[1][1:].astype(np.float64) for g in gt]) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["eiso_square", "a3d_cube"])
def test_binary_model_gives_the_same_traces_as_ascii(name, tmp_path):
    """A model given as a binary file (no text parsing) runs exactly as the
    same values in the reference's ASCII format: identical trace files."""
    p, kind, program, _, _ = G.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))
    out = {}
    for fmt in ("ascii", "bin"):
        d = tmp_path / fmt
        if kind == "eiso":
            par = p.write(str(d), shot=0, basename=p.name)
            if fmt == "bin":
                F.write_model_bin(os.path.join(str(d), "model.dat"), [p.vp, p.vs, p.rho],
                                  (p.h, p.h), (p.x0, p.z0))
            r = run("e_iso_gpu", ["-p", os.path.basename(par)], d)
        else:
            par = p.write(str(d))
            if fmt == "bin":
                F.write_model_bin(os.path.join(str(d), "model.dat"), [p.vp, p.rho], p.d, p.origin)
            r = run("a_iso_3d_gpu", ["-p", os.path.basename(par)], d)
        assert r.returncode == 0, r.stderr
        out[fmt] = [open(F.trace_path(str(d), p.name, n + 1)).read()
                    for n in range(len(p.receivers))]
    assert out["ascii"] == out["bin"]


def test_binary_model_header_errors_are_reported(tmp_path):
    """A truncated binary model is an input error, not a crash (CPU path)."""
    p = W.cfg0(nx=20, nz=20, npml=3, nsteps=10, nrec=2)
    par = p.write(str(tmp_path), shot=0, basename="b")
    with open(os.path.join(str(tmp_path), "model.dat"), "wb") as f:
        f.write(b"SEISMODB" + bytes(10))
    r = run("e_iso_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode != 0 and "binary model" in r.stderr


@pytest.mark.gpu
def test_pressure_traces_from_the_drop_in_program(tmp_path):
    """a_iso_3d accepts P records but its loop leaves them undefined
    (a_iso_3d.c:703-715); here they are the pressure at the node, written like
    the velocity traces (1e3 * value), and equal what the library records."""
    from seismod_b200 import api
    p = W.cfg1(n=24, npml=5, nsteps=140, seed=17)
    p.receivers = [("P", 40.0, 45.0, 30.0, 0.0, p.dt_ms), ("Vz", 40.0, 45.0, 30.0, 0.0, p.dt_ms),
                   ("P", 10.0, 70.0, 80.0, 0.0, 2 * p.dt_ms)]
    par = p.write(str(tmp_path))
    r = run("a_iso_3d_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode == 0, r.stderr
    t, v = F.read_traces(str(tmp_path), p.name, len(p.receivers))
    ref = api.run_a3d(p, "fp32")
    assert [len(a) for a in v] == [len(a) for a in ref]
    assert H.rel_l2(v, [1e3 * a for a in ref]) < 1e-6
    assert np.abs(v[0]).max() > 0


def _snapshot_file(d, base, n):
    files = glob.glob(os.path.join(str(d), "ssh", base, f"{base}_{n}_*.ssh"))
    assert len(files) == 1, files
    return files[0]


@pytest.mark.gpu
@pytest.mark.parametrize("strips", [0, 1])
def test_eiso_snapshots_in_the_reference_text_format(strips, tmp_path):
    """Snapshot records are written as write_snapshot writes them (netCDF is
    not available): one file per snapshot time, x, z and 1e3 * value per
    node, the interior or, with plstr 1, the whole padded grid."""
    from seismod_b200 import api
    p = W.cfg0(nx=48, nz=40, npml=6, nsteps=120, nrec=2)
    k = 60
    par = p.write(str(tmp_path), shot=0, basename="snap", plstr=strips)
    recs = [(c, (x, z), t0, r) for (c, x, z, t0, r) in p.receivers]
    recs.append(("Vz", (0.0, 0.0), k * p.dt, 1e6, "Snapshot"))
    F.write_rcv(os.path.join(str(tmp_path), "rcv.dat"), recs)
    r = run("e_iso_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode == 0, r.stderr
    x, z, val = F.read_snapshot(_snapshot_file(tmp_path, "snap", len(recs)))
    dev, _ = api.eiso_device(p, "fp32")
    dev.run(k)
    vz = dev.get_field("vz")
    dev.close()
    np_ = p.npml
    ref = vz if strips else vz[np_:np_ + p.nx, np_:np_ + p.nz]
    assert val.size == ref.size
    np.testing.assert_allclose(val.reshape(ref.shape), 1e3 * ref, rtol=1e-5,
                               atol=1e-5 * np.abs(1e3 * ref).max())
    assert x[0] == (-np_ * p.h if strips else 0.0)
    # the trace records are unchanged by the stops for the snapshot
    t, v = F.read_traces(str(tmp_path), "snap", len(p.receivers))
    assert H.rel_l2(v, [1e3 * a for a in api.run_eiso(p, "fp32")[0]]) < 1e-6


@pytest.mark.gpu
def test_a3d_snapshot_plane(tmp_path):
    from seismod_b200 import api
    p = W.cfg1(n=20, npml=4, nsteps=90, seed=19, rec_stride=10)
    k = 40
    par = p.write(str(tmp_path))
    recs = [(c, (x, y, z), t0, r) for (c, x, y, z, t0, r) in p.receivers]
    recs.append(("Vz", (0.0, 0.0, 0.0), k * p.dt, 1e6, "Snapshot"))
    F.write_rcv(os.path.join(str(tmp_path), "rcv.dat"), recs)
    r = run("a_iso_3d_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode == 0, r.stderr
    _, _, val = F.read_snapshot(_snapshot_file(tmp_path, p.name, len(recs)))
    dev, _ = api.a3d_device(p, "fp32")
    dev.run(k)
    vol = dev.get_field("vz")
    dev.close()
    iy = int((p.sources[0][4] - p.origin[1]) / p.d[1])   # a_iso_3d.c: plane index as it takes it
    n = p.npml
    ref = vol[n:-n, iy, n:-n]
    np.testing.assert_allclose(val.reshape(ref.shape), 1e3 * ref, rtol=1e-5,
                               atol=1e-5 * np.abs(1e3 * ref).max())


def _check_ecyl_drop_in(p, ref_t, ref_v, tmp_path, precision):
    """e_cyl_iso_gpu against the reference's traces, per record component:
    1e-5 in FP32 (1e-4 for div and curl, differences of neighbouring
    velocities), text precision (2e-6) in FP64."""
    par = p.write(str(tmp_path))
    r = run("e_cyl_iso_gpu", ["-p", os.path.basename(par), "-P", precision], tmp_path)
    assert r.returncode == 0, r.stderr
    t, v = F.read_traces(str(tmp_path), p.name, len(p.receivers))
    assert [len(a) for a in v] == [len(a) for a in ref_v]
    for a, b in zip(t, ref_t):
        np.testing.assert_allclose(a, b, rtol=1e-6)
    for comp in sorted({q[0] for q in p.receivers}):
        ks = [k for k, q in enumerate(p.receivers) if q[0] == comp]
        a = np.concatenate([v[k] for k in ks])
        b = np.concatenate([ref_v[k] for k in ks])
        if np.abs(b).max() < 1e-300:
            assert np.abs(a).max() < 1e-300, comp
            continue
        tol = 2e-6 if precision == "fp64" else (1e-4 if comp in ("div", "curl") else 1e-5)
        assert H.rel_l2([a], [b]) < tol, (comp, H.rel_l2([a], [b]))


ECYL_GOLDEN = [q for q in GOLDEN if os.path.basename(q).startswith("ecyl_")]


@pytest.mark.gpu
@pytest.mark.parametrize("path", ECYL_GOLDEN, ids=[os.path.basename(q)[:-4] for q in ECYL_GOLDEN])
def test_ecyl_drop_in_fp64_matches_the_reference_to_text_precision(path, tmp_path):
    p, kind, program, ref_t, ref_v = G.load(path)
    _check_ecyl_drop_in(p, ref_t, ref_v, tmp_path, "fp64")


def test_ecyl_drop_in_refuses_what_it_cannot_run(tmp_path):
    p = W.ecyl_case(nx=20, nz=24, npml=4, nsteps=10, nrec=2)
    par = p.write(str(tmp_path))
    F.write_src(os.path.join(str(tmp_path), "src.dat"), p.sources, ntemplate=9)
    r = run("e_cyl_iso_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode != 0 and "1-point sources" in r.stderr
    (tmp_path / "model.dat").write_text("4 4\n1.0 1.0\n0 0\nisotropic_elastic\n" +
                                        "3000 1700 2000\n" * 16)
    r = run("e_cyl_iso_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode != 0 and "not isotropic_elastic_cyl" in r.stderr
    q = W.ecyl_case(nx=20, nz=24, npml=4, nsteps=10, nrec=2)
    q.dt_ms *= 3.0
    par = q.write(str(tmp_path / "cfl"))
    r = run("e_cyl_iso_gpu", ["-p", "run.par"], tmp_path / "cfl")
    assert r.returncode != 0 and "Time step too large" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("strips", [0, 1])
def test_ecyl_snapshots(strips, tmp_path):
    """e_cyl_iso_gpu writes snapshot records as text snapshots on the
    cylindrical grid (radii from the axis, no columns before it): a field
    (Vz) and a derived one (div), against the device state after the same
    number of steps."""
    from seismod_b200 import api
    p = W.ecyl_case(nx=36, nz=44, npml=6, nsteps=90, nrec=2, n=1, src="Fz")
    k = 50
    par = p.write(str(tmp_path), plstr=strips)
    recs = [(c, (x, z), t0, r) for (c, x, z, t0, r) in p.receivers]
    recs.append(("Vz", (0.0, 0.0), k * p.dt, 1e6, "Snapshot"))
    recs.append(("div", (0.0, 0.0), k * p.dt, 1e6, "Snapshot"))
    F.write_rcv(os.path.join(str(tmp_path), "rcv.dat"), recs)
    r = run("e_cyl_iso_gpu", ["-p", os.path.basename(par)], tmp_path)
    assert r.returncode == 0, r.stderr
    dev, _ = api.ecyl_device(p, "fp32")
    dev.run(k)
    vr, vt, vz = dev.get_field("vr"), dev.get_field("vt"), dev.get_field("vz")
    dev.close()
    n, np_ = p.n, p.np_used
    nx2, nz2 = vz.shape
    div = np.zeros_like(vz)
    i = np.arange(nx2 - 1)[:, None].astype(float)
    div[:-1, :-1] = (((i + 1) * vr[1:, :-1] - i * vr[:-1, :-1]) / (i + 0.5) +
                     n * vt[:-1, :-1] / ((i + 0.5) * p.dx) + (vz[:-1, 1:] - vz[:-1, :-1]) / p.dz)
    for rec_no, ref in ((len(recs) - 1, vz), (len(recs), div)):
        x, z, val = F.read_snapshot(_snapshot_file(tmp_path, p.name, rec_no))
        want = ref if strips else ref[:p.nx, np_:np_ + p.nz]
        assert val.size == want.size
        np.testing.assert_allclose(val.reshape(want.shape), 1e3 * want, rtol=1e-5,
                                   atol=1e-5 * np.abs(1e3 * want).max())
        assert x[0] == 0.0   # the axis: no absorbing columns before r = 0
        assert z[0] == (-np_ * p.dz if strips else 0.0)
