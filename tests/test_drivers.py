"""The drop-in programs e_iso_gpu / a_iso_3d_gpu: argument and input errors
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
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


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
