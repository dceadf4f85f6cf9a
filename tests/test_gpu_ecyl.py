"""e_cyl_iso on the GPU against the FP64 oracle and the reference's traces.

Tolerances (relative L2, per record component over all of its records):
  FP64 device vs FP64 oracle        1e-12  (same operations, no contraction)
  FP32 device vs oracle / reference 1e-5   (the FP32 bound of this path)
  FP32 div and curl records         1e-4   (differences of neighbouring
        velocities: their cancellation magnifies the fields' FP32 error;
        measured 1.6e-5 to 5.4e-5 on these cases)
"""
import glob
import os

import numpy as np
import pytest

import harness as H
from golden import make_golden as G
from oracle import oracle as O
from seismod_b200 import api
from seismod_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5}
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ecyl_*.npz")))
COMPS = ("Vr", "Vz", "Vtheta", "trr", "tzz", "trz", "trtheta", "tthetatheta", "tthetaz", "div",
         "curl")


def _by_comp(p, got, ref, tol, scale=1.0):
    for comp in sorted({r[0] for r in p.receivers}):
        ks = [k for k, r in enumerate(p.receivers) if r[0] == comp]
        a = scale * np.concatenate([got[k] for k in ks])
        b = np.concatenate([ref[k] for k in ks])
        assert a.shape == b.shape, comp
        if np.abs(b).max() < 1e-300:
            assert np.abs(a).max() < 1e-300, comp
        else:
            lim = max(tol, 1e-4) if (comp in ("div", "curl") and tol >= 1e-5) else tol
            assert O.rel_l2(a, b) < lim, (comp, O.rel_l2(a, b))


CASES = [dict(n=0, src="Fz"), dict(n=1, src="Fr"), dict(n=2, src="Ftheta", dx=1.5, dz=1.0),
         dict(n=1, src="Kurkjian"), dict(n=0, src="Fz", absorb=0)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", CASES + [dict(n=3, src="Bulk")])
def test_traces_against_oracle(precision, case):
    """Mode 3 runs in FP64 only: the reference's axis update for n >= 3 grows
    without bound (about 1e18 every 40 steps at the first column here); FP64
    follows that growth bit for bit, FP32 overflows."""
    if case.get("n") == 3 and precision == "fp32":
        pytest.skip("the reference scheme is unstable at the axis for n = 3")
    p = W.ecyl_case(nx=52, nz=64, npml=7, nsteps=180, nrec=22, comps=COMPS, seed=31, **case)
    got = api.run_ecyl(p, precision)
    ref, _, _ = H.run_ecyl_oracle(p)
    _by_comp(p, got, ref, TOL[precision], scale=1e3)


@pytest.mark.parametrize("n", [0, 1, 2])
def test_fp64_fields_follow_the_oracle_bit_for_bit(n):
    """Every field after 120 steps, interior and both absorbing layers."""
    p = W.ecyl_case(nx=40, nz=48, npml=6, nsteps=120, nrec=4, n=n, src="Bulk", seed=32)
    fields = ("vr", "vt", "vz", "trr", "ttt", "tzz", "trz", "trt", "ttz")
    _, _, orc = H.run_ecyl_oracle(p, fields_at=fields)
    dev, nsteps = api.ecyl_device(p, "fp64")
    dev.run(nsteps)
    for f in fields:
        np.testing.assert_array_equal(dev.get_field(f), orc[f], err_msg=f)
    dev.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_fp32_against_reference_traces(path):
    p, kind, program, ref_t, ref_v = G.load(path)
    got = api.run_ecyl(p, "fp32")
    assert [len(a) for a in got] == [len(a) for a in ref_v]
    _by_comp(p, got, ref_v, 1e-5, scale=1e3)


def test_reset_and_rerun_give_the_same_traces():
    p = W.ecyl_case(nx=30, nz=36, npml=5, nsteps=80, nrec=6, n=1, src="Fz", seed=33)
    dev, n = api.ecyl_device(p, "fp32")
    dev.run(n)
    a = dev.traces()
    dev.reset()
    dev.run(n)
    for x, y in zip(dev.traces(), a):
        np.testing.assert_array_equal(x, y)
    dev.close()
