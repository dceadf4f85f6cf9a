"""a_iso_3d on the GPU against the FP64 oracle and the reference's golden
traces.  Tolerances as for e_iso: FP64 1e-10, FP32 1e-5 relative L2."""
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

TOL = {"fp64": 1e-10, "fp32": 1e-5}
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "a3d_*.npz")))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [((12, 10, 14), 2), ((20, 20, 20), 5), ((9, 17, 33), 3),
                                   # 48 x 58 x 98 padded: tiles clear of the frame, on one
                                   # face (y or z), on two, and planes inside the x frame
                                   ((40, 50, 90), 4),
                                   # abs 0: no frame, the edges alone (index 0 never updated)
                                   ((40, 50, 90), 0)])
def test_steps_from_random_state(shape, precision):
    (nx, ny, nz), npml = shape
    rng = np.random.default_rng(nx * ny + nz)
    vp = 1500 + 3000 * rng.random((nx, ny, nz))
    rho = 1800 + 600 * rng.random((nx, ny, nz))
    p = W.A3DProblem(vp, rho, (4.0, 5.0, 3.0), npml, 0.2, 1.0, [("Bulk", 1.0, 30.0, 0, 0, 0)],
                     [], Rc=1e-3, kappa_max=2.0, alpha_max=1)
    vmax = vp.max()
    p.dt_ms = 0.5 / (vmax * np.sqrt(1 / 16 + 1 / 25 + 1 / 9)) * 1e3
    s = H.a3d_setup(p)
    orc = O.A3D(s["vpp"], s["rhop"], *p.d, s["dt"], s["coef"])
    dev = api.A3DDevice(s["vpp"], s["rhop"], npml, p.d, s["dt"], s["coef"], precision)
    shp = s["vpp"].shape
    for f, sc in (("p", 1e5), ("vx", 1e-2), ("vy", 1e-2), ("vz", 1e-2)):
        a = sc * rng.standard_normal(shp)
        orc.set(f, a)
        dev.set_field(f, a)
    for _ in range(4):
        orc.velocity()
        orc.pressure()
    dev.run(4)
    for f in ("p", "vx", "vy", "vz"):
        e = O.rel_l2(dev.get_field(f), orc.get(f))
        assert e < TOL[precision], (f, e)
    dev.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden_traces(path, precision):
    p, kind, program, ref_t, ref_v = G.load(path)
    got = [1e3 * t for t in api.run_a3d(p, precision)]
    assert [len(a) for a in got] == [len(a) for a in ref_v]
    assert H.rel_l2(got, ref_v) < max(TOL[precision], 2e-6)
    if precision == "fp64":
        orc, _, _ = H.run_a3d_oracle(p)
        assert H.rel_l2(got, orc) < TOL["fp64"]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cfg1_family_against_oracle(precision):
    # the cfg1 model family at 48^3 (+2x8 CPML), 300 steps, 16x16 surface receivers
    p = W.cfg1(n=48, npml=8, nsteps=300, seed=21, rec_stride=3, nrec_side=16)
    got = [1e3 * t for t in api.run_a3d(p, precision)]
    orc, _, _ = H.run_a3d_oracle(p)
    assert H.rel_l2(got, orc) < TOL[precision]


def test_pressure_receivers_and_reset():
    p = W.cfg1(n=24, npml=4, nsteps=100, seed=5, rec_stride=6, nrec_side=3)
    p.receivers = p.receivers + [("P", 60.0, 60.0, 60.0, 0.0, p.dt_ms)]
    dev, n = api.a3d_device(p, "fp64")
    dev.run(n)
    a = dev.traces()
    orc, _, _ = H.run_a3d_oracle(p)
    assert H.rel_l2([1e3 * t for t in a], orc) < TOL["fp64"]
    dev.reset()
    dev.run(n)
    b = dev.traces()
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    dev.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_every_launch_configuration_gives_identical_results(precision):
    # 120^3 + 2x6: tiles with k0 = 32, 64 lie inside the frame, so both the
    # interior fast path and the general path run
    p = W.cfg1(n=120, npml=6, nsteps=90, seed=8, rec_stride=10, nrec_side=12)
    dev, n = api.a3d_device(p, precision)
    _, ncfg = dev.get_config()
    base = None
    for c in range(ncfg):
        dev.reset()
        try:
            dev.set_config(c)
        except Exception:
            continue   # does not fit this precision's shared-memory budget
        dev.run(n)
        tr = dev.traces_array()
        f = dev.get_field("p")
        if base is None:
            base = (tr, f)
        else:
            np.testing.assert_array_equal(tr, base[0])
            np.testing.assert_array_equal(f, base[1])
    dev.close()
    orc, _, fo = H.run_a3d_oracle(p, fields_at=["p"])
    assert H.rel_l2([1e3 * t for t in base[0]], orc) < TOL[precision]
    assert O.rel_l2(base[1], fo["p"]) < TOL[precision]


# 16-bit storage (per-field power-of-two scales, FP32 arithmetic): the bound
# is the one this storage meets on these short runs, not the FP32 bound
TOL16 = {"fp16": 2.5e-2, "bf16": 1.5e-1}


@pytest.mark.parametrize("precision", ["fp16", "bf16"])
def test_16bit_storage_stays_in_range_and_close_to_fp64(precision):
    p = W.cfg1(n=48, npml=8, nsteps=300, seed=21, rec_stride=3, nrec_side=16)
    got = api.run_a3d(p, precision)
    assert all(np.isfinite(t).all() for t in got)
    ref = api.run_a3d(p, "fp64")
    err = H.rel_l2(got, ref)
    assert err < TOL16[precision], err
    # the scale is a power of two: an FP16 run reproduces itself exactly
    again = api.run_a3d(p, precision)
    for a, b in zip(got, again):
        np.testing.assert_array_equal(a, b)


# ---------------------------------------------------------------------------
# Block floating point (SM_BFP16): 16-bit mantissas sharing one exponent per
# 4 consecutive y rows of a z column, FP32 arithmetic.  The oracle's
# storage-rounding mode applies the same rounding to its FP64 state, so it
# predicts what the storage alone costs.  Bounds: each stored value is
# rounded to 2^-16 of its block's largest magnitude once per step, so 4 steps
# from a random state stay within 1e-4 of the FP64 oracle; the device and
# the rounding oracle differ only where FP32 and FP64 arithmetic fall on
# opposite sides of a rounding boundary (2e-5).  Traces of whole shots:
# the 1e-3 gate against FP64.
# ---------------------------------------------------------------------------
BFP_BLOCK = 4


@pytest.mark.parametrize("shape", [((12, 10, 14), 2), ((9, 17, 33), 3), ((40, 50, 90), 4),
                                   ((40, 50, 90), 0)])
def test_bfp16_steps_from_random_state(shape):
    (nx, ny, nz), npml = shape
    rng = np.random.default_rng(nx * ny + nz + 1)
    vp = 1500 + 3000 * rng.random((nx, ny, nz))
    rho = 1800 + 600 * rng.random((nx, ny, nz))
    p = W.A3DProblem(vp, rho, (4.0, 5.0, 3.0), npml, 0.2, 1.0, [("Bulk", 1.0, 30.0, 0, 0, 0)],
                     [], Rc=1e-3, kappa_max=2.0, alpha_max=1)
    p.dt_ms = 0.5 / (vp.max() * np.sqrt(1 / 16 + 1 / 25 + 1 / 9)) * 1e3
    s = H.a3d_setup(p)
    plain = O.A3D(s["vpp"], s["rhop"], *p.d, s["dt"], s["coef"])
    rounded = O.A3D(s["vpp"], s["rhop"], *p.d, s["dt"], s["coef"])
    rounded.set_bfp(BFP_BLOCK, "y")
    dev = api.A3DDevice(s["vpp"], s["rhop"], npml, p.d, s["dt"], s["coef"], "bfp16")
    shp = s["vpp"].shape
    for f, sc in (("p", 1e5), ("vx", 1e-2), ("vy", 1e-2), ("vz", 1e-2)):
        dev.set_field(f, sc * rng.standard_normal(shp))
        a = dev.get_field(f)           # the stored (rounded) start state
        plain.set(f, a)
        rounded.set(f, a)
    for _ in range(4):
        for o in (plain, rounded):
            o.velocity()
            o.pressure()
    dev.run(4)
    for f in ("p", "vx", "vy", "vz"):
        got = dev.get_field(f)
        assert O.rel_l2(got, rounded.get(f)) < 2e-5, (f, O.rel_l2(got, rounded.get(f)))
        assert O.rel_l2(got, plain.get(f)) < 1e-4, (f, O.rel_l2(got, plain.get(f)))
    dev.close()


def test_bfp16_every_launch_configuration_gives_identical_results():
    p = W.cfg1(n=120, npml=6, nsteps=90, seed=8, rec_stride=10, nrec_side=12)
    dev, n = api.a3d_device(p, "bfp16")
    _, ncfg = dev.get_config()
    base = None
    for c in range(ncfg):
        dev.reset()
        try:
            dev.set_config(c)
        except Exception:
            continue
        dev.run(n)
        tr = dev.traces_array()
        f = dev.get_field("p")
        if base is None:
            base = (tr, f)
        else:
            np.testing.assert_array_equal(tr, base[0])
            np.testing.assert_array_equal(f, base[1])
    dev.close()


def test_bfp16_shot_within_gate_and_as_the_rounding_oracle_predicts():
    # the cfg1 model family at 48^3 (+2x8 CPML), 300 steps, 16x16 surface
    # receivers, Vz and a pressure record
    p = W.cfg1(n=48, npml=8, nsteps=300, seed=21, rec_stride=3, nrec_side=16)
    p.receivers = p.receivers + [("P", 60.0, 60.0, 60.0, 0.0, p.dt_ms)]
    got = api.run_a3d(p, "bfp16")
    assert all(np.isfinite(t).all() for t in got)
    ref = api.run_a3d(p, "fp64")
    err = H.rel_l2(got, ref)
    assert err < 1e-3, err
    plain, _, _ = H.run_a3d_oracle(p)
    pred, _, _ = H.run_a3d_oracle(p, bfp_block=BFP_BLOCK, bfp_axis="y")
    predicted = H.rel_l2(pred, plain)
    assert 0.5 * predicted < err < 2.0 * predicted, (err, predicted)
    # deterministic: a second run reproduces the first bit for bit
    again = api.run_a3d(p, "bfp16")
    for a, b in zip(got, again):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp32", "fp64", "bfp16", "fp16"])
def test_unpadded_create_equals_the_padded_one(precision):
    """sm_a3d_create_unpadded pads the model as it stages the materials:
    the same handle, bit for bit, as sm_a3d_create on the padded model
    (traces and the whole state), on a grid whose padding is uneven in
    every axis."""
    rng = np.random.default_rng(77)
    shape = (23, 31, 45)
    vp = 1500 + 3000 * rng.random(shape)
    rho = 1800 + 600 * rng.random(shape)
    d = (4.0, 5.0, 3.0)
    dt_ms = 0.5 / (vp.max() * np.sqrt(sum(1 / h ** 2 for h in d))) * 1e3
    rec = [(c, float(rng.integers(0, shape[0])) * d[0], float(rng.integers(0, shape[1])) * d[1],
            float(rng.integers(0, shape[2])) * d[2], 0.0, dt_ms)
           for c in ("Vx", "Vy", "Vz", "P")]
    p = W.A3DProblem(vp, rho, d, 6, dt_ms, W.steps_duration(60, dt_ms),
                     [("Bulk", 1.0, 40.0, 11 * d[0], 7 * d[1], 20 * d[2])], rec,
                     Rc=1e-3, kappa_max=2.0, alpha_max=1)
    a, n = api.a3d_device(p, precision, pad_on_host=True)
    b, _ = api.a3d_device(p, precision)
    assert a.shape == b.shape
    for d in (a, b):
        d.run(n)
        d.sync()
    for x, y in zip(a.traces(), b.traces()):
        np.testing.assert_array_equal(x, y)
    for f in ("p", "vx", "vy", "vz"):
        np.testing.assert_array_equal(a.get_field(f), b.get_field(f))
    a.close()
    b.close()
