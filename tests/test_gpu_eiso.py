"""e_iso on the GPU against the FP64 oracle and the reference's golden traces.

Tolerances (relative L2 over all compared values):
  FP64 device vs FP64 oracle      1e-10  (same arithmetic up to operation order)
  FP32 device vs oracle/reference 1e-5   (the FP32 bound stated for this path)
"""
import glob
import math
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
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "eiso_*.npz")))
FIELDS = ("vx", "vz", "txx", "tzz", "txz")


def _pair(nx, nz, P, seed, precision):
    rng = np.random.default_rng(seed)
    vp = 3000 + 1000 * rng.random((nx, nz))
    vs = vp / (1.6 + 0.3 * rng.random((nx, nz)))
    rho = 2000 + 400 * rng.random((nx, nz))
    la, mu, l2m, b, bm, vpmax = O.eiso_materials(vp, vs, rho)
    h = 1.0
    dt = 0.5 * h / (math.sqrt(2) * vpmax)
    d, dh, dH = O.eiso_profiles(P, h, vp)
    orc = O.EIso(nx, nz, P, h, dt, la, mu, l2m, b, bm, d, dh, dH)
    dev = api.EIsoDevice(nx, nz, P, h, dt, la, mu, l2m, b, bm, d, dh, dH, precision)
    NX, NZ = nx + 2 * P, nz + 2 * P
    inter = np.zeros((NX, NZ), bool)
    inter[P:P + nx, P:P + nz] = True
    for f in FIELDS:
        scale = 1e-3 if f.startswith("v") else 1e4
        tot, xp, zp = (scale * rng.standard_normal((NX, NZ)) for _ in range(3))
        xp[inter] = 0
        zp[inter] = 0
        for tgt in (orc, dev):
            if tgt is orc:
                orc.set(f, "x", xp)
                orc.set(f, "z", zp)
                orc.set(f, "total", np.where(inter, tot, 0))
            else:
                dev.set_field(f, xp, part="x")
                dev.set_field(f, zp, part="z")
                dev.set_field(f, np.where(inter, tot, 0), part="total")
    return orc, dev


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(13, 9, 3), (9, 14, 4), (33, 40, 8), (8, 8, 1), (40, 12, 2)])
def test_steps_from_random_state(shape, precision):
    nx, nz, P = shape
    orc, dev = _pair(nx, nz, P, sum(shape), precision)
    for _ in range(4):
        orc.velocity()
        orc.stress()
    dev.run(4)
    for f in FIELDS:
        for part in ("total", "x", "z"):
            a, b = dev.get_field(f, part=part), orc.get(f, part)
            assert O.rel_l2(a, b) < TOL[precision], (f, part, O.rel_l2(a, b))
    dev.close()


def _dev_traces_mm(p, precision):
    return [1e3 * t for t in api.run_eiso(p, precision, shots=[0])[0]]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden_traces(path, precision):
    p, kind, program, ref_t, ref_v = G.load(path)
    got = _dev_traces_mm(p, precision)
    assert [len(a) for a in got] == [len(a) for a in ref_v]
    # reference values carry 7 printed digits
    assert H.rel_l2(got, ref_v) < max(TOL[precision], 2e-6)
    if precision == "fp64":
        orc, _, _ = H.run_eiso_oracle(p)
        assert H.rel_l2(got, orc) < TOL["fp64"]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cfg0_full_size_against_oracle(precision):
    p = W.cfg0()
    got = api.run_eiso(p, precision)[0]
    orc, _, _ = H.run_eiso_oracle(p)
    assert [len(a) for a in got] == [len(a) for a in orc]
    assert H.rel_l2([1e3 * g for g in got], orc) < TOL[precision]


def _state_after(nx, nz, P, precision, steps, config=None):
    orc, dev = _pair(nx, nz, P, 7, precision)
    if config is not None:
        dev.set_config(config)
    dev.run(steps)
    got = {(f, part): dev.get_field(f, part=part) for f in FIELDS for part in ("total", "x", "z")}
    nconf = dev.get_config()[1]
    dev.close()
    return orc, got, nconf


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_every_launch_config_gives_identical_results(precision):
    """The step kernel's variants (tiles, slabs with materials from L2 or in
    the TMA box, every shape) must not show in the results: halo cells are
    recomputed bitwise by neighbours."""
    nx, nz, P = 70, 95, 5       # NZ = 105: ragged against every tile width
    orc, ref, nconf = _state_after(nx, nz, P, precision, 6)
    for _ in range(6):
        orc.velocity()
        orc.stress()
    for (f, part), a in ref.items():
        assert O.rel_l2(a, orc.get(f, part)) < TOL[precision], (f, part)
    for config in range(nconf):
        _, got, _ = _state_after(nx, nz, P, precision, 6, config=config)
        for k, a in got.items():
            np.testing.assert_array_equal(a, ref[k], err_msg=f"config {config} {k}")


def test_every_launch_config_batched_shots_identical():
    """Kernels that take several shots per CTA (and every other variant)
    must give each shot of a batch the same bits, including a last group
    with fewer shots than the CTA holds."""
    p = W.cfg2(nx=150, nz=130, npml=9, nsteps=90, nshots=5, nrec=12)
    dev, n = api.eiso_device(p, "fp32")
    nconf = dev.get_config()[1]
    dev.run(n)
    ref = [dev.traces(s) for s in range(5)]
    for config in range(nconf):
        dev.reset()
        dev.set_config(config)
        dev.run(n)
        for s in range(5):
            for x, y in zip(dev.traces(s), ref[s]):
                np.testing.assert_array_equal(x, y, err_msg=f"config {config} shot {s}")
    dev.close()


def test_every_launch_config_16bit_storage_identical():
    """16-bit storage: every launch configuration gives the same bits,
    through the power-of-two rescales (every 16 steps) and the source."""
    p = W.cfg2(nx=150, nz=130, npml=9, nsteps=90, nshots=3, nrec=12)
    dev, n = api.eiso_device(p, "fp16")
    nconf = dev.get_config()[1]
    dev.run(n)
    ref = [dev.traces(s) for s in range(3)]
    for config in range(nconf):
        dev.reset()
        dev.set_config(config)
        dev.run(n)
        for s in range(3):
            for x, y in zip(dev.traces(s), ref[s]):
                np.testing.assert_array_equal(x, y, err_msg=f"config {config} shot {s}")
    dev.close()


def test_batched_shots_equal_single_shots():
    p = W.cfg2(nx=120, nz=80, npml=10, nsteps=250, nshots=5, nrec=12)
    batch = api.run_eiso(p, "fp32")
    for s in (0, 2, 4):
        alone = api.run_eiso(p, "fp32", shots=[s])[0]
        for a, b in zip(batch[s], alone):
            np.testing.assert_array_equal(a, b)
    # and each shot matches the oracle
    for s in (1, 3):
        q = W.cfg2(nx=120, nz=80, npml=10, nsteps=250, nshots=5, nrec=12)
        q.shots = [q.shots[s]]
        orc, _, _ = H.run_eiso_oracle(q)
        assert H.rel_l2([1e3 * g for g in batch[s]], orc) < TOL["fp32"]


def test_every_source_type_and_edge_positions():
    p = W.cfg0(nx=48, nz=56, npml=5, nsteps=220, nrec=4)
    p.shots = [[("Sx", 1.0, 80.0, 0.0, 0.0), ("Sz", 2.0, 80.0, 47.0, 55.0),
                ("Sxz", 0.7, 80.0, 10.0, 55.0), ("Bulk", 1.3, 80.0, 47.0, 0.0)]]
    p.receivers = [("Vx", 0.0, 0.0, 0.0, p.dt_ms), ("Vz", 47.0, 55.0, 0.0, p.dt_ms),
                   ("txx", 20.0, 20.0, 0.0, p.dt_ms), ("Vx", 47.0, 0.0, 0.0, 2 * p.dt_ms)]
    got = api.run_eiso(p, "fp64")[0]
    orc, _, _ = H.run_eiso_oracle(p)
    assert H.rel_l2([1e3 * g for g in got], orc) < TOL["fp64"]
    got32 = api.run_eiso(p, "fp32")[0]
    assert H.rel_l2([1e3 * g for g in got32], orc) < TOL["fp32"]


def test_reset_reproduces_run_and_step_count():
    p = W.cfg0(nx=40, nz=40, npml=6, nsteps=120, nrec=3)
    dev, n = api.eiso_device(p, "fp32")
    dev.run(n)
    a = dev.traces(0)
    dev.reset()
    dev.run(n // 2)
    dev.run(n - n // 2)
    b = dev.traces(0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    dev.close()


TOL16 = {"fp16": 2.5e-2, "bf16": 1.5e-1}


@pytest.mark.parametrize("precision", ["fp16", "bf16"])
def test_16bit_storage_stays_in_range_and_close_to_fp64(precision):
    p = W.cfg0(nx=120, nz=100, npml=10, nsteps=400, nrec=8)
    got = api.run_eiso(p, precision)[0]
    assert all(np.isfinite(t).all() for t in got)
    ref = api.run_eiso(p, "fp64")[0]
    err = H.rel_l2(got, ref)
    assert err < TOL16[precision], err


# ---------------------------------------------------------------------------
# Block floating point (SM_BFP16): the five wavefields as 16-bit mantissas
# sharing one exponent per 4 consecutive x rows of a z column, split parts
# FP32, FP32 arithmetic.  The oracle's storage-rounding mode applies the same
# rounding to its FP64 state.  Bounds as for a_iso_3d: 4 steps from a random
# state within 1e-4 of the plain FP64 oracle and 2e-5 of the rounding oracle
# (the device's FP32 arithmetic lands on the other side of a rounding
# boundary now and then); whole shots within the 1e-3 gate.
# ---------------------------------------------------------------------------
BFP_BLOCK = 4


def _bfp_pair(nx, nz, P, seed):
    rng = np.random.default_rng(seed)
    vp = 3000 + 1000 * rng.random((nx, nz))
    vs = vp / (1.6 + 0.3 * rng.random((nx, nz)))
    rho = 2000 + 400 * rng.random((nx, nz))
    la, mu, l2m, b, bm, vpmax = O.eiso_materials(vp, vs, rho)
    h = 1.0
    dt = 0.5 * h / (math.sqrt(2) * vpmax)
    d, dh, dH = O.eiso_profiles(P, h, vp)
    args = (nx, nz, P, h, dt, la, mu, l2m, b, bm, d, dh, dH)
    plain, rounded = O.EIso(*args), O.EIso(*args)
    rounded.set_bfp(BFP_BLOCK, "x")
    dev = api.EIsoDevice(*args, "bfp16")
    NX, NZ = nx + 2 * P, nz + 2 * P
    inter = np.zeros((NX, NZ), bool)
    inter[P:P + nx, P:P + nz] = True
    for f in FIELDS:
        scale = 1e-3 if f.startswith("v") else 1e4
        tot, xp, zp = (scale * rng.standard_normal((NX, NZ)) for _ in range(3))
        xp[inter] = 0
        zp[inter] = 0
        dev.set_field(f, xp, part="x")
        dev.set_field(f, zp, part="z")
        dev.set_field(f, np.where(inter, tot, 0), part="total")
        # the oracles start from the stored (rounded) state
        for o in (plain, rounded):
            o.set(f, "x", dev.get_field(f, part="x"))
            o.set(f, "z", dev.get_field(f, part="z"))
            o.set(f, "total", dev.get_field(f, part="total"))
    return plain, rounded, dev


@pytest.mark.parametrize("shape", [(13, 9, 3), (9, 14, 4), (33, 40, 8), (40, 12, 2), (37, 29, 5)])
def test_bfp16_steps_from_random_state(shape):
    nx, nz, P = shape
    plain, rounded, dev = _bfp_pair(nx, nz, P, sum(shape) + 3)
    for _ in range(4):
        for o in (plain, rounded):
            o.velocity()
            o.stress()
    dev.run(4)
    for f in FIELDS:
        got = dev.get_field(f, part="total")
        e_r = O.rel_l2(got, rounded.get(f, "total"))
        e_p = O.rel_l2(got, plain.get(f, "total"))
        assert e_r < 2e-5 and e_p < 1e-4, (f, e_r, e_p)
        for part in ("x", "z"):
            e = O.rel_l2(dev.get_field(f, part=part), rounded.get(f, part))
            assert e < 2e-5, (f, part, e)
    dev.close()


def test_bfp16_every_launch_config_and_batch_identical():
    p = W.cfg2(nx=150, nz=130, npml=9, nsteps=90, nshots=3, nrec=12)
    dev, n = api.eiso_device(p, "bfp16")
    nconf = dev.get_config()[1]
    dev.run(n)
    ref = [dev.traces(s) for s in range(3)]
    for config in range(nconf):
        dev.reset()
        dev.set_config(config)
        dev.run(n)
        for s in range(3):
            for x, y in zip(dev.traces(s), ref[s]):
                np.testing.assert_array_equal(x, y, err_msg=f"config {config} shot {s}")
    dev.close()
    alone = api.run_eiso(p, "bfp16", shots=[2])[0]
    for a, b in zip(ref[2], alone):
        np.testing.assert_array_equal(a, b)


def test_bfp16_shot_within_gate_and_as_the_rounding_oracle_predicts():
    p = W.cfg2(nx=300, nz=160, npml=12, nsteps=800, nshots=1, nrec=24)
    p.shots = [[("Bulk", 1.0, 50.0, 150.0, 5.0), ("Sxz", 0.5, 40.0, 40.0, 100.0)]]
    got = api.run_eiso(p, "bfp16")[0]
    assert all(np.isfinite(t).all() for t in got)
    ref = api.run_eiso(p, "fp64")[0]
    err = H.rel_l2(got, ref)
    assert err < 1e-3, err
    plain, _, _ = H.run_eiso_oracle(p)
    pred, _, _ = H.run_eiso_oracle(p, bfp_block=BFP_BLOCK, bfp_axis="x")
    predicted = H.rel_l2(pred, plain)
    assert 0.5 * predicted < err < 2.0 * predicted, (err, predicted)


def test_traces_array_equals_the_per_receiver_traces():
    """EIsoDevice.traces_array(shot): one [nrec, nsamples] copy per shot,
    the same samples as the per-receiver read, mid-run and at the end."""
    p = W.cfg2(nx=120, nz=80, npml=10, nsteps=120, nshots=3, nrec=12)
    dev, n = api.eiso_device(p, "fp32")
    for steps in (n // 3, n - n // 3):
        dev.run(steps)
        for s in range(3):
            a = dev.traces_array(s)
            rows = dev.traces(s)
            assert a.shape[0] == len(rows)
            for r, x in enumerate(rows):
                np.testing.assert_array_equal(a[r, :len(x)], x)
                assert not a[r, len(x):].any()
    dev.close()
