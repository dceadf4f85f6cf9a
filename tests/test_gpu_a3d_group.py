"""Grouped a_iso_3d stepping (sm_a3d_group_run): several 3-D models of
different grid sizes, sources and receivers advanced by one launch per step
must end bit for bit where each model's own run leaves it -- traces and the
whole state -- in FP32, FP64, 16-bit (through the power-of-two rescales) and
block storage."""
import numpy as np
import pytest

from seismod_b200 import _lib as L
from seismod_b200 import api
from seismod_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _problem(shape, npml, seed, nrec=6, nsteps=70):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    vp = 1500 + 2500 * rng.random((nx, ny, nz))
    rho = 1800 + 500 * rng.random((nx, ny, nz))
    d = (5.0, 4.0, 3.0)
    dt_ms = 0.5 / (vp.max() * np.sqrt(sum(1 / h ** 2 for h in d))) * 1e3
    src = [("Bulk", 1.0, 40.0, (nx // 2) * d[0], (ny // 3) * d[1], (nz // 2) * d[2])]
    comps = ["P", "Vx", "Vy", "Vz"]
    rec = [(comps[r % 4], float(rng.integers(0, nx)) * d[0], float(rng.integers(0, ny)) * d[1],
            float(rng.integers(0, nz)) * d[2], 0.0, dt_ms) for r in range(nrec)]
    return W.A3DProblem(vp, rho, d, npml, dt_ms, W.steps_duration(nsteps, dt_ms), src, rec,
                        Rc=1e-3, kappa_max=2.0, alpha_max=1, name=f"g{seed}")


def _problems():
    # uneven sizes: tiles clear of the frame and ring tiles, a grid narrower
    # than one tile in z, one without an interior class, uneven x chunks
    return [_problem((40, 50, 90), 4, 1),
            _problem((24, 30, 20), 6, 2),
            _problem((70, 21, 37), 3, 3),
            _problem((17, 64, 64), 8, 4, nrec=9)]


def _state(d):
    return [d.get_field(f) for f in ("p", "vx", "vy", "vz")]


@pytest.mark.parametrize("precision", ["fp32", "fp64", "fp16", "bfp16"])
def test_a3d_group_equals_separate_runs(precision):
    probs = _problems()
    devs, ns = zip(*[api.a3d_device(p, precision) for p in probs])
    n = min(ns)
    alone = []
    for p in probs:
        dev, _ = api.a3d_device(p, precision)
        dev.run(n)
        alone.append((dev.traces(), _state(dev)))
        dev.close()
    # two calls of uneven length: single steps, a graph of 16, a 16-bit
    # rescale period crossed inside a call
    api.a3d_group_run(list(devs), 21)
    api.a3d_group_run(list(devs), n - 21)
    for d, (tr, st) in zip(devs, alone):
        d.sync()
        for x, y in zip(d.traces(), tr):
            np.testing.assert_array_equal(x, y)
        for x, y in zip(_state(d), st):
            np.testing.assert_array_equal(x, y)
        d.close()


def test_a3d_group_mixed_with_own_runs():
    """A handle may take steps alone (another launch configuration, so other
    tensor maps) before and after a grouped call."""
    probs = _problems()[:3]
    devs, ns = zip(*[api.a3d_device(p, "fp32") for p in probs])
    n = min(ns)
    alone = []
    for p in probs:
        dev, _ = api.a3d_device(p, "fp32")
        dev.run(n)
        alone.append(dev.traces())
        dev.close()
    devs[0].set_config(0)
    devs[0].run(9)
    api.a3d_group_run([devs[1]], 9)
    devs[2].run(9)
    api.a3d_group_run(list(devs), 33)
    for d in devs:
        d.run(n - 42)
    for d, ref in zip(devs, alone):
        for x, y in zip(d.traces(), ref):
            np.testing.assert_array_equal(x, y)
        d.close()


def test_a3d_group_rejects_mixed_precision_and_repeats():
    p = _problems()[1]
    a, _ = api.a3d_device(p, "fp32")
    b, _ = api.a3d_device(p, "fp64")
    with pytest.raises(L.SeismodError):
        api.a3d_group_run([a, b], 1)
    with pytest.raises(L.SeismodError):
        api.a3d_group_run([a, a], 1)
    a.close()
    b.close()


def test_a3d_group_more_than_one_launch():
    """More handles than one launch takes (16): two launches per step."""
    probs = [_problem((12 + k, 14, 16 + 2 * k), 2, 40 + k, nrec=2, nsteps=20) for k in range(18)]
    devs, ns = zip(*[api.a3d_device(p, "fp32") for p in probs])
    n = min(ns)
    api.a3d_group_run(list(devs), n)
    for p, d in zip(probs, devs):
        ref, _ = api.a3d_device(p, "fp32")
        ref.run(n)
        for x, y in zip(d.traces(), ref.traces()):
            np.testing.assert_array_equal(x, y)
        ref.close()
        d.close()
