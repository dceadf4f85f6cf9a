"""Grouped e_iso stepping (sm_eiso_group_run): several models of different
grid sizes, shot counts and sources advanced by one launch per step must end
bit for bit where each model's own run leaves it, in FP32, FP64 and 16-bit
storage (through the power-of-two rescales)."""
import numpy as np
import pytest

from seismod_b200 import _lib as L
from seismod_b200 import api
from seismod_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _problems():
    # uneven sizes and shot counts; one grid narrower than a slab column
    return [W.cfg2(nx=150, nz=130, npml=9, nsteps=120, nshots=3, nrec=12, seed=3),
            W.cfg0(nx=96, nz=140, npml=7, nsteps=120, nrec=5),
            W.cfg2(nx=61, nz=23, npml=4, nsteps=120, nshots=2, nrec=4, seed=5),
            W.cfg0(nx=210, nz=180, npml=12, nsteps=120, nrec=9)]


@pytest.mark.parametrize("precision", ["fp32", "fp64", "fp16", "bfp16"])
def test_group_equals_separate_runs(precision):
    probs = _problems()
    devs, ns = zip(*[api.eiso_device(p, precision) for p in probs])
    n = min(ns)
    alone = []
    for p in probs:
        dev, _ = api.eiso_device(p, precision)
        dev.run(n)
        alone.append([dev.traces(s) for s in range(dev.nshots)])
        dev.close()
    # in two calls of uneven length, to cross the 16-step rescale period
    api.group_run(list(devs), 37)
    api.group_run(list(devs), n - 37)
    for d, ref in zip(devs, alone):
        d.sync()
        for s in range(d.nshots):
            for x, y in zip(d.traces(s), ref[s]):
                np.testing.assert_array_equal(x, y)
        d.close()


def test_group_mixed_with_own_runs():
    """A handle may take steps alone before and after a grouped call."""
    probs = _problems()[:2]
    devs, ns = zip(*[api.eiso_device(p, "fp32") for p in probs])
    n = min(ns)
    alone = []
    for p in probs:
        dev, _ = api.eiso_device(p, "fp32")
        dev.run(n)
        alone.append([dev.traces(s) for s in range(dev.nshots)])
        dev.close()
    devs[0].run(11)
    api.group_run([devs[1]], 11)
    api.group_run(list(devs), 50)
    for d in devs:
        d.run(n - 61)
    for d, ref in zip(devs, alone):
        for s in range(d.nshots):
            for x, y in zip(d.traces(s), ref[s]):
                np.testing.assert_array_equal(x, y)
        d.close()


def test_group_rejects_mixed_precision_and_repeats():
    p = _problems()[1]
    a, _ = api.eiso_device(p, "fp32")
    b, _ = api.eiso_device(p, "fp64")
    with pytest.raises(L.SeismodError):
        api.group_run([a, b], 1)
    with pytest.raises(L.SeismodError):
        api.group_run([a, a], 1)
    a.close()
    b.close()
