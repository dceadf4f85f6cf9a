"""CUDA-graph replay and the launch-configuration autotuner must not change
results: every comparison here is bitwise against the plain launch loop."""
import numpy as np
import pytest

from seismod_b200 import api
from seismod_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def _eiso_traces(p, precision, graph=0, tune=False, pieces=None):
    dev, n = api.eiso_device(p, precision)
    if tune:
        dev.autotune(trial_steps=4)
    if graph:
        dev.set_graph(graph)
    for k in (pieces or [n]):
        dev.run(k)
    out = [dev.traces(s) for s in range(dev.nshots)]
    dev.close()
    return out


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_eiso_graphs_equal_plain_launches(precision):
    p = W.cfg2(nx=96, nz=70, npml=8, nsteps=230, nshots=3, nrec=10)
    ref = _eiso_traces(p, precision)
    for graph in (2, 16):
        # uneven run lengths: eager steps up to a graph boundary, graphs, a tail
        got = _eiso_traces(p, precision, graph=graph, pieces=[7, 100, 3, 120])
        for a, b in zip(ref, got):
            _same(a, b)


def test_eiso_autotune_keeps_results_and_leaves_handle_reset():
    p = W.cfg0(nx=120, nz=90, npml=10, nsteps=180, nrec=6)
    ref = _eiso_traces(p, "fp32")
    dev, n = api.eiso_device(p, "fp32")
    dev.run(3)
    with pytest.raises(api.L.SeismodError):
        dev.autotune()                      # only at step 0
    dev.reset()
    config, ms = dev.autotune(trial_steps=4)
    assert 0 <= config < dev.get_config()[1] and ms > 0
    assert dev.step_count() == 0
    dev.run(n)
    _same(ref[0], dev.traces(0))
    dev.close()
    # a second handle of the same shape takes the cached choice
    dev, _ = api.eiso_device(p, "fp32")
    assert dev.autotune(trial_steps=4)[0] == config
    dev.close()


def _a3d_traces(p, precision, graph=0, tune=False, pieces=None):
    dev, n = api.a3d_device(p, precision)
    if tune:
        dev.autotune(trial_steps=3)
    if graph:
        dev.set_graph(graph)
    for k in (pieces or [n]):
        dev.run(k)
    out = dev.traces()
    dev.close()
    return out


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_a3d_graphs_equal_plain_launches(precision):
    p = W.cfg1(n=40, npml=6, nsteps=150, rec_stride=8)
    ref = _a3d_traces(p, precision)
    got = _a3d_traces(p, precision, graph=8, pieces=[5, 64, 1, 80])
    _same(ref, got)


def test_a3d_autotune_keeps_results():
    p = W.cfg1(n=40, npml=6, nsteps=120, rec_stride=8)
    ref = _a3d_traces(p, "fp32")
    got = _a3d_traces(p, "fp32", tune=True, graph=16)
    _same(ref, got)
