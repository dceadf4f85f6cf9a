"""Per-kernel timing (sm_*_set_timing / sm_*_kernel_stats): every update
launch is timed once, with and without CUDA-graph replay (inside graphs the
events are the graph's own event nodes), the durations are positive and no
longer than the steps they sit in, and timing changes no result."""
import numpy as np
import pytest
import torch

from seismod_b200 import api
from seismod_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _whole_ms(dev, n):
    st = torch.cuda.ExternalStream(dev.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dev.sync()
    e0.record(st)
    dev.run(n)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _check(make, fields, graph):
    plain, _ = make()
    timed, _ = make()
    for d in (plain, timed):
        d.set_graph(graph)
    n = 3 * 16 + 5   # whole graphs and single steps
    plain.run(n)
    timed.set_timing(True)
    timed.kernel_stats(reset=True)
    timed.run(n)
    ms, k, _ = timed.kernel_stats(reset=True)
    assert k == n
    assert ms > 0
    # the timed launches sit inside the steps: their mean is below the
    # whole step's (measured untimed, graphs replayed)
    timed.set_timing(False)
    whole = _whole_ms(timed, 32) / 32
    assert ms / k < 1.5 * whole
    # timing on and off again mid-run: same state as the plain run
    plain.run(32)
    timed_state = fields(timed)
    for a, b in zip(fields(plain), timed_state):
        np.testing.assert_array_equal(a, b)
    plain.close()
    timed.close()


@pytest.mark.parametrize("graph", [0, 16])
@pytest.mark.parametrize("precision", ["fp32", "bfp16"])
def test_a3d_timing(graph, precision):
    p = W.cfg1(n=64, nsteps=200, rec_stride=8)
    _check(lambda: api.a3d_device(p, precision),
           lambda d: [d.get_field(c) for c in ("p", "vx", "vy", "vz")] + list(d.traces()), graph)


@pytest.mark.parametrize("graph", [0, 16])
def test_eiso_timing(graph):
    p = W.cfg2(nx=200, nz=120, nsteps=200, nshots=4, nrec=16)
    _check(lambda: api.eiso_device(p, "fp32"),
           lambda d: [d.get_field(c, shot=s) for c in ("vx", "txx") for s in (0, 3)]
           + [d.traces(shot=3)], graph)
