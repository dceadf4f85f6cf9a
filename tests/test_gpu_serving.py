"""The request loop (sm_server_*): every result is bitwise the result of the
same shot run alone on a handle of its own, whatever ran beside it;
admission keeps the admitted device memory within the budget."""
import numpy as np
import pytest

from seismod_b200 import api
from seismod_b200 import serving
from seismod_b200 import workloads as W
from seismod_b200._lib import SeismodError, SM_EBUSY

pytestmark = pytest.mark.gpu


def _mix():
    return [("eiso", W.eiso_request(120, 300, 11)), ("a3d", W.a3d_request(40, 160, 12)),
            ("eiso", W.eiso_request(260, 220, 13)), ("eiso", W.eiso_request(90, 400, 14)),
            ("a3d", W.a3d_request(56, 120, 15)), ("eiso", W.eiso_request(200, 150, 16))]


def _alone(kind, p, precision):
    if kind == "eiso":
        return api.run_eiso(p, precision)[0]
    return api.run_a3d(p, precision)


def _same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("precision,graph,group", [("fp32", 0, False), ("fp32", 16, False),
                                                   ("fp16", 16, False), ("fp32", 16, True),
                                                   ("fp16", 0, True)])
def test_results_in_the_mix_equal_results_alone(precision, graph, group):
    """With group=True the running e_iso requests are stepped together, one
    launch per step over their uneven grids; results stay those of each shot
    alone."""
    mix = _mix()
    srv = serving.Server(max_active=4, slice_steps=32, graph_steps=graph, group=group)
    tickets = [srv.submit(k, p, precision) for k, p in mix]
    srv.drain(timeout=300)
    st = srv.stats()
    assert st["completed"] == len(mix) and st["failed"] == 0
    assert st["max_running"] >= 2           # requests did overlap
    assert 0 < st["latency_p50"] <= st["latency_p99"] <= st["latency_max"]
    for t, (k, p) in zip(tickets, mix):
        assert srv.status(t)[0] == 2
        _same(srv.traces(t), _alone(k, p, precision))
        srv.release(t)
    srv.close()


def test_admission_keeps_within_the_budget_and_rejects_oversize():
    mix = [("eiso", W.eiso_request(300, 120, 21 + i)) for i in range(5)]
    one = serving.device_bytes("eiso", mix[0][1])
    budget = int(2.5 * one)                 # room for two at a time
    srv = serving.Server(hbm_budget=budget, max_active=8, slice_steps=16)
    tickets = [srv.submit(k, p) for k, p in mix]
    with pytest.raises(SeismodError) as e:
        srv.submit("eiso", W.eiso_request(2500, 50, 30))
    assert e.value.code == SM_EBUSY
    srv.drain(timeout=300)
    st = srv.stats()
    assert st["completed"] == 5
    assert st["hbm_peak"] <= budget
    assert st["max_running"] <= 2
    for t, (k, p) in zip(tickets, mix):
        _same(srv.traces(t), _alone(k, p, "fp32"))
    srv.close()
