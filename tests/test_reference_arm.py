"""The reference arm of bench.py on the CPU: the reference program built from
its sources (oracle/_ref) timed over a bounded sample, as a positive rate
whatever the start-up noise of its runs."""
import pytest

from oracle import oracle as O


@pytest.mark.timeout(300)
def test_reference_rate_is_positive_on_a_small_shot():
    if not O.ref_available():
        pytest.skip("reference build absent (oracle/_ref)")
    import bench
    from seismod_b200 import workloads as W
    p = W.cfg0(nx=64, nz=48, npml=8, nsteps=200, nrec=6)
    # 2 steps: the (2 + S) - 2 difference is mostly start-up noise here, the
    # case that once gave a negative rate
    for steps in (2, 50):
        rate, sample = bench.reference_rate("eiso", p, steps)
        assert rate is not None and rate > 0, sample
        assert f"{steps} steps of the full grid" in sample
        assert "fastest of two runs" in sample or "start-up included" in sample
