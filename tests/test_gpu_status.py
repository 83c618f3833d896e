"""Bounded device waits: a wait that runs out reports VR_ERR_TIMEOUT through
the context's status word and leaves the context usable.

The failure is made without a fault: vr_wait_selftest launches one warp that
waits on an mbarrier nothing completes, with a 10 ms limit.
"""
import numpy as np
import pytest

VR_ERR_TIMEOUT = 5


def _ring(V, nth=16, nr=16, nz=32):
    from vring_b200.synthetic import ring_fields
    run = V.Run(nth, nr, nz, 4.0, 12.0, 2e-3, 1000.0, 1.0, 1.0, theta_wavenumber="modified")
    for n, a in zip(("q1", "q2", "q3"), ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-4, seed=3)):
        run.set(n, a)
    return run


@pytest.mark.gpu
def test_wait_that_runs_out_reports_timeout_and_context_stays_usable():
    import vring_b200 as V
    ref, run = _ring(V), _ring(V)
    ref.iterate(1)
    run.iterate(1)
    assert run.wait_selftest(10_000_000) == VR_ERR_TIMEOUT
    with pytest.raises(V.VrError) as e:
        run.count_nonfinite()
    assert e.value.code == VR_ERR_TIMEOUT
    run.clear_status()
    assert run.count_nonfinite() == 0
    # the context keeps stepping, with the same results as one that never timed out
    ref.iterate(2)
    run.iterate(2)
    for n in ("q1", "q2", "q3", "pres"):
        assert np.array_equal(run.get(n), ref.get(n)), n
    assert run.count_nonfinite() == 0
    ref.close()
    run.close()


@pytest.mark.gpu
def test_wait_selftest_rejects_limits_out_of_range():
    import vring_b200 as V
    run = _ring(V)
    assert run.wait_selftest(10) == 8  # VR_ERR_ARG
    assert run.wait_selftest(5_000_000_000) == 8
    assert run.count_nonfinite() == 0
    run.close()
