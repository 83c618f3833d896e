"""The mixed form (float storage of dq, ru, prg and pres; double velocity,
sweep work arrays, Poisson solve and dph) against the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# stated tolerance of the mixed form: max |u_mixed - u_fp64| over each
# component, relative to the velocity scale max |u| over all components,
# after 5 steps of the ring at 16 x 32 x 64 (float rounding of the predicted
# velocity reaches every component through the pressure correction)
TOL_U = 2e-6


def _pair(nth, nr, nz, seed=6):
    from oracle import oracle as O
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    orc = O.Oracle(nth, nr, nz, 4.0, 12.0, 1e-3, 1000.0, 1.0, 1.0, 1, 0)
    gpu = V.Run(nth, nr, nz, 4.0, 12.0, 1e-3, 1000.0, 1.0, 1.0, precision="mixed",
                theta_wavenumber="modified")
    for n, a in zip(("q1", "q2", "q3"), ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=seed)):
        orc.field(n)[...] = a
        gpu.set(n, a)
    return orc, gpu


def test_mixed_against_fp64_oracle():
    orc, gpu = _pair(16, 32, 64)
    gpu.iterate(5)
    orc.iterate(5)
    scale = max(np.abs(orc.field(n)).max() for n in ("q1", "q2", "q3"))
    for n in ("q1", "q2", "q3"):
        g, r = gpu.get(n), orc.field(n)
        err = np.abs(g - r).max() / scale
        print("mixed", n, err)
        assert err <= TOL_U, (n, err)
    p, pr = gpu.get("pres"), orc.field("pres")
    print("mixed pres", np.abs(p - pr).max() / np.abs(pr).max())
    assert np.abs(p - pr).max() <= 1e-4 * np.abs(pr).max()
    print("mixed max div", gpu.max_divergence())
    assert gpu.max_divergence() <= 1e-9


def test_mixed_refuses_per_routine_calls_and_converts_fields():
    import vring_b200 as V
    orc, gpu = _pair(8, 16, 32)
    with pytest.raises(V.VrError) as e:
        gpu.step()
    assert e.value.code == 7
    a = np.random.default_rng(1).uniform(-1, 1, gpu.extents("ru1")[:3])
    gpu.set("ru1", a)
    np.testing.assert_array_equal(gpu.get("ru1"), a.astype(np.float32).astype(np.float64))
