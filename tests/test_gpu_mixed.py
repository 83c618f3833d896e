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


def test_mixed_particles_against_fp64_oracle():
    """Mixed form particles: the fit and transforms in float, positions and
    the state in double; cell indices from the double positions."""
    from oracle import oracle as O
    import vring_b200 as V
    orc, gpu = _pair(16, 32, 64, seed=3)
    op = O.OraclePart(orc, 4, 300, 0)
    gp = V.Part(gpu, 4, 300, 0)
    rng = np.random.default_rng(12)
    n = 200
    r = rng.uniform(0.3, 3.5, n)
    th = rng.uniform(0, 2 * np.pi, n)
    z = rng.uniform(0.5, 11.5, n)
    xyz = np.stack([r * np.cos(th), r * np.sin(th), z], 1)
    vel, dvel, dd, cells = gp.probe(xyz)
    for i in range(0, n, 7):
        ref = op.probe(*xyz[i])
        idx, _ = op.cell(*xyz[i])
        assert tuple(cells[i]) == tuple(idx)
        np.testing.assert_allclose(vel[i], ref[:3], rtol=0, atol=1e-5 * np.abs(ref[:3]).max() + 1e-7)
        np.testing.assert_allclose(dvel[i].reshape(-1, order="F"), ref[3:12], rtol=0,
                                   atol=1e-4 * np.abs(ref[3:12]).max() + 1e-6)
    for i in range(n):
        op.injc(*xyz[i])
        gp.injc(*xyz[i])
    for _ in range(3):
        op.iter_part(1)
        gp.iter_part(1)
    u, v, isf, cnt = gp.state()
    assert cnt["npart"] == op.npart
    ou = op.u
    # positions (double state advanced with float velocities): relative to the domain size
    assert np.abs(u[:n, :3] - ou[:n, :3]).max() <= 1e-9 * 12.0
    gp.close()
