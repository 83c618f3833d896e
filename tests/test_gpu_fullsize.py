"""The benchmark configuration itself (256 x 128 x 512, Re 3000, dt 5e-4,
1,048,576 tracers) through size-independent properties, in both forms:
max |div u| <= 1e-9 after the projection, every value finite, the kinetic
energy of the ring decaying (viscous flow, no forcing), the particles staying
in the domain, and the mixed form tracking the FP64 form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NTH, NR, NZ = 128, 256, 512


def _energy(run):
    # sum of q1^2 + (q2/rc)^2 + q3^2 weighted by the cell volume r dr dtheta dz
    q1, q2, q3 = run.get("q1"), run.get("q2"), run.get("q3")
    dr = 4.0 / NR
    rm = (np.arange(NR + 3) - 0.5) * dr
    rc = np.maximum((np.arange(NR + 3) - 1.0) * dr, 1e-30)
    w = rm[None, 1:NR + 1, None]
    e = (q1[:, 1:NR + 1, 1:NZ + 1] ** 2 + (q2[:, 1:NR + 1, 1:NZ + 1] / rc[None, 1:NR + 1, None]) ** 2
         + q3[:, 1:NR + 1, 1:NZ + 1] ** 2) * w
    return float(e.sum())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_benchmark_configuration_properties(precision):
    import vring_b200 as V
    from vring_b200.synthetic import annulus_particles, ring_fields
    run = V.Run(NTH, NR, NZ, 4.0, 12.0, 5e-4, 3000.0, 1.0, 1.0, precision=precision,
                theta_wavenumber="modified")
    q = ring_fields(NTH, NR, NZ, 4.0, 12.0, R=1.0, sigma=0.2, gamma=1.0, z0=3.0, noise=1e-4, seed=0)
    for n, a in zip(("q1", "q2", "q3"), q):
        run.set(n, a)
    npart = 1 << 16
    p = V.Part(run, 8, npart, 1)
    x, y, z = annulus_particles(npart, 0.3, 1.7, 2.0, 4.0, seed=0)
    u = np.zeros((npart, 117), order="F")
    u[:, 0], u[:, 1], u[:, 2] = x, y, z
    p.set_state(u, np.zeros((npart, 3), order="F"), None, npart)
    p.attach(True)
    e0 = _energy(run)
    run.iterate(4)
    assert run.count_nonfinite() == 0
    assert run.max_divergence() <= 1e-9
    e1 = _energy(run)
    assert e1 < e0 and e1 > 0.95 * e0
    uu, vv, isf, cnt = p.state()
    assert cnt["npart"] == npart                       # no tracer left the ring region
    r = np.hypot(uu[:, 0], uu[:, 1])
    assert r.max() < 2.0 and uu[:, 2].min() > 1.5 and uu[:, 2].max() < 4.5
    p.close()
    if precision == "mixed":
        ref = V.Run(NTH, NR, NZ, 4.0, 12.0, 5e-4, 3000.0, 1.0, 1.0, theta_wavenumber="modified")
        for n, a in zip(("q1", "q2", "q3"), q):
            ref.set(n, a)
        ref.iterate(4)
        scale = max(np.abs(ref.get(n)).max() for n in ("q1", "q2", "q3"))
        for n in ("q1", "q2", "q3"):
            assert np.abs(run.get(n) - ref.get(n)).max() <= 2e-6 * scale
