"""The workloads beside the benchmark, at their own shapes.

- the 64 x 32 x 128 single ring with 16,384 tracers (Re 1000, dt 2e-3),
  against the oracle step by step;
- an ensemble of independent rings drawn at random (Nr in {64, 96, 128},
  Ntheta in {32, 64}, Nz in {128, 256}, Re in [500, 4000], R in [0.8, 1.2],
  sigma/R in [0.1, 0.3]) in the mixed form, one context per ring on one GPU:
  each ring of the ensemble must match the same ring run alone;
- the lines longer than the register-resident sweeps and transforms take
  (Ntheta 256, Nz 1024), against the oracle;
- the head-on collision of two opposite rings at 512 x 256 x 1024 (about
  134 M cells), run at full size in both precision forms: the projected
  velocity stays divergence-free and finite.

The reference's z boundaries (wall/inflow and convective outflow) replace the
periodic z of the collision and single-ring descriptions, as everywhere in
this library.
"""
import numpy as np
import pytest

from parity_util import STATE, assert_field_close, make_pair, prep


def _inject_annulus(parts, n, r0, r1, z0, z1, seed):
    from vring_b200.synthetic import annulus_particles
    x, y, z = annulus_particles(n, r0, r1, z0, z1, seed=seed)
    for i in range(n):
        slots = [p.injc(float(x[i]), float(y[i]), float(z[i])) for p in parts]
        assert len(set(slots)) == 1


@pytest.mark.gpu
def test_single_ring_64x32x128_with_tracers_matches_oracle():
    from oracle import oracle as O
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 32, 64, 128
    orc, gpu = make_pair(nth, nr, nz, dt=2e-3, re=1000.0, slip=1.0)
    q = ring_fields(nth, nr, nz, 4.0, 12.0, R=1.0, sigma=0.2, gamma=1.0, z0=3.0, noise=1e-4, seed=0)
    for n, a in zip(("q1", "q2", "q3"), q):
        orc.field(n)[...] = a
        gpu.set(n, a)
    npart = 16384
    op = O.OraclePart(orc, 8, npart, 1)
    gp = V.Part(gpu, 8, npart, 1)
    _inject_annulus([op, gp], npart, 0.5, 1.5, 2.0, 4.0, seed=0)
    gp.attach(True)
    gpu.iterate(3)
    for _ in range(3):  # loop.F90:65-68: iter_part, then the three substeps
        op.iter_part(1)
        orc.iterate(1)
    for n in ("q1", "q2", "q3", "pres"):
        assert_field_close(gpu, orc, n, rel=1e-10)
    u, v, isf, cnt = gp.state()
    assert cnt["npart"] == op.npart
    scale = np.maximum(np.abs(op.u).max(axis=0), 1e-30)
    assert (np.abs(u - op.u) / scale).max() <= 1e-10
    # with the reference's theta wavenumber m^2 the projection leaves an
    # O(dtheta^2) divergence (the round-off bound needs the discrete one)
    gp.attach(False)
    gp.close()
    gpu.close()


@pytest.mark.gpu
def test_ensemble_of_random_rings_matches_each_ring_alone():
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    rng = np.random.default_rng(1)
    specs = []
    for _ in range(6):
        specs.append(dict(nr=int(rng.choice([64, 96, 128])), nth=int(rng.choice([32, 64])),
                          nz=int(rng.choice([128, 256])), re=float(rng.uniform(500.0, 4000.0)),
                          R=float(rng.uniform(0.8, 1.2)), sr=float(rng.uniform(0.1, 0.3))))

    def make(s, seed):
        run = V.Run(s["nth"], s["nr"], s["nz"], 4.0, 12.0, 1e-3, s["re"], 1.0, 1.0, precision="mixed",
                    theta_wavenumber="modified")
        q = ring_fields(s["nth"], s["nr"], s["nz"], 4.0, 12.0, R=s["R"], sigma=s["sr"] * s["R"], gamma=1.0,
                        z0=3.0, noise=1e-4, seed=seed)
        for n, a in zip(("q1", "q2", "q3"), q):
            run.set(n, a)
        part = V.Part(run, 8, 4096, 1)
        _inject_annulus([part], 4096, 0.5 * s["R"], 1.5 * s["R"], 2.0, 4.0, seed=seed)
        part.attach(True)
        return run, part

    # the ensemble: every ring resident at once, stepped in turn
    ens = [make(s, i) for i, s in enumerate(specs)]
    for _ in range(2):
        for run, _p in ens:
            run.iterate(1)
    got = []
    for run, part in ens:
        assert run.count_nonfinite() == 0
        assert run.max_divergence() <= 1e-9
        got.append([run.get(n) for n in ("q1", "q2", "q3", "pres")] + [part.state()[0]])
    for run, part in ens:
        part.attach(False)
        part.close()
        run.close()
    # each ring alone, in a fresh context
    for i, s in enumerate(specs):
        run, part = make(s, i)
        run.iterate(2)
        alone = [run.get(n) for n in ("q1", "q2", "q3", "pres")] + [part.state()[0]]
        for a, b in zip(got[i], alone):
            assert np.array_equal(a, b), (i, s)
        part.attach(False)
        part.close()
        run.close()


@pytest.mark.gpu
def test_long_theta_and_z_lines_match_oracle():
    # Ntheta 256 and Nz 1024: the fused right-hand side with 8-element theta
    # chunks, the 16 x 16 theta transform, the 1024-point DCT, and z lines of
    # 1025 unknowns in the shared-memory sweep
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 256, 8, 1024
    orc, gpu = make_pair(nth, nr, nz, dt=5e-4, re=2000.0, slip=1.0)
    q = ring_fields(nth, nr, nz, 4.0, 12.0, R=1.0, sigma=0.3, noise=1e-3, seed=4)
    for n, a in zip(("q1", "q2", "q3"), q):
        orc.field(n)[...] = a
        gpu.set(n, a)
    prep(orc, gpu, 1, 0.0, 0)
    orc.substep(1)
    gpu.substep(1)
    # (the fused substep takes divq inside the theta transform and leaves the
    # rhs array alone; dph is the Poisson solve of that right-hand side)
    for n in STATE + ["dph"]:
        assert_field_close(gpu, orc, n, rel=1e-11)
    gpu.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_head_on_collision_512x256x1024_full_size(precision):
    import vring_b200 as V
    from vring_b200.synthetic import annulus_particles, ring_fields
    nth, nr, nz = 256, 512, 1024
    run = V.Run(nth, nr, nz, 4.0, 16.0, 2.5e-4, 5000.0, 1.0, 1.0, precision=precision,
                theta_wavenumber="modified")
    q = ring_fields(nth, nr, nz, 4.0, 16.0, noise=1e-3, seed=3,
                    rings=[(1.0, 0.15, 1.0, 5.0), (1.0, 0.15, -1.0, 11.0)])
    for n, a in zip(("q1", "q2", "q3"), q):
        run.set(n, a)
    del q
    npart = 1 << 20
    part = V.Part(run, 8, npart, 1)
    u = np.zeros((npart, 117), order="F")
    for h, zc in enumerate((5.0, 11.0)):
        x, y, z = annulus_particles(npart // 2, 0.7, 1.3, zc - 0.3, zc + 0.3, seed=3 + h)
        sl = slice(h * (npart // 2), (h + 1) * (npart // 2))
        u[sl, 0], u[sl, 1], u[sl, 2] = x, y, z
    part.set_state(u, np.zeros((npart, 3), order="F"), None, npart)
    del u
    part.attach(True)
    run.iterate(2)
    assert run.count_nonfinite() == 0
    assert run.max_divergence() <= 1e-9
    assert part.counts["npart"] == npart
    part.attach(False)
    part.close()
    run.close()
