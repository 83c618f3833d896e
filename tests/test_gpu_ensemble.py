"""Ensembles of independent rings on one GPU (vr_ens_*) and the tile
autotuner (vr_autotune, vr_set_tiles).

- Rings of the seeded ensemble draw stepped together (one graph launch per
  RK substep for all rings) are bit-identical to each ring stepped alone,
  particles included.
- Every sweep tile variant the autotuner chooses among gives the oracle's
  substep to 1e-11, and the autotuner leaves the context's state as it found
  it.
"""
import numpy as np
import pytest

from tests.parity_util import STATE, assert_field_close, make_pair, prep

pytestmark = pytest.mark.gpu


def _state(run, part):
    return [run.get(n) for n in ("q1", "q2", "q3", "pres", "prg", "ru1")] + ([part.state()[0]] if part else [])


def test_ensemble_graph_matches_each_ring_alone():
    import vring_b200 as V
    from vring_b200 import ensemble as E
    specs = E.ensemble_specs(6, seed=1)
    rings = [E.make_ring(s, npart=4096) for s in specs]
    ens = V.Ensemble([r for r, _ in rings])
    ens.iterate(3)
    ens.sync()
    assert ens.launch_count > 0
    got = [_state(r, p) for r, p in rings]
    for r, p in rings:
        assert r.count_nonfinite() == 0 and r.max_divergence() <= 1e-9
    ens.close()
    for r, p in rings:
        p.attach(False)
        p.close()
        r.close()
    for i, s in enumerate(specs):
        r, p = E.make_ring(s, npart=4096)
        r.iterate(3)
        alone = _state(r, p)
        for a, b in zip(got[i], alone):
            assert np.array_equal(a, b), (i, s)
        p.attach(False)
        p.close()
        r.close()


@pytest.mark.parametrize("rv,zv", [(0, 0), (1, 1), (2, 2), (1, 0), (0, 2), (2, 1)])
def test_every_tile_variant_matches_oracle(rv, zv):
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 32, 96, 256
    orc, gpu = make_pair(nth, nr, nz, dt=1e-3, re=2000.0, slip=1.0)
    V.set_tiles(gpu, rv, zv)
    q = ring_fields(nth, nr, nz, 4.0, 12.0, R=1.0, sigma=0.2, noise=1e-3, seed=5)
    for n, a in zip(("q1", "q2", "q3"), q):
        orc.field(n)[...] = a
        gpu.set(n, a)
    prep(orc, gpu, 1, 0.0, 0)
    orc.substep(1)
    gpu.substep(1)
    for n in STATE + ["dph"]:
        assert_field_close(gpu, orc, n, rel=1e-11)
    gpu.close()


@pytest.mark.parametrize("rv,zv", [(0, 0), (0, 1), (1, 1)])
def test_long_line_tile_variants_match_oracle(rv, zv):
    # radial lines of 300-301 positions and axial lines of 513-514: beyond
    # the 16 x 17 positions of the 256-thread tiles, so the 16-line tiles run
    # as 32 chunks in one 512-thread CTA per SM (r and z by default; variant
    # 1 the 8-line tiles)
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 16, 300, 512
    orc, gpu = make_pair(nth, nr, nz, dt=1e-3, re=2000.0, slip=1.0)
    V.set_tiles(gpu, rv, zv)
    q = ring_fields(nth, nr, nz, 4.0, 12.0, R=1.0, sigma=0.2, noise=1e-3, seed=6)
    for n, a in zip(("q1", "q2", "q3"), q):
        orc.field(n)[...] = a
        gpu.set(n, a)
    prep(orc, gpu, 2, 0.0, 0)
    orc.substep(2)
    gpu.substep(2)
    for n in STATE + ["dph"]:
        assert_field_close(gpu, orc, n, rel=1e-11)
    gpu.close()


def test_autotune_restores_state_and_caches():
    import vring_b200 as V
    from vring_b200 import ensemble as E
    s = E.ensemble_specs(1, seed=1)[0]
    run, part = E.make_ring(s, npart=1024)
    run.iterate(1)
    before = _state(run, part)
    clk = run.clock
    choice = V.autotune(run, force=True)
    assert all(0 <= c <= 2 for c in choice)
    after = _state(run, part)
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
    assert run.clock == clk
    assert V.autotune(run) == choice            # cached per grid class
    print("autotuned (r, z) tile variants for", (s["nth"], s["nr"], s["nz"]), choice)
    part.attach(False)
    part.close()
    run.close()
