"""GPU parity: every routine of the RK3 core through the C ABI against the CPU
restatement on the same seeded state.

Grids cover the transform paths: power-of-two theta and z below 32 (shared
memory radix-2 FFT), from 32 up (warp-register FFT and DCT), odd theta (the
reference's own case; direct DFT), even non-power-of-two theta (Nyquist slot,
direct DFT) and non-power-of-two z (direct DCT); the last tests run the
production transform sizes (theta 128, z 512) on a thin radial grid.  Tolerance: FP64, max |gpu - oracle| <= 1e-12 x max |oracle| per
field (1e-11 where a near-singular Poisson mode amplifies round-off).
"""
import numpy as np
import pytest

from parity_util import STATE, assert_field_close, copy_to_gpu, make_pair, prep, seed_random

pytestmark = pytest.mark.gpu

GRIDS = [(16, 16, 32), (9, 12, 20), (12, 16, 24), (32, 8, 64), (64, 12, 128)]


@pytest.fixture(params=GRIDS, ids=lambda g: "x".join(map(str, g)))
def grid(request):
    return request.param


def _pair(grid, **kw):
    return make_pair(*grid, **kw)


@pytest.mark.parametrize("irk", [1, 2, 3])
def test_hdnbc(grid, irk):
    orc, gpu = _pair(grid, inflow="reference")
    seed_random(orc, gpu, ["q3", "csort", "dq3no"], seed=irk)
    prep(orc, gpu, irk, 0.15, 3)
    orc.hdnbc()
    gpu.hdnbc()
    for n in ("csort", "tconv", "corr3n", "dq3no", "corr3s"):
        assert_field_close(gpu, orc, n)


@pytest.mark.parametrize("comp", [1, 2, 3])
def test_hdnl(grid, comp):
    orc, gpu = _pair(grid)
    seed_random(orc, gpu, ["q1", "q2", "q3", "dq1", "dq2", "dq3"], seed=comp)
    prep(orc, gpu)
    getattr(orc, "hdnl%d" % comp)()
    getattr(gpu, "hdnl%d" % comp)()
    assert_field_close(gpu, orc, "dq%d" % comp)


@pytest.mark.parametrize("irk", [1, 2, 3])
@pytest.mark.parametrize("slip", [1.0, 0.0])
def test_step(grid, irk, slip):
    orc, gpu = _pair(grid, slip=slip)
    seed_random(orc, gpu, ["q1", "q2", "q3", "dq1", "dq2", "dq3", "ru1", "ru2", "ru3", "prg",
                           "corr3s", "corr3n"], seed=10 + irk)
    prep(orc, gpu, irk)
    orc.step()
    gpu.step()
    for n in ("dq1", "dq2", "dq3", "ru1", "ru2", "ru3"):
        assert_field_close(gpu, orc, n)


@pytest.mark.parametrize("irk", [1, 3])
def test_divq(grid, irk):
    orc, gpu = _pair(grid)
    seed_random(orc, gpu, ["dq1", "dq2", "dq3"], seed=20 + irk)
    prep(orc, gpu, irk)
    orc.divq()
    gpu.divq()
    assert_field_close(gpu, orc, "rhs")


@pytest.mark.parametrize("wth", ["exact", "modified"])
def test_laplace_solve(grid, wth):
    orc, gpu = _pair(grid, wth=wth)
    seed_random(orc, gpu, ["rhs"], seed=30)
    prep(orc, gpu)
    orc.laplace_solve()
    gpu.laplace_solve()
    nth, nr, nz = grid
    g = gpu.get("dph")[:, 1:nr + 1, 1:nz + 1]
    r = orc.field("dph")[:, 1:nr + 1, 1:nz + 1]
    assert np.abs(g - r).max() <= 1e-11 * np.abs(r).max()


@pytest.mark.parametrize("irk", [1, 2])
def test_upsol(grid, irk):
    orc, gpu = _pair(grid)
    seed_random(orc, gpu, ["q1", "q2", "q3", "dq1", "dq2", "dq3", "dph"], seed=40 + irk)
    prep(orc, gpu, irk)
    orc.upsol()
    gpu.upsol()
    for n in ("q1", "q2", "q3", "dph"):
        assert_field_close(gpu, orc, n)


@pytest.mark.parametrize("irk", [1, 3])
def test_uppres(grid, irk):
    orc, gpu = _pair(grid)
    seed_random(orc, gpu, ["dph", "prg", "pres"], seed=50 + irk)
    prep(orc, gpu, irk)
    orc.uppres()
    gpu.uppres()
    for n in ("prg", "pres", "dph"):
        assert_field_close(gpu, orc, n)


def _ring_state(orc, gpu, grid, seed=0):
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = grid
    q1, q2, q3 = ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=seed)
    for n, a in (("q1", q1), ("q2", q2), ("q3", q3)):
        orc.field(n)[...] = a
    copy_to_gpu(orc, gpu, ["q1", "q2", "q3"])


@pytest.mark.parametrize("wth", ["exact", "modified"])
def test_fused_substep_matches_routine_sequence(grid, wth):
    orc, gpu = _pair(grid, wth=wth)
    _ring_state(orc, gpu, grid)
    prep(orc, gpu, 1, 2e-3, 0)
    orc.substep(1)
    gpu.substep(1)
    # the fused substep takes divq inside the forward theta transform and
    # leaves the rhs array alone; dph is the Poisson solve of that divq
    for n in STATE + ["dph"]:
        assert_field_close(gpu, orc, n, rel=1e-11)


def test_iterate_two_steps(grid):
    orc, gpu = _pair(grid, inflow="reference")
    _ring_state(orc, gpu, grid, seed=1)
    orc.iterate(2)
    gpu.iterate(2)
    gpu.sync()
    assert gpu.clock[1] == pytest.approx(4e-3)
    for n in STATE:
        assert_field_close(gpu, orc, n, rel=1e-10)


def test_projection_removes_divergence_with_modified_wavenumber():
    """With the discrete theta wavenumber the projection is exact up to the
    (m=0, kz=0) closure; the reference's exact m^2 leaves O(dtheta^2)."""
    grid = (16, 16, 32)
    res = {}
    for wth in ("exact", "modified"):
        orc, gpu = _pair(grid, wth=wth)
        _ring_state(orc, gpu, grid)
        gpu.iterate(1)
        res[wth] = gpu.max_divergence()
    assert res["modified"] < 1e-9
    assert res["exact"] > 10 * res["modified"]


def test_nonfinite_detection():
    orc, gpu = _pair((16, 16, 32))
    assert gpu.count_nonfinite() == 0
    q = gpu.get("q1")
    q[3, 4, 5] = np.nan
    gpu.set("q1", q)
    assert gpu.count_nonfinite() == 1


def test_batched_thomas_and_block_thomas():
    import vring_b200 as V
    from oracle import oracle as O
    rng = np.random.default_rng(7)
    nb, n = 33, 57
    a, c = rng.uniform(-1, 0, (nb, n)), rng.uniform(-1, 0, (nb, n))
    b, r = 3 + rng.uniform(0, 1, (nb, n)), rng.normal(size=(nb, n))
    x = V.solve_lap_thom(r, a, b, c)
    for i in range(nb):
        np.testing.assert_allclose(x[i], O.solve_lap_thom(r[i], a[i], b[i], c[i]), rtol=0, atol=1e-14)
    m, nblk = 6, 9
    b1, b3 = rng.uniform(-1, 0, (4, m * nblk)), rng.uniform(-1, 0, (4, m * nblk))
    b2, rr = 7 + rng.uniform(0, 1, (4, m * nblk)), rng.normal(size=(4, m * nblk))
    xs = V.solve_lap_bthom(rr, b1, b2, b3, m, nblk)
    for i in range(4):
        ref = O.solve_lap_bthom(rr[i], b1[i], b2[i], b3[i], m, nblk)
        np.testing.assert_allclose(xs[i], ref, rtol=0, atol=1e-13)


@pytest.mark.parametrize("wth", ["exact", "modified"])
def test_production_transform_sizes(wth):
    grid = (128, 8, 512)
    orc, gpu = _pair(grid, wth=wth)
    seed_random(orc, gpu, ["rhs"], seed=60)
    prep(orc, gpu)
    orc.laplace_solve()
    gpu.laplace_solve()
    g = gpu.get("dph")[:, 1:9, 1:513]
    r = orc.field("dph")[:, 1:9, 1:513]
    assert np.abs(g - r).max() <= 1e-11 * np.abs(r).max()
    orc, gpu = _pair(grid, wth=wth)
    _ring_state(orc, gpu, grid)
    prep(orc, gpu, 1, 5e-4, 0)
    orc.substep(1)
    gpu.substep(1)
    # the fused substep takes divq inside the forward theta transform and
    # leaves the rhs array alone; dph is the Poisson solve of that divq
    for n in STATE + ["dph"]:
        assert_field_close(gpu, orc, n, rel=1e-11)


def test_streamed_z_transform_many_tiles_per_cta():
    # 128 x 64 x 512: 512 tiles of the TMA-streamed 512-point z transform, so
    # each persistent CTA takes three or four and its three buffers are reused
    grid = (128, 64, 512)
    orc, gpu = _pair(grid, wth="modified")
    seed_random(orc, gpu, ["rhs"], seed=61)
    prep(orc, gpu)
    orc.laplace_solve()
    gpu.laplace_solve()
    g = gpu.get("dph")[:, 1:65, 1:513]
    r = orc.field("dph")[:, 1:65, 1:513]
    assert np.abs(g - r).max() <= 1e-11 * np.abs(r).max()


@pytest.mark.parametrize("wth", ["exact", "modified"])
def test_streamed_z_transform_three_tiles_per_radius(wth):
    # Ntheta 48: three 16-slot tiles per radial index (the theta transform
    # takes the direct sums at this length), 7 radii, 512 planes
    grid = (48, 7, 512)
    orc, gpu = _pair(grid, wth=wth)
    seed_random(orc, gpu, ["rhs"], seed=62)
    prep(orc, gpu)
    orc.laplace_solve()
    gpu.laplace_solve()
    g = gpu.get("dph")[:, 1:8, 1:513]
    r = orc.field("dph")[:, 1:8, 1:513]
    assert np.abs(g - r).max() <= 1e-11 * np.abs(r).max()


def test_slab_transforms_match_separate_transforms():
    # Ntheta 128, Nz 512: the fused substep's transforms as slab cluster
    # kernels (divq + theta + z forward, z + theta inverse) against the
    # separate transform kernels; the theta transforms pair other lines, so
    # the two agree to rounding
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 128, 24, 512
    q = ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=9)
    out = []
    for slab in (True, False):
        gpu = V.Run(nth, nr, nz, 4.0, 12.0, 5e-4, 3000.0, 1.0, 1.0, theta_wavenumber="modified")
        gpu.set_slab_transforms(slab)
        for n, a in zip(("q1", "q2", "q3"), q):
            gpu.set(n, a)
        gpu.iterate(2)
        out.append({n: gpu.get(n) for n in STATE + ["dph"]})
        gpu.close()
    for n in STATE + ["dph"]:
        a, b = out[0][n], out[1][n]
        scale = max(np.abs(b).max(), 1e-300)
        # dph carries the near-singular low modes' amplification of rounding
        # (the tolerance of every dph comparison with the oracle)
        rel = 1e-11 if n == "dph" else 1e-12
        assert np.abs(a - b).max() <= rel * scale, (n, np.abs(a - b).max() / scale)
