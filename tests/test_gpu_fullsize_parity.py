"""The timed configuration itself against the oracle, and the reference's
manufactured Poisson solution solved on the GPU.

- One FP64 RK3 step of the benchmark ring at 256 x 128 x 512 (Re 3000,
  dt 5e-4, free slip, discrete theta wavenumber) with 65,536 of the benchmark's
  tracers attached, on the GPU and in the oracle from the same state: q1..q3,
  pres, prg, ru1..ru3 and dph within 1e-11 of each field's scale, the tracer
  state within 1e-11, and the cell index of every tracer identical.  This
  covers the kernels only the benchmark size reaches: the r sweeps over 256/257
  unknowns, the radial Poisson table of 65 modes x 512 z modes x 256 rows, the
  streamed z transform and the fused right-hand side over its full grid.
- The mixed form after three steps of the same workload against the FP64
  oracle, one error per field (velocity, pressure, tracer positions), each
  within the tolerance stated in the test.
- The reference's manufactured solution sol_ex/rhs_ex (solp_tools.F90:95-126)
  through the GPU's laplace_solve: the error falls by 3.7-4.3x per grid
  doubling (second order), as the oracle's does.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NTH, NR, NZ = 128, 256, 512
RMAX, ZMAX, DT, RE, SLIP = 4.0, 12.0, 5e-4, 3000.0, 1.0
NPART = 1 << 16
FIELDS = ("q1", "q2", "q3", "pres", "prg", "ru1", "ru2", "ru3", "dph")


def _tracers(n):
    from vring_b200.synthetic import annulus_particles
    x, y, z = annulus_particles(n, 0.3, 1.7, 2.0, 4.0, seed=0)
    u = np.zeros((n, 117), order="F")
    v = np.zeros((n, 3), order="F")
    u[:, 0], u[:, 1], u[:, 2] = x, y, z
    u[:, 6] = u[:, 10] = u[:, 14] = 1.0
    return u, v


def _pair(precision):
    from oracle import oracle as O
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    q = ring_fields(NTH, NR, NZ, RMAX, ZMAX, R=1.0, sigma=0.2, gamma=1.0, z0=3.0, noise=1e-4, seed=0)
    orc = O.Oracle(NTH, NR, NZ, RMAX, ZMAX, DT, RE, 1.0, SLIP, 1, 0, 0)
    gpu = V.Run(NTH, NR, NZ, RMAX, ZMAX, DT, RE, 1.0, SLIP, precision=precision,
                theta_wavenumber="modified")
    for n, a in zip(("q1", "q2", "q3"), q):
        orc.field(n)[...] = a
        gpu.set(n, a)
    u, v = _tracers(NPART)
    gp = V.Part(gpu, 8, NPART, 1)
    gp.set_state(u, v, None, NPART)
    gp.attach(True)
    op = O.OraclePart(orc, 8, NPART, 1)
    op.u[...] = u
    op.v[...] = v
    op._s.nlast = op._s.npart = NPART
    return orc, gpu, op, gp


def _steps(orc, gpu, op, n):
    gpu.iterate(n)
    for _ in range(n):
        op.iter_part(1)   # loop.F90:65-68: particles first, in the velocity at the step start
        orc.iterate(1)


def _rel(g, r):
    return float(np.abs(g - r).max() / max(np.abs(r).max(), 1e-300))


def test_benchmark_step_matches_oracle_fp64():
    orc, gpu, op, gp = _pair("fp64")
    _steps(orc, gpu, op, 1)
    errs = {n: _rel(gpu.get(n), orc.field(n)) for n in FIELDS}
    print("full-size FP64 step, max|gpu - oracle| / scale:", errs)
    for n, e in errs.items():
        assert e <= 1e-11, (n, e)
    uu, _, _, cnt = gp.state()
    assert cnt["npart"] == NPART
    live = slice(0, NPART)
    ou = op.u[live]
    # position, velocity and the interpolated fluid velocity/gradient/Hessian
    for c0, c1 in ((0, 3), (3, 6), (78, 81), (81, 90), (90, 117)):
        e = _rel(uu[live, c0:c1], ou[:, c0:c1])
        assert e <= 1e-11, (c0, c1, e)
    # cell index of every tracer at its new position, bit for bit
    _, _, _, cells = gp.probe(uu[live, 0:3])
    for i in range(NPART):
        idx, _ = op.cell(*ou[i, 0:3])
        assert tuple(cells[i]) == tuple(idx), (i, cells[i], idx)
    gp.close()
    gpu.close()


def test_benchmark_mixed_form_error_per_field():
    """Stated tolerances of the mixed form after 3 steps of the benchmark
    workload, against the FP64 oracle: velocity 2e-5 of max|u|, pressure 2e-3
    of max|pres|, tracer positions 1e-9 of the domain length."""
    orc, gpu, op, gp = _pair("mixed")
    _steps(orc, gpu, op, 3)
    uscale = max(np.abs(orc.field(n)).max() for n in ("q1", "q2", "q3"))
    eu = max(np.abs(gpu.get(n) - orc.field(n)).max() for n in ("q1", "q2", "q3")) / uscale
    ep = _rel(gpu.get("pres"), orc.field("pres"))
    uu, _, _, _ = gp.state()
    ex = float(np.abs(uu[:NPART, 0:3] - op.u[:, 0:3]).max() / ZMAX)
    print("mixed form after 3 steps vs FP64 oracle: velocity %.3e, pressure %.3e, positions %.3e"
          % (eu, ep, ex))
    assert gpu.max_divergence() <= 1e-9
    assert eu <= 2e-5
    assert ep <= 2e-3
    assert ex <= 1e-9
    gp.close()
    gpu.close()


def _mms_gpu(n, nth=13):
    """Error of the GPU laplace_solve against sol_ex on an n x n grid (r, z in
    [0, 1]) with the reference's real*4 pi (solp_tools.F90:95-126)."""
    import vring_b200 as V
    pi = np.float64(np.float32(4 * np.arctan(np.float32(1))))

    def sol_ex(th, rr, zz):
        return np.cos(2 * pi * zz) / (4 * pi ** 2) * (rr ** 3 - 1.5 * rr ** 2) * (1 - 0.5 * np.cos(5 * th))

    def rhs_ex(th, rr, zz):
        return (np.cos(2 * pi * zz) * (rr ** 3 - 1.5 * rr ** 2) * (1 - 0.5 * np.cos(5 * th))
                + np.cos(2 * pi * zz) * (6 - 9 * rr) / (4 * pi ** 2) * (1 - 0.5 * np.cos(5 * th))
                + np.cos(2 * pi * zz) / (4 * pi ** 2) * (rr ** 3 - 1.5 * rr ** 2)
                * (-0.5 * 25 * np.cos(5 * th)) / rr ** 2)

    run = V.Run(nth, n, n, 1.0, 1.0, 1e-3, 100.0)
    dth, dr = 2 * np.pi / nth, 1.0 / n
    th = (np.arange(1, nth + 1) - 0.5) * dth
    rm = (np.arange(1, n + 1) - 0.5) * dr
    T, R, Z = np.meshgrid(th, rm, rm, indexing="ij")
    run.set("rhs", np.asfortranarray(rhs_ex(T, R, Z)))
    run.laplace_solve()
    ph = run.get("dph")[:, 1:n + 1, 1:n + 1]
    run.close()
    return float(np.abs(ph - sol_ex(T, R, Z)).max())


def test_poisson_manufactured_solution_on_gpu():
    from oracle import oracle as O
    th_orc = O.Oracle(13, 8, 8, 1.0, 1.0, 1e-3, 100.0).mesh("thm")[1:14]
    assert np.allclose(th_orc, (np.arange(1, 14) - 0.5) * 2 * np.pi / 13)
    e = [_mms_gpu(n) for n in (16, 32, 64, 128)]
    print("manufactured solution, max error per grid:", e)
    assert e[2] < 2e-5
    for a, b in zip(e, e[1:]):
        assert 3.7 < a / b < 4.3, e
