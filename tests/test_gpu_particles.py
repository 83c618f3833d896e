"""GPU particles (part_tools.F90) against the oracle, through the C ABI.

- the reference's dertest known answers (u_theta = 0, u_r = r^2, u_z = 1 on
  the dertest r-z mesh) interpolated by the CUDA kernel;
- interpolation/transform at random points of a vortex-ring field: cell
  indices bit-exact, values to 1e-12;
- iter_part (inertial and tracer classes) over several calls, with particles
  leaving the domain: state arrays, free list and counters;
- injc_part / remv_part slot bookkeeping;
- particles attached to vr_iterate, advanced before substep 1 of every step.
"""
import os

import numpy as np
import pytest

from tests.parity_util import make_pair

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "dertest_kat.npz")


def _ring(orc, gpu, nth, nr, nz, seed=0):
    from vring_b200.synthetic import ring_fields
    q1, q2, q3 = ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=seed)
    for n, a in (("q1", q1), ("q2", q2), ("q3", q3)):
        orc.field(n)[...] = a
        gpu.set(n, a)


def test_dertest_kat_on_gpu():
    """The dertest dumps (8 significant digits) through the CUDA kernel. The
    dumps come from an axisymmetric run (ntheta = 1); the field is independent
    of theta, so the same answers hold on an 8-cell theta mesh."""
    import vring_b200 as V
    g = np.load(GOLD)
    _, nr, nz, rmax, zmax = g["mesh"]
    run = V.Run(8, int(nr), int(nz), float(rmax), float(zmax), 1e-3, 1000.0)
    ext = run.extents("q2")
    dr = float(rmax) / int(nr)
    rc = (np.arange(ext[1]) - 1.0) * dr
    q2 = np.broadcast_to((rc ** 3)[None, :, None], ext[:3])
    run.set("q1", 0.0)
    run.set("q2", q2)
    run.set("q3", 1.0)
    p = V.Part(run, 1, 4, 0)
    vel, dvel, dd, _ = p.probe(g["pos"])
    got = np.concatenate([vel, dvel.reshape(-1, 9, order="F"), dd[:, 0].reshape(-1, 9, order="F"),
                          dd[:, 1].reshape(-1, 9, order="F"), dd[:, 2].reshape(-1, 9, order="F")], 1)
    ref = np.concatenate([g["vel"], g["dvel"], g["ddvel1"], g["ddvel2"], g["ddvel3"]], 1)
    np.testing.assert_allclose(got, ref, rtol=2e-7, atol=2e-13)
    p.close()


@pytest.mark.parametrize("grid", [(16, 16, 32), (12, 24, 40)])
def test_probe_matches_oracle(grid):
    from oracle import oracle as O
    import vring_b200 as V
    nth, nr, nz = grid
    orc, gpu = make_pair(nth, nr, nz)
    _ring(orc, gpu, nth, nr, nz, seed=3)
    op = O.OraclePart(orc, 3, 8, 0)
    gp = V.Part(gpu, 3, 8, 0)
    rng = np.random.default_rng(7)
    n = 600
    r = rng.uniform(0.02, 3.98, n)
    th = rng.uniform(0, 2 * np.pi, n)
    z = rng.uniform(0.01, 11.99, n)
    xyz = np.stack([r * np.cos(th), r * np.sin(th), z], 1)
    # points on cell faces and the theta = 0 / pi seams
    dr, dz = 4.0 / nr, 12.0 / nz
    extra = np.array([[dr * 5, 0.0, dz * 7], [-dr * 3, 0.0, dz * 2], [0.0, dr * 4, dz * 3],
                      [0.0, -dr * 4, dz * 3], [dr * 2, -1e-13, 6.0], [1e-3, 1e-3, 0.5]])
    xyz = np.concatenate([xyz, extra])
    vel, dvel, dd, cells = gp.probe(xyz)
    for i, pt in enumerate(xyz):
        idx, _ = op.cell(*pt)
        assert tuple(cells[i]) == tuple(idx), (i, pt, cells[i], idx)
        ref = op.probe(*pt)
        got = np.concatenate([vel[i], dvel[i].reshape(-1, order="F"), dd[i].reshape(-1, order="F")])
        scale = max(np.abs(ref).max(), 1e-30)
        err = np.abs(got - ref).max()
        assert err <= 1e-12 * scale, (i, pt, err / scale)
    gp.close()


def _inject_cloud(ps, n, seed, out_frac=0.1):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.3, 3.6, n)
    th = rng.uniform(0, 2 * np.pi, n)
    z = rng.uniform(0.5, 11.5, n)
    w = rng.uniform(-0.5, 0.5, n)
    nout = int(out_frac * n)
    z[:nout] = 11.97          # inertial: these leave through z = zmax within a step
    w[:nout] = 40.0
    r[nout:2 * nout] = 4.0005  # start just beyond r = rmax: removed after one substep
    slots = []
    for i in range(n):
        s = [p.injc(r[i] * np.cos(th[i]), r[i] * np.sin(th[i]), z[i], 0.1, -0.1, w[i]) for p in ps]
        assert s[0] == s[1]
        slots.append(s[0])
    return slots


def _compare_parts(op, gp, rel=1e-11):
    u, v, isf, cnt = gp.state()
    assert cnt == {"npart": op.npart, "nlast": op.nlast, "nfree": op.nfree, "nids": op.nids}
    ou, ov = op.u, op.v
    assert np.array_equal(isf[:op.nlast] != 0, op.isfre[1:op.nlast + 1] != 0)
    scale = np.maximum(np.abs(ou).max(axis=0), 1e-30)
    err = (np.abs(u - ou) / scale).max()
    assert err <= rel, err
    np.testing.assert_array_equal(v, ov)


@pytest.mark.parametrize("pid,mode", [(4, 0), (8, 0), (6, 1)])
def test_iter_part_matches_oracle(pid, mode):
    from oracle import oracle as O
    import vring_b200 as V
    nth, nr, nz = 16, 32, 64
    orc, gpu = make_pair(nth, nr, nz, dt=1e-3)
    _ring(orc, gpu, nth, nr, nz, seed=5)
    naloc = 700
    op = O.OraclePart(orc, pid, naloc, mode)
    gp = V.Part(gpu, pid, naloc, mode)
    assert (gp.nsubdt, gp.st, gp.r, gp.c) == (op.nsubdt, op.st, op.r, op.c)
    _inject_cloud([op, gp], 600, seed=pid)
    for call in range(3):
        op.iter_part(1)
        gp.iter_part(1)
        _compare_parts(op, gp)
    assert op.npart < 600          # the fast particles left through z = zmax
    # refill freed slots after removals
    _inject_cloud([op, gp], 50, seed=11, out_frac=0.0)
    op.iter_part(1)
    gp.iter_part(1)
    _compare_parts(op, gp)
    gp.close()


@pytest.mark.parametrize("scale,mode", [(3e4, 1), (1e8, 0), (1e8, 1)])
def test_iter_part_full_iteration_matches_oracle(scale, mode):
    # Velocities scaled until the stencil differences pass the bound below
    # which the fit's second pass is rounding noise: the reference then runs
    # its Richardson iteration for several passes (up to 100).  At 3e4 part of
    # the particles cross the bound, at 1e8 all of them: the main launch
    # defers them and the full-iteration launch advances them.
    from oracle import oracle as O
    import vring_b200 as V
    nth, nr, nz = 16, 32, 64
    orc, gpu = make_pair(nth, nr, nz, dt=1e-2 / scale)
    from vring_b200.synthetic import ring_fields
    for n, a in zip(("q1", "q2", "q3"), ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=6)):
        orc.field(n)[...] = scale * a
        gpu.set(n, scale * a)
    op = O.OraclePart(orc, 6, 700, mode)
    gp = V.Part(gpu, 6, 700, mode)
    _inject_cloud([op, gp], 600, seed=13, out_frac=0.0)
    u0 = gp.state()[0].copy()
    for call in range(2):
        op.iter_part(1)
        gp.iter_part(1)
        _compare_parts(op, gp)
    moved = np.abs(gp.state()[0][:600, 0:3] - u0[:600, 0:3]).max(axis=1)
    assert (moved > 0).all()  # every particle was advanced
    gp.close()


def test_inject_remove_bookkeeping():
    from oracle import oracle as O
    import vring_b200 as V
    orc, gpu = make_pair(8, 16, 32)
    op = O.OraclePart(orc, 2, 12, 0)
    gp = V.Part(gpu, 2, 12, 0)
    seq = [("i", 1.0), ("i", 1.1), ("i", 1.2), ("i", 1.3), ("r", 2), ("r", 4), ("i", 1.4),
           ("r", 1), ("i", 1.5), ("i", 1.6), ("r", 3), ("r", 2), ("i", 1.7), ("i", 1.8)]
    for op_, a in seq:
        if op_ == "i":
            s0 = op.injc(a, 0.5, 2.0, 0.1, 0.2, 0.3, icall=1)
            s1 = gp.injc(a, 0.5, 2.0, 0.1, 0.2, 0.3, icall=1)
            assert s0 == s1
        else:
            op.remv(a)
            gp.remv(a)
        _compare_parts(op, gp, rel=0.0)
    # capacity: the GPU refuses the slot past naloc
    while gp.counts["nlast"] < 12 or gp.counts["nfree"] > 0:
        gp.injc(1.0, 1.0, 1.0)
    with pytest.raises(V.VrError) as e:
        gp.injc(1.0, 1.0, 1.0)
    assert e.value.code == 9
    gp.close()


def test_iterate_with_attached_particles():
    from oracle import oracle as O
    import vring_b200 as V
    nth, nr, nz = 16, 32, 64
    orc, gpu = make_pair(nth, nr, nz, dt=1e-3, wth="modified")
    _ring(orc, gpu, nth, nr, nz, seed=9)
    op = O.OraclePart(orc, 5, 300, 0)
    gp = V.Part(gpu, 5, 300, 0)
    _inject_cloud([op, gp], 250, seed=2)
    gp.attach(True)
    gpu.iterate(3)
    for _ in range(3):      # loop.F90:65-68: iter_part, then the three substeps
        op.iter_part(1)
        orc.iterate(1)
    _compare_parts(op, gp, rel=1e-10)
    for n in ("q1", "q2", "q3"):
        g, r = gpu.get(n), orc.field(n)
        assert np.abs(g - r).max() <= 1e-10 * np.abs(r).max()
    gp.attach(False)
    gp.close()


def test_context_refuses_destroy_with_live_particles():
    import vring_b200 as V
    from vring_b200.api import lib
    run = V.Run(8, 16, 32, 4.0, 12.0, 1e-3, 1000.0)
    p = V.Part(run, 1, 4, 0)
    assert lib().vr_destroy(run._h) == 7
    p.close()
    run.close()
    assert not run._h


def _south_inflow(orc, gpu, seed):
    rng = np.random.default_rng(seed)
    q3 = orc.field("q3")
    q3[:, :, 1] = rng.uniform(0.5, 2.0, size=q3[:, :, 1].shape)
    gpu.set("q3", q3)


def test_inlt_part_matches_oracle():
    """inlt_part: same slots, positions, velocities, ids and random stream."""
    from oracle import oracle as O
    import vring_b200 as V
    nth, nr, nz = 16, 32, 32
    orc, gpu = make_pair(nth, nr, nz, dt=0.002)
    _south_inflow(orc, gpu, 4)
    op = O.OraclePart(orc, 3, 20000, 0)
    gp = V.Part(gpu, 3, 20000, 0)
    so, sg = 77, 77
    for call in range(3):
        no, so = op.inlt(0.6, so)
        ng, sg = gp.inlt(0.6, sg)
        assert (no, so) == (ng, sg) and no > 0
        _compare_parts(op, gp, rel=1e-15)
    # removals in between, then refill through the free list
    for ip in (3, 10, 11, op.nlast):
        op.remv(ip)
        gp.remv(ip)
    no, so = op.inlt(0.6, so)
    ng, sg = gp.inlt(0.6, sg)
    assert (no, so) == (ng, sg)
    _compare_parts(op, gp, rel=1e-15)
    gp.close()


def test_iterate_with_inflow_injection():
    """vr_iterate with inflow on: inlt_part at nstep = 0, 10, 20 (loop.F90:54-58),
    then iter_part, then the three substeps, against the same loop on the oracle."""
    from oracle import oracle as O
    import vring_b200 as V
    nth, nr, nz = 16, 32, 64
    orc, gpu = make_pair(nth, nr, nz, dt=1e-3, wth="modified")
    _ring(orc, gpu, nth, nr, nz, seed=9)
    _south_inflow(orc, gpu, 5)
    op = O.OraclePart(orc, 6, 4000, 1)
    gp = V.Part(gpu, 6, 4000, 1)
    gp.set_inflow(0.6, 2024, True)
    gp.attach(True)
    gpu.iterate(21)
    so = 2024
    for step in range(21):
        if step % 10 == 0:
            _, so = op.inlt(0.6, so)
        op.iter_part(1)
        orc.iterate(1)
    assert op.nlast > 0
    _compare_parts(op, gp, rel=1e-10)
    gp.attach(False)
    gp.close()


def _fortran_e(x, w=20, d=8):
    """Ew.d as gfortran writes it (independent of the library's formatter)."""
    if x == 0:
        s = "0." + "0" * d + "E+00"
    else:
        m, e = ("%.*E" % (d - 1, abs(x))).split("E")
        e = int(e) + 1
        s = "0." + m.replace(".", "") + ("E%+03d" % e if abs(e) <= 99 else "%+04d" % e)
    if x < 0:
        s = "-" + s
    return s.rjust(w)


def test_part_dump_layout(tmp_path):
    """part_tools.F90:444-491: the part file's header lines, one (200(E20.8))
    line per live particle with d(1) = det of the Jacobian, and the trajectory
    file with the particles whose id is 1 modulo 1000."""
    import vring_b200 as V
    gpu = V.Run(8, 16, 32, 4.0, 12.0, 1e-3, 1000.0, 1.0, 1.0)
    naloc = 1300
    p = V.Part(gpu, 3, naloc, 0)
    rng = np.random.default_rng(8)
    u = np.asfortranarray(rng.uniform(-2, 2, (naloc, 117)))
    v = np.zeros((naloc, 3), order="F")
    v[:, 1] = p.c
    v[:, 2] = np.arange(1, naloc + 1)
    isf = np.zeros(naloc, dtype=np.int32)
    isf[[5, 600, 999]] = 1           # free slots: not written
    p.set_state(u, v, isf, 1250)
    p.dump(tmp_path)
    lines = (tmp_path / "part00000size03.dat").read_text().split("\n")
    assert lines[0] == ('title = "particles diameter: '.rjust(32) + _fortran_e(p.r) + " stokes: ".rjust(12)
                        + _fortran_e(p.st) + '"'.rjust(2))
    assert lines[1] == ('variables = "id", "time", "c",'.rjust(32) + "".join("   u%03d" % i for i in range(1, 118))
                        + "".join("   d%03d" % i for i in range(1, 11)))
    live = [ip for ip in range(1250) if isf[ip] == 0]
    body = [l for l in lines[2:] if l]
    assert len(body) == len(live)

    def det(ip):
        J = u[ip, 6:15].reshape(3, 3, order="F")
        return np.linalg.det(J)

    for l, ip in zip(body[::97], live[::97]):
        vals = np.array([float(l[20 * i:20 * (i + 1)]) for i in range(130)])
        np.testing.assert_allclose(vals[:3], v[ip], rtol=1e-7, atol=0)
        np.testing.assert_allclose(vals[3:120], u[ip], rtol=1e-7, atol=1e-300)
        np.testing.assert_allclose(vals[120], det(ip), rtol=1e-7)
        assert np.all(vals[121:] == 0)
    traj = (tmp_path / "trajectory_size03.dat").read_text().split("\n")
    ids = [float(l[40:60]) for l in traj if l]
    assert ids == [1.0, 1001.0]      # id 1 mod 1000, in slot order
    last_d = float(body[-1][20 * 120:20 * 121])
    assert all(float(l[20 * 120:20 * 121]) == last_d for l in traj if l)   # the dump loop's last d
    assert traj[-2] == "" and traj[-1] == ""
    p.close()


def test_iterate_writes_dumps_every_expstp(tmp_path):
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    gpu = V.Run(8, 16, 32, 4.0, 12.0, 1e-3, 1000.0, 1.0, 1.0)
    for n, a in zip(("q1", "q2", "q3"), ring_fields(8, 16, 32, 4.0, 12.0, seed=1)):
        gpu.set(n, a)
    p = V.Part(gpu, 2, 50, 1)
    for i in range(10):
        p.injc(1.0 + 0.01 * i, 0.2, 3.0)
    p.set_dump(2, tmp_path)
    p.attach(True)
    gpu.iterate(5)
    names = sorted(f.name for f in tmp_path.iterdir())
    assert names == ["part00000size02.dat", "part00002size02.dat", "part00004size02.dat",
                     "trajectory_size02.dat"]
    p.attach(False)
    p.close()


def _cloud_state(naloc, n, seed, vel_scale=1.0):
    """u (naloc, 117) with n particles at random points of the ring domain,
    some of them fast enough to leave it; v = 0."""
    rng = np.random.default_rng(seed)
    u = np.zeros((naloc, 117))
    r = rng.uniform(0.05, 3.95, n)
    r[n // 100:n // 50] = 4.0005  # just beyond r = rmax: removed after one substep
    th = rng.uniform(0, 2 * np.pi, n)
    u[:n, 0], u[:n, 1], u[:n, 2] = r * np.cos(th), r * np.sin(th), rng.uniform(0.05, 11.95, n)
    u[:n, 3:6] = vel_scale * rng.uniform(-0.5, 0.5, (n, 3))
    u[:n // 100, 2] = 11.97
    u[:n // 100, 5] = 60.0 * vel_scale  # inertial: these leave through z = zmax
    return u, np.zeros((naloc, 3))


@pytest.mark.parametrize("mode,scale", [(1, 1.0), (0, 1.0), (1, 3e4)])
def test_walk_order_changes_no_result(mode, scale):
    # The main launch walks the slots grouped by cell bucket (order 1) or in
    # slot order (order 0): every particle's update reads only its own state,
    # so both must leave the same bits.  Covers removals, slots injected above
    # the sorted range and, at the scaled velocity, blocks that defer to the
    # full-iteration launch after carrying positions through some substeps.
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 32, 64, 128
    naloc, n = 40000, 30000
    runs, parts = [], []
    for order in (0, 1):
        gpu = V.Run(nth, nr, nz, 4.0, 12.0, 1e-3 / scale, 1000.0, 1.0, 1.0)
        for nm, a in zip(("q1", "q2", "q3"), ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=3)):
            gpu.set(nm, scale * a)
        gp = V.Part(gpu, 6, naloc, mode)
        gp.set_order(order)
        u, v = _cloud_state(naloc, n, seed=21, vel_scale=scale)
        gp.set_state(u, v, nlast=n)
        runs.append(gpu)
        parts.append(gp)
    for call in range(4):
        for gp in parts:
            gp.iter_part(1)
        if call == 1:
            rng = np.random.default_rng(5)
            pts = rng.uniform(0.5, 2.5, (1000, 3))
            for gp in parts:  # free slots first, then slots above nlast
                for x, y, z in pts:
                    gp.injc(x, y, z, 0.1, -0.1, 0.2)
        sa, sb = parts[0].state(), parts[1].state()
        assert sa[3] == sb[3]
        np.testing.assert_array_equal(sa[2], sb[2])
        np.testing.assert_array_equal(sa[0], sb[0])
        np.testing.assert_array_equal(sa[1], sb[1])
    assert sa[3]["npart"] < n + 1000  # some left the domain
    assert sa[3]["nlast"] > n  # and some injections went above the first nlast
    for gp in parts:
        gp.close()
