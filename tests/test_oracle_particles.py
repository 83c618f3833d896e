"""CPU checks of the particle bookkeeping in the oracle: the splitmix64
stream used in place of Fortran random_number against an independent Python
statement of the published algorithm, and inlt_part (part_tools.F90:95-142)
conservation: every unit of accumulated inflow becomes one particle placed in
its entry cell, with the fractional remainder kept per radial row."""
import numpy as np

MASK = (1 << 64) - 1


def splitmix64_uniform(state):
    state = (state + 0x9E3779B97F4A7C15) & MASK
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    z = z ^ (z >> 31)
    return (z >> 11) * (1.0 / 9007199254740992.0), state


def test_rng_is_splitmix64(oracle_mod):
    import ctypes as C
    L = oracle_mod.lib()
    st = C.c_uint64(12345)
    ps = 12345
    for _ in range(1000):
        a = L.orc_rng_uniform(C.byref(st))
        b, ps = splitmix64_uniform(ps)
        assert a == b
    assert st.value == ps


def test_inlt_part_conserves_inflow(oracle_mod):
    O = oracle_mod
    nth, nr, nz, rmax, zmax, dt = 16, 32, 32, 4.0, 12.0, 0.002
    o = O.Oracle(nth, nr, nz, rmax, zmax, dt, 1000.0)
    rng = np.random.default_rng(4)
    q3 = o.field("q3")
    q3[:, :, 1] = rng.uniform(0.5, 2.0, size=q3[:, :, 1].shape)
    p = O.OraclePart(o, 3, 20000, 0)
    rc, thc, r0 = o.mesh("rc"), o.mesh("thc"), 0.6
    dth, dr, dz = 2 * np.pi / nth, rmax / nr, zmax / nz
    c = p.c
    flux = np.zeros(nr + 2)
    state, total = 99, 0
    for call in range(3):
        n0 = p.nlast
        n, state = p.inlt(r0, state)
        assert n > 0
        total += n
        u, v = p.u, p.v
        for ip in range(n0, p.nlast):
            x, y, z = u[ip, 0], u[ip, 1], u[ip, 2]
            r = np.hypot(x, y)
            assert 0.0 <= z <= dz and r < r0 + dr
            th = np.arctan2(y, x) % (2 * np.pi)
            ir, it = int(r // dr) + 1, int(th // dth) + 1
            edge = min(abs(th / dth - round(th / dth)), abs(r / dr - round(r / dr))) < 1e-9
            # w is the entry cell's axial velocity (uz = q3(it, ir, 1))
            assert edge or u[ip, 5] == q3[it - 1, ir, 1]
            assert v[ip, 1] == c and v[ip, 2] == float(np.float32(ip + 1))
        for ir in range(1, nr + 1):
            if rc[ir] < r0:
                a = dth * (rc[ir + 1] ** 2 - rc[ir] ** 2)
                flux[ir] += sum(c * a * q3[it, ir, 1] * dt * 10.0 / np.float64(np.float32(0.001))
                                for it in range(nth))
    assert p.npart == total
    np.testing.assert_allclose(total + p.inflow[1:nr + 1].sum(), flux.sum(), rtol=1e-12)
    assert np.all((p.inflow >= 0) & (p.inflow < 1))
