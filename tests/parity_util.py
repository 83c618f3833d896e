"""Helpers shared by the GPU parity tests: one oracle run and one GPU run on
the same grid, the same seeded state, and field-by-field comparison."""
import numpy as np

STATE = ["q1", "q2", "q3", "dq1", "dq2", "dq3", "ru1", "ru2", "ru3", "pres", "prg", "csort",
         "dq3no"]


def make_pair(nth, nr, nz, rmax=4.0, zmax=12.0, dt=2e-3, re=1000.0, slip=1.0, wth="exact",
              inflow="off"):
    from oracle import oracle as O
    import vring_b200 as V
    wm = {"exact": 0, "modified": 1}[wth]
    im = {"off": 0, "reference": 1}[inflow]
    orc = O.Oracle(nth, nr, nz, rmax, zmax, dt, re, 1.0, slip, wm, im)
    gpu = V.Run(nth, nr, nz, rmax, zmax, dt, re, 1.0, slip, theta_wavenumber=wth, inflow=inflow)
    return orc, gpu


def seed_random(orc, gpu, names, seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    for n in names:
        a = orc.field(n)
        a[...] = scale * rng.uniform(-1.0, 1.0, size=a.shape)
        gpu.set(n, a)


def copy_to_gpu(orc, gpu, names):
    for n in names:
        gpu.set(n, orc.field(n))


def assert_field_close(gpu, orc, name, rel=1e-12, floor=1e-300):
    g = gpu.get(name)
    r = orc.field(name)
    assert g.shape == r.shape, (name, g.shape, r.shape)
    scale = max(np.abs(r).max(), floor)
    d = np.abs(g - r)
    err = d.max()
    where = np.unravel_index(np.argmax(d), d.shape)
    assert err <= rel * scale, "%s: max |gpu - oracle| = %.3e at %s, scale %.3e (rel %.2e)" % (
        name, err, where, scale, err / scale)
    return err / scale


def prep(orc, gpu, irk=1, ntime=0.0, nstep=0):
    """Set the clock and build the substep's coefficients on both sides
    (loop.F90:71-74 calls ucoeff and coesys before every substep)."""
    for o in (orc, gpu):
        o.set_clock(irk, ntime, nstep)
        o.ucoeff()
        o.coesys()
