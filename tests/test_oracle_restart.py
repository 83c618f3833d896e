"""The oracle's restart files (run.F90:390-539) against the byte layout of
gfortran unformatted sequential I/O that the reference's `write (22)` /
`read (22)` produce: every record framed by its 4-byte little-endian length,
a header record (nstep int32, ntime real64, ntheta, nr, nz int32), then one
(q1, q2, q3) record per interior cell, theta fastest, then r, then z."""
import struct

import numpy as np


def _seed(o, seed):
    rng = np.random.default_rng(seed)
    for n in ("q1", "q2", "q3"):
        a = o.field(n)
        a[...] = rng.uniform(-1, 1, a.shape)


def test_restart_file_is_gfortran_sequential(oracle_mod, tmp_path):
    O = oracle_mod
    nth, nr, nz = 3, 4, 5
    o = O.Oracle(nth, nr, nz, 4.0, 12.0, 1e-3, 1000.0)
    _seed(o, 1)
    o.set_clock(2, 0.125, 37)
    path = tmp_path / "restart00037RK02.dat"
    assert o.restart_save(path) == 0
    rec = lambda b: struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))
    want = rec(struct.pack("<idiii", 37, 0.125, nth, nr, nz))
    q1, q2, q3 = o.field("q1"), o.field("q2"), o.field("q3")
    for iz in range(1, nz + 1):
        for ir in range(1, nr + 1):
            for ith in range(nth):
                want += rec(struct.pack("<ddd", q1[ith, ir, iz], q2[ith, ir, iz], q3[ith, ir, iz]))
    assert path.read_bytes() == want


def test_restart_round_trip_and_grid_check(oracle_mod, tmp_path):
    O = oracle_mod
    a = O.Oracle(6, 8, 10, 4.0, 12.0, 1e-3, 1000.0)
    _seed(a, 2)
    a.set_clock(1, 0.75, 12)
    path = tmp_path / "RESTART"
    assert a.restart_save(path) == 0
    b = O.Oracle(6, 8, 10, 4.0, 12.0, 1e-3, 1000.0)
    assert b.restart_load(path) == 0
    for n in ("q1", "q2", "q3"):
        np.testing.assert_array_equal(b.field(n)[:, 1:9, 1:11], a.field(n)[:, 1:9, 1:11])
    assert b.clock[1:] == (0.75, 12)
    c = O.Oracle(6, 8, 12, 4.0, 12.0, 1e-3, 1000.0)
    assert c.restart_load(path) == -2
