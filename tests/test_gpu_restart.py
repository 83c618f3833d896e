"""Restart files through the C ABI: the library writes the reference's
restart file byte for byte as the oracle does (run.F90:390-460), reads the
oracle's, refuses a different grid, and with the full-state extension a
resumed run -- fields and particles -- continues bit for bit."""
import numpy as np
import pytest

from tests.parity_util import make_pair

pytestmark = pytest.mark.gpu


def _ring(orc, gpu, nth, nr, nz, seed):
    from vring_b200.synthetic import ring_fields
    for n, a in zip(("q1", "q2", "q3"), ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=seed)):
        orc.field(n)[...] = a
        gpu.set(n, a)


def test_restart_file_matches_oracle_bytes(tmp_path):
    nth, nr, nz = 12, 16, 24
    orc, gpu = make_pair(nth, nr, nz)
    _ring(orc, gpu, nth, nr, nz, 3)
    orc.set_clock(3, 0.0421, 42)
    gpu.set_clock(3, 0.0421, 42)
    a, b = tmp_path / "gpu.dat", tmp_path / "orc.dat"
    gpu.restart_save(a)
    assert orc.restart_save(b) == 0
    assert a.read_bytes() == b.read_bytes()


def test_library_reads_oracle_restart(tmp_path):
    import vring_b200 as V
    nth, nr, nz = 12, 16, 24
    orc, gpu = make_pair(nth, nr, nz)
    _ring(orc, gpu, nth, nr, nz, 4)
    orc.set_clock(1, 1.5, 300)
    path = tmp_path / "RESTART"
    assert orc.restart_save(path) == 0
    fresh = V.Run(nth, nr, nz, 4.0, 12.0, 2e-3, 1000.0, 1.0, 1.0)
    assert fresh.restart_load(path) is False
    for n in ("q1", "q2", "q3"):
        np.testing.assert_array_equal(fresh.get(n)[:, 1:nr + 1, 1:nz + 1], orc.field(n)[:, 1:nr + 1, 1:nz + 1])
    assert fresh.clock[1:] == (1.5, 300)
    other = V.Run(nth, nr, nz + 8, 4.0, 12.0, 2e-3, 1000.0, 1.0, 1.0)
    with pytest.raises(V.VrError) as e:
        other.restart_load(path)
    assert e.value.code == 6


def test_full_restart_resumes_bit_for_bit(tmp_path):
    import vring_b200 as V
    from vring_b200.synthetic import annulus_particles
    nth, nr, nz = 16, 32, 64
    args = (nth, nr, nz, 4.0, 12.0, 1e-3, 1000.0, 1.0, 1.0)
    a = V.Run(*args, theta_wavenumber="modified")
    from vring_b200.synthetic import ring_fields
    for n, q in zip(("q1", "q2", "q3"), ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=5)):
        a.set(n, q)
    pa = V.Part(a, 4, 500, 0)
    x, y, z = annulus_particles(400, 0.5, 1.5, 2.0, 4.0, seed=1)
    for i in range(400):
        pa.injc(x[i], y[i], z[i])
    pa.attach(True)
    a.iterate(3)
    a.restart_save(tmp_path / "full.dat", full=True)
    pa.restart_save(tmp_path / "part.dat")
    a.iterate(2)
    b = V.Run(*args, theta_wavenumber="modified")
    pb = V.Part(b, 4, 500, 0)
    assert b.restart_load(tmp_path / "full.dat") is True
    pb.restart_load(tmp_path / "part.dat")
    pb.attach(True)
    assert b.clock[2] == 3
    b.iterate(2)
    assert a.clock == b.clock
    for n in ("q1", "q2", "q3", "pres", "prg", "ru1", "ru2", "ru3", "dq3no", "csort"):
        np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)
    ua, va, ia, ca = pa.state()
    ub, vb, ib, cb = pb.state()
    assert ca == cb
    np.testing.assert_array_equal(ua, ub)
    np.testing.assert_array_equal(va, vb)
    np.testing.assert_array_equal(ia, ib)
    pa.close()
    pb.close()
