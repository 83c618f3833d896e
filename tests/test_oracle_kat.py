"""The CPU restatement against the reference's known answers.

- particle interpolation + cylindrical->Cartesian transform against the
  reference's dertest dumps (tests/golden/dertest_kat.npz, made by
  tests/golden/make_golden.py from dertest/VR2D/fort.3000-3233);
- the Poisson solve against the reference's manufactured solution
  (solp_tools.F90:95-126), second-order convergence;
- the FFTW transform definitions (fastfouriertransform.F90) against scipy.fft;
- the tridiagonal solvers (tripar.F90, step.F90:487-534, btrithom.F90)
  against dense solves;
- the acos used for cell indices against libm.
"""
import os

import numpy as np
import pytest
import scipy.fft as sf

GOLD = os.path.join(os.path.dirname(__file__), "golden", "dertest_kat.npz")


def test_dertest_interpolation_kat(oracle_mod):
    O = oracle_mod
    g = np.load(GOLD)
    nth, nr, nz, rmax, zmax = g["mesh"]
    orc = O.Oracle(int(nth), int(nr), int(nz), rmax, zmax, 1e-3, 1000.0)
    rc = orc.mesh("rc")
    q2 = orc.field("q2")
    for j in range(q2.shape[1]):
        q2[:, j, :] = rc[j] ** 3          # q2 / rc = u_r = r**2
    orc.field("q3")[:] = 1.0              # u_z = 1, u_theta = 0
    p = O.OraclePart(orc, 1, 4, 0)
    for n, xyz in enumerate(g["pos"]):
        out = p.probe(*xyz)
        dvel = out[3:12].reshape(3, 3, order="F")
        dd = out[12:].reshape(3, 3, 3, order="F")
        got = np.concatenate([out[:3], dvel.reshape(-1), dd[0].reshape(-1), dd[1].reshape(-1),
                              dd[2].reshape(-1)])
        ref = np.concatenate([g["vel"][n], g["dvel"][n], g["ddvel1"][n], g["ddvel2"][n],
                              g["ddvel3"][n]])
        # the dumps carry 8 significant digits (E20.8)
        np.testing.assert_allclose(got, ref, rtol=2e-7, atol=2e-13)


def _mms(O, n, wth_mode=0, nth=13):
    pi = np.float64(np.float32(4 * np.arctan(np.float32(1))))   # pi = 4.0*atan(1.0), real*4

    def sol_ex(th, rr, zz):
        return np.cos(2 * pi * zz) / (4 * pi ** 2) * (rr ** 3 - 1.5 * rr ** 2) * (1 - 0.5 * np.cos(5 * th))

    def rhs_ex(th, rr, zz):
        return (np.cos(2 * pi * zz) * (rr ** 3 - 1.5 * rr ** 2) * (1 - 0.5 * np.cos(5 * th))
                + np.cos(2 * pi * zz) * (6 - 9 * rr) / (4 * pi ** 2) * (1 - 0.5 * np.cos(5 * th))
                + np.cos(2 * pi * zz) / (4 * pi ** 2) * (rr ** 3 - 1.5 * rr ** 2)
                * (-0.5 * 25 * np.cos(5 * th)) / rr ** 2)

    o = O.Oracle(nth, n, n, 1.0, 1.0, 1e-3, 100.0, wth_mode=wth_mode)
    th = o.mesh("thm")[1:nth + 1]
    rm = o.mesh("rm")[1:n + 1]
    zm = o.mesh("zm")[1:n + 1]
    T, R, Z = np.meshgrid(th, rm, zm, indexing="ij")
    o.field("rhs")[:] = rhs_ex(T, R, Z)
    o.laplace_solve()
    ph = o.field("dph")[:, 1:n + 1, 1:n + 1]
    return np.abs(ph - sol_ex(T, R, Z)).max()


def test_poisson_manufactured_solution_second_order(oracle_mod):
    e = [_mms(oracle_mod, n) for n in (16, 32, 64)]
    assert e[-1] < 2e-5
    for a, b in zip(e, e[1:]):
        assert 3.7 < a / b < 4.3


@pytest.mark.parametrize("n", [8, 9, 33, 128])
def test_packed_real_fft_matches_fftw_definition(oracle_mod, n):
    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, 7))
    p = oracle_mod.fft_ptf(a)
    F = sf.rfft(a, axis=0)
    ref = np.zeros_like(a)
    ref[0] = F[0].real / n
    for k in range(1, n // 2 + 1):
        ref[2 * k - 1] = 2 * F[k].real / n
        if 2 * k < n:
            ref[2 * k] = -2 * F[k].imag / n
    np.testing.assert_allclose(p, ref, atol=1e-14)
    np.testing.assert_allclose(oracle_mod.fft_ftp(p), a, atol=1e-13)


@pytest.mark.parametrize("nz", [8, 12, 64, 512])
def test_dct_matches_redft10_redft01(oracle_mod, nz):
    rng = np.random.default_rng(nz)
    a = rng.normal(size=(5, nz))
    d = oracle_mod.fft_cos(a, 1)
    np.testing.assert_allclose(d, sf.dct(a, type=2, axis=1) / (2 * nz), atol=1e-15)
    i = oracle_mod.fft_cos(d, -1)
    np.testing.assert_allclose(i, sf.dct(d, type=3, axis=1), atol=1e-14)
    np.testing.assert_allclose(i, a, atol=1e-13)


def test_thomas_and_periodic_solvers(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(1)
    n = 40
    a, c = rng.uniform(-1, 0, n), rng.uniform(-1, 0, n)
    b, r = 3 + rng.uniform(0, 1, n), rng.normal(size=n)
    A = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
    np.testing.assert_allclose(A @ O.solve_lap_thom(r, a, b, c), r, atol=1e-14)
    np.testing.assert_allclose(A @ O.solve_lap_par(r, a, b, c), r, atol=1e-14)
    nj, ni = 5, 11
    ami, api = rng.uniform(-1, 0, (nj, ni)), rng.uniform(-1, 0, (nj, ni))
    aci, fi = 3 + rng.uniform(0, 1, (nj, ni)), rng.normal(size=(nj, ni))
    X = O.tripij(ami, aci, api, fi)
    for j in range(nj):
        M = np.diag(aci[j])
        for i in range(ni):
            M[i, (i - 1) % ni] += ami[j, i]
            M[i, (i + 1) % ni] += api[j, i]
        np.testing.assert_allclose(M @ X[j], fi[j], atol=1e-14)


def test_block_thomas_identity_coupling(oracle_mod):
    rng = np.random.default_rng(2)
    m, n = 4, 6
    b1, b3 = rng.uniform(-1, 0, m * n), rng.uniform(-1, 0, m * n)
    b2, r = 6 + rng.uniform(0, 1, m * n), rng.normal(size=m * n)
    x = oracle_mod.solve_lap_bthom(r, b1, b2, b3, m, n)
    A = np.zeros((m * n, m * n))
    for k in range(n):
        o = k * m
        for l in range(m):
            A[o + l, o + l] = b2[o + l]
            if l > 0:
                A[o + l, o + l - 1] = b1[o + l]
            if l < m - 1:
                A[o + l, o + l + 1] = b3[o + l]
        if k > 0:
            A[o:o + m, o - m:o] += np.eye(m)
        if k < n - 1:
            A[o:o + m, o + m:o + 2 * m] += np.eye(m)
    np.testing.assert_allclose(A @ x, r, atol=1e-12)


def test_vr_acos_within_one_ulp_of_libm(oracle_mod):
    rng = np.random.default_rng(3)
    xs = np.concatenate([np.linspace(-1, 1, 20001), rng.uniform(-1, 1, 20000), [-1.0, 1.0, 0.0]])
    got = np.array([oracle_mod.vr_acos(x) for x in xs])
    ref = np.arccos(xs)
    assert np.all(np.abs(got - ref) <= np.spacing(np.abs(ref)) + 0.0)
