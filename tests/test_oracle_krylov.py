"""The CPU restatement of the axisymmetric pressure problem (oracle/krylov2d.py)
and of the learned preconditioner's network (oracle/unet_ref.py).

- On the reference's uniform mesh the physical-space operator reproduces the
  reference's fftp solve at Ntheta = 1 (the oracle's laplace_solve,
  poisson_solve.F90:140-179, 270-323) to round-off.
- On the tanh-stretched mesh the DCT/radial-Thomas direct solve agrees with a
  scipy.sparse LU solve of the assembled symmetric operator.
- CG, Jacobi CG and BiCGSTAB (numpy) converge to 1e-10 to the same answer.
- The network's hand-written reverse pass agrees with central differences
  (rounding switched off; the network is linear, so they are exact to
  round-off), and the network is homogeneous.
"""
import numpy as np


def test_uniform_operator_is_the_reference_solve_at_ntheta_1(oracle_mod):
    from oracle import krylov2d as K
    nr, nz, R, Z = 24, 40, 5.0, 15.0
    ax = K.Axisym(K.uniform_faces(nr, R), nz, Z)
    f = np.random.default_rng(0).standard_normal((nr, nz))
    x = ax.solve_direct(f)
    assert np.abs(ax.apply_K(x) - f).max() <= 1e-12 * np.abs(f).max() * 1e3
    o = oracle_mod.Oracle(1, nr, nz, R, Z, 1e-3, 100.0)
    o.field("rhs")[...] = f.reshape(1, nr, nz)
    o.laplace_solve()
    dph = o.field("dph")[0, 1:nr + 1, 1:nz + 1]
    assert np.abs(dph - x).max() <= 1e-12 * np.abs(x).max()


def test_stretched_direct_solve_matches_scipy_sparse():
    import scipy.sparse.linalg as spla
    from oracle import krylov2d as K
    nr, nz = 48, 64
    faces = K.stretched_faces(nr, 5.0)
    dr = np.diff(faces)
    assert faces[0] == 0.0 and abs(faces[-1] - 5.0) < 1e-15 and np.all(dr > 0)
    rm = 0.5 * (faces[1:] + faces[:-1])
    assert abs(rm[np.argmin(dr)] - 1.0) < 2 * dr.min()          # clustered at the ring radius
    assert 4.0 < dr.max() / dr.min() < 8.0
    ax = K.Axisym(faces, nz, 15.0)
    S = ax.matrix_S()
    assert abs(S - S.T).max() == 0.0
    f = np.random.default_rng(1).standard_normal((nr, nz))
    xs = spla.spsolve(S.tocsc(), (f * ax.vol[:, None]).ravel(order="F")).reshape(nr, nz, order="F")
    xd = ax.solve_direct(f)
    assert np.abs(xs - xd).max() <= 1e-11 * np.abs(xd).max()


def test_numpy_krylov_methods_converge_to_the_direct_solve():
    from oracle import krylov2d as K
    nr, nz = 32, 48
    ax = K.Axisym(K.stretched_faces(nr, 5.0), nz, 15.0)
    f = np.random.default_rng(2).standard_normal((nr, nz))
    xd = ax.solve_direct(f)
    for kw in ({}, {"jacobi": True}):
        x, it, rr = ax.cg(f, 1e-10, **kw)
        assert rr <= 1e-10 and np.abs(x - xd).max() <= 1e-7 * np.abs(xd).max()
    x, it, rr = ax.bicgstab(f, 1e-10)
    assert rr <= 1e-10 and np.abs(x - xd).max() <= 1e-7 * np.abs(xd).max()


def test_unet_reverse_pass_matches_central_differences():
    from oracle import unet_ref as U
    ch = (8, 8, 8, 8)
    rng = np.random.default_rng(0)
    w = rng.standard_normal(U.nparams(ch)) * 0.2
    x, g = rng.standard_normal((16, 32)), rng.standard_normal((16, 32))
    ident = lambda a: np.asarray(a, dtype=np.float64)  # noqa: E731
    gw, gx = U.backward(w, ch, x, g, rnd=ident)
    L = lambda w_, x_: np.sum(g * U.forward(w_, ch, x_, rnd=ident))  # noqa: E731
    for idx in rng.choice(w.size, 12, replace=False):
        e = np.zeros_like(w)
        e[idx] = 1e-4
        fd = (L(w + e, x) - L(w - e, x)) / 2e-4
        assert abs(fd - gw[idx]) <= 1e-6 * max(1.0, abs(fd))
    for j, k in ((0, 0), (5, 9), (15, 31)):
        e = np.zeros_like(x)
        e[j, k] = 1e-4
        fd = (L(w, x + e) - L(w, x - e)) / 2e-4
        assert abs(fd - gx[j, k]) <= 1e-6 * max(1.0, abs(fd))
    assert np.abs(U.forward(w, ch, 3 * x, rnd=ident) - 3 * U.forward(w, ch, x, rnd=ident)).max() < 1e-9
    assert U.nparams((16, 32, 48, 64)) == 225952


def test_bf16_rounding_is_nearest_even():
    from oracle import unet_ref as U
    import struct
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
    assert U.bf16(1.0 + 2.0 ** -8) == 1.0
    assert U.bf16(1.0 + 3 * 2.0 ** -8) == 1.0 + 2.0 ** -6
    assert U.bf16(-2.5) == -2.5
    v = struct.unpack("f", struct.pack("I", 0x3F808001))[0]
    assert U.bf16(v) == 1.0 + 2.0 ** -7


def test_unet_reverse_pass_with_4x4_pooling():
    from oracle import unet_ref as U
    ch = (8, 8, 8, 8)
    rng = np.random.default_rng(5)
    w = rng.standard_normal(U.nparams(ch)) * 0.2
    x, g = rng.standard_normal((64, 64)), rng.standard_normal((64, 64))
    ident = lambda a: np.asarray(a, dtype=np.float64)  # noqa: E731
    gw, gx = U.backward(w, ch, x, g, rnd=ident, F=4)
    L = lambda w_, x_: np.sum(g * U.forward(w_, ch, x_, rnd=ident, F=4))  # noqa: E731
    for idx in rng.choice(w.size, 8, replace=False):
        e = np.zeros_like(w)
        e[idx] = 1e-4
        assert abs((L(w + e, x) - L(w - e, x)) / 2e-4 - gw[idx]) <= 1e-6 * max(1.0, abs(gw[idx]))
    e = np.zeros_like(x)
    e[17, 40] = 1e-4
    assert abs((L(w, x + e) - L(w, x - e)) / 2e-4 - gx[17, 40]) <= 1e-6 * max(1.0, abs(gx[17, 40]))
