"""CPU restatement of the axisymmetric (Ntheta = 1) pressure problem that the
GPU Krylov solvers of ``vring_b200`` solve.  TEST INFRASTRUCTURE ONLY: the
tests, ``__graft_entry__.smoke`` and the CPU legs of ``bench.py`` use it as the
checker; the product package never imports it.

The operator is the reference's radial Poisson operator at Ntheta = 1
(poisson.F90:379-381 for the bands aa/bb/cc, poisson_solve.F90:270-323 for the
per-mode closure), written in physical space instead of per z mode:

  K phi = -(1/r) d/dr (r dphi/dr) - d2phi/dz2

on cell centres (rm_j, zm_k), Neumann on the axis (the axis face has r = 0),
at r = rmax and at z = 0, zmax (the DCT-II/III pair of
fastfouriertransform.F90:250-339 diagonalises the Neumann z operator), and
the (m = 0, kz = 0) closure of poisson_solve.F90:305-317: the z-mean of phi
obeys a Dirichlet condition at the wall face (ghost = -phi), i.e. row nr gains
gam * mean_k phi(nr, k).  On a uniform radial grid the finite-volume form
below reproduces the reference's finite-difference rows exactly
(aa = -rc_j / (rm_j dr^2), cc = -rc_{j+1} / (rm_j dr^2)); on a stretched grid
it is the conservative generalisation (no reference counterpart: the
reference mesh is uniform, mesh_tools.F90:325-330).

Symmetric form: S = V K with V_j = rm_j dr_j dz (cell volume over 2 pi), so
S is symmetric positive definite and CG applies to S x = V f.

Stretched grid (no reference counterpart): the uniform index coordinate
xi = 0..1 is a tanh of the radius, xi = A + B tanh(beta (r - rc) / rmax), with
A and B fixed by r(0) = 0 and r(1) = rmax, so dr/dxi ~ cosh^2(beta (r - rc) /
rmax) and the spacing is smallest at r = rc (the ring radius); with beta = 2,
rc = 1, rmax = 5 the widest cell is about 6x the narrowest.
"""
from __future__ import annotations

import numpy as np


def uniform_faces(nr: int, rmax: float) -> np.ndarray:
    """Radial faces rc_1..rc_{nr+1} of the reference's uniform mesh
    (mesh_tools.F90:325-330)."""
    return np.arange(nr + 1, dtype=np.float64) * (rmax / nr)


def stretched_faces(nr: int, rmax: float, beta: float = 2.0, rclust: float = 1.0) -> np.ndarray:
    """Faces clustered toward r = rclust: xi = A + B tanh(beta (r - rclust) / rmax)."""
    t0 = np.tanh(beta * (0.0 - rclust) / rmax)
    t1 = np.tanh(beta * (rmax - rclust) / rmax)
    B = 1.0 / (t1 - t0)
    A = -B * t0
    xi = np.arange(nr + 1, dtype=np.float64) / nr
    r = rclust + rmax / beta * np.arctanh((xi - A) / B)
    r[0], r[-1] = 0.0, rmax
    return r


class Axisym:
    """The operator on faces rc (nr+1 values from 0 to rmax) and nz uniform
    z cells on [0, zmax].  Vectors are (nr, nz) arrays, index [j, k], stored
    r fastest (Fortran order) on the device."""

    def __init__(self, faces: np.ndarray, nz: int, zmax: float):
        rc = np.asarray(faces, dtype=np.float64)
        self.nr, self.nz = rc.size - 1, nz
        self.rc, self.dz = rc, zmax / nz
        self.dr = np.diff(rc)
        self.rm = 0.5 * (rc[:-1] + rc[1:])
        nr, dz = self.nr, self.dz
        h = np.diff(self.rm)                      # centre spacings h_{j+1/2}
        self.aw = np.zeros(nr)                    # coupling to j-1 (S form)
        self.ae = np.zeros(nr)                    # coupling to j+1
        self.aw[1:] = rc[1:nr] * dz / h
        self.ae[:-1] = rc[1:nr] * dz / h
        self.az = self.rm * self.dr / dz          # coupling to k +- 1
        self.vol = self.rm * self.dr * dz
        # (m, kz) = (0, 0) Dirichlet closure at the wall face for the z-mean
        self.gam = 2.0 * rc[nr] * dz / self.dr[nr - 1]

    def apply_S(self, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, dtype=np.float64).reshape(self.nr, self.nz)
        y = np.zeros_like(x)
        y[1:] += self.aw[1:, None] * (x[1:] - x[:-1])
        y[:-1] += self.ae[:-1, None] * (x[:-1] - x[1:])
        az = self.az[:, None]
        y[:, 1:] += az * (x[:, 1:] - x[:, :-1])
        y[:, :-1] += az * (x[:, :-1] - x[:, 1:])
        y[-1] += self.gam * x[-1].mean()
        return y

    def apply_K(self, x: np.ndarray) -> np.ndarray:
        return self.apply_S(x) / self.vol[:, None]

    def matrix_S(self):
        """S as a scipy sparse matrix (index j + nr k)."""
        import scipy.sparse as sp
        nr, nz = self.nr, self.nz
        idx = np.arange(nr * nz).reshape(nz, nr).T          # idx[j, k] = j + nr k
        rows, cols, vals = [], [], []

        def add(r, c, v):
            rows.append(r.ravel()), cols.append(c.ravel()), vals.append(np.broadcast_to(v, r.shape).ravel())
        w = np.broadcast_to(self.aw[1:, None], (nr - 1, nz))
        add(idx[1:], idx[1:], w), add(idx[1:], idx[:-1], -w)
        e = np.broadcast_to(self.ae[:-1, None], (nr - 1, nz))
        add(idx[:-1], idx[:-1], e), add(idx[:-1], idx[1:], -e)
        a = np.broadcast_to(self.az[:, None], (nr, nz - 1))
        add(idx[:, 1:], idx[:, 1:], a), add(idx[:, 1:], idx[:, :-1], -a)
        add(idx[:, :-1], idx[:, :-1], a), add(idx[:, :-1], idx[:, 1:], -a)
        last = idx[-1]
        rr, cc = np.meshgrid(last, last, indexing="ij")
        add(rr, cc, np.full(rr.shape, self.gam / nz))
        n = nr * nz
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(n, n))

    def solve_direct(self, f: np.ndarray) -> np.ndarray:
        """K phi = f by the reference's fftp method at Ntheta = 1
        (poisson_solve.F90:140-179, 270-323): DCT-II in z scaled 1/(2 nz),
        one radial tridiagonal per kz with wz = 2/dz^2 (1 - cos(pi kz / nz)),
        Neumann closures except the Dirichlet wall row of kz = 0, then DCT-III."""
        import scipy.fft as sf
        from scipy.linalg import solve_banded
        nr, nz, dz = self.nr, self.nz, self.dz
        fh = sf.dct(np.asarray(f, dtype=np.float64).reshape(nr, nz), type=2, axis=1) / (2.0 * nz)
        # K rows from S / V: off-diagonals -aw/V, -ae/V; radial diagonal (aw + ae)/V
        lo = -self.aw / self.vol
        up = -self.ae / self.vol
        dg0 = (self.aw + self.ae) / self.vol
        sol = np.empty_like(fh)
        for kz in range(nz):
            wz = 2.0 / (dz * dz) * (1.0 - np.cos(kz * np.pi / nz))
            dg = dg0 + wz
            if kz == 0:
                dg = dg.copy()
                dg[-1] += self.gam / self.vol[-1]
            ab = np.zeros((3, nr))
            ab[0, 1:] = up[:-1]
            ab[1] = dg
            ab[2, :-1] = lo[1:]
            sol[:, kz] = solve_banded((1, 1), ab, fh[:, kz])
        return sf.dct(sol, type=3, axis=1)

    def cg(self, f, tol=1e-10, maxit=100000, x0=None, jacobi=False):
        """Plain (or diagonally preconditioned) CG on S x = V f; returns
        (x, iterations, relative residual ||V f - S x|| / ||V f||)."""
        b = (np.asarray(f, dtype=np.float64).reshape(self.nr, self.nz) * self.vol[:, None])
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64).reshape(b.shape)
        d = self.diag_S() if jacobi else None
        r = b - self.apply_S(x)
        bn = np.linalg.norm(b)
        z = r / d if jacobi else r
        p = z.copy()
        rz = np.vdot(r, z)
        it = 0
        while np.linalg.norm(r) > tol * bn and it < maxit:
            q = self.apply_S(p)
            a = rz / np.vdot(p, q)
            x += a * p
            r -= a * q
            z = r / d if jacobi else r
            rz_new = np.vdot(r, z)
            p = z + (rz_new / rz) * p
            rz = rz_new
            it += 1
        return x, it, np.linalg.norm(b - self.apply_S(x)) / bn

    def bicgstab(self, f, tol=1e-10, maxit=100000, x0=None):
        """BiCGSTAB on the unsymmetric form K x = f; returns (x, iterations,
        relative residual ||f - K x|| / ||f||)."""
        b = np.asarray(f, dtype=np.float64).reshape(self.nr, self.nz)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64).reshape(b.shape)
        r = b - self.apply_K(x)
        rh = r.copy()
        bn = np.linalg.norm(b)
        rho = alpha = om = 1.0
        v = np.zeros_like(b)
        p = np.zeros_like(b)
        it = 0
        while np.linalg.norm(r) > tol * bn and it < maxit:
            rho_new = np.vdot(rh, r)
            beta = (rho_new / rho) * (alpha / om)
            p = r + beta * (p - om * v)
            v = self.apply_K(p)
            alpha = rho_new / np.vdot(rh, v)
            s = r - alpha * v
            t = self.apply_K(s)
            om = np.vdot(t, s) / np.vdot(t, t)
            x += alpha * p + om * s
            r = s - om * t
            rho = rho_new
            it += 1
        return x, it, np.linalg.norm(b - self.apply_K(x)) / bn

    def diag_S(self) -> np.ndarray:
        d = np.broadcast_to((self.aw + self.ae)[:, None], (self.nr, self.nz)).copy()
        d[:, 1:] += self.az[:, None]
        d[:, :-1] += self.az[:, None]
        d[-1] += self.gam / self.nz
        return d
