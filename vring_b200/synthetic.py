"""Seeded synthetic inputs: a Gaussian-core vortex ring on the staggered grid.

The reference builds its initial condition from Bessel-function quadratures
(gen_tools_swirl.F90:177-241, solu_toolsII.F90:206-305); the workloads here
instead prescribe a Gaussian-core ring, computed once on the host and fed
identically to the GPU and to the CPU checker:

  omega_theta(r, z) = Gamma / (pi sigma^2) exp(-((r-R)^2 + (z-z0)^2) / sigma^2)

The Stokes streamfunction psi solves E^2 psi = psi_rr - psi_r / r + psi_zz =
-r omega_theta at the cell corners (rc_j, zc_k) with psi = 0 on the axis and on
the other three boundaries (a sparse direct solve).  The staggered fluxes are
differences of psi, so the discrete divergence of divergence.F90:37-41
vanishes to round-off:

  q2(j, k) = r v_r at (rc_j, zm_k) = -(psi[j, k+1] - psi[j, k]) / dz
  q3(j, k) =   v_z at (rm_j, zc_k) =  (psi[j+1, k] - psi[j, k]) / (dr rm_j)

q1 = v_theta = 0.  A seeded perturbation of the given amplitude is then added
to q1, q2, q3 (normal, numpy default_rng(seed)) over the interior cells.
"""
from __future__ import annotations

import numpy as np


def ring_fields(ntheta, nr, nz, rmax, zmax, R=1.0, sigma=0.2, gamma=1.0, z0=3.0, noise=1e-4,
                seed=0, rings=None):
    """Return q1, q2, q3 in the ghosted (ntheta, nr+3, nz+3) Fortran layout.

    ``rings`` may list several (R, sigma, gamma, z0) tuples whose vorticity
    adds up (e.g. a head-on pair with opposite circulation)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    dr, dz = rmax / nr, zmax / nz
    if rings is None:
        rings = [(R, sigma, gamma, z0)]
    # corners (rc_j, zc_k), j = 1..nr+1, k = 1..nz+1 ; interior j = 2..nr, k = 2..nz
    rcs = (np.arange(1, nr + 2) - 1.0) * dr
    zcs = (np.arange(1, nz + 2) - 1.0) * dz
    ri = rcs[1:nr]            # interior radii
    zi = zcs[1:nz]
    nj, nk = nr - 1, nz - 1
    Rg, Zg = np.meshgrid(ri, zi, indexing="ij")
    om = np.zeros_like(Rg)
    for (Rr, s, g, zz0) in rings:
        om += g / (np.pi * s * s) * np.exp(-((Rg - Rr) ** 2 + (Zg - zz0) ** 2) / (s * s))
    b = (-Rg * om).ravel()
    # 5-point operator of E^2 on the interior corners (index j fastest)
    idx = np.arange(nj * nk).reshape(nj, nk)
    cm = 1.0 / dr ** 2 + 1.0 / (2.0 * Rg * dr)   # psi_{j-1}
    cp = 1.0 / dr ** 2 - 1.0 / (2.0 * Rg * dr)   # psi_{j+1}
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [np.full(nj * nk, -2.0 / dr ** 2 - 2.0 / dz ** 2)]
    for (sl_a, sl_b, coef) in (((slice(1, None), slice(None)), (slice(None, -1), slice(None)), cm[1:, :]),
                               ((slice(None, -1), slice(None)), (slice(1, None), slice(None)), cp[:-1, :]),
                               ((slice(None), slice(1, None)), (slice(None), slice(None, -1)), np.full((nj, nk - 1), 1.0 / dz ** 2)),
                               ((slice(None), slice(None, -1)), (slice(None), slice(1, None)), np.full((nj, nk - 1), 1.0 / dz ** 2))):
        rows.append(idx[sl_a].ravel())
        cols.append(idx[sl_b].ravel())
        vals.append(np.asarray(coef).ravel())
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nj * nk, nj * nk))
    psi_i = spla.spsolve(A.tocsc(), b).reshape(nj, nk)
    psi = np.zeros((nr + 2, nz + 2))          # psi[j, k] with j,k = 1-based corner index
    psi[2:nr + 1, 2:nz + 1] = psi_i
    shape = (ntheta, nr + 3, nz + 3)
    q1 = np.zeros(shape, order="F")
    q2 = np.zeros(shape, order="F")
    q3 = np.zeros(shape, order="F")
    rm = (np.arange(nr + 3) - 0.5) * dr
    # q2 at faces j = 1..nr+1, centres k = 1..nz
    q2v = -(psi[1:nr + 2, 2:nz + 2] - psi[1:nr + 2, 1:nz + 1]) / dz
    q2[:, 1:nr + 2, 1:nz + 1] = q2v[None]
    # q3 at centres j = 1..nr, faces k = 1..nz+1
    q3v = (psi[2:nr + 2, 1:nz + 2] - psi[1:nr + 1, 1:nz + 2]) / (dr * rm[1:nr + 1, None])
    q3[:, 1:nr + 1, 1:nz + 2] = q3v[None]
    if noise:
        rng = np.random.default_rng(seed)
        for q, (j0, j1, k0, k1) in ((q1, (1, nr, 1, nz)), (q2, (2, nr, 1, nz)), (q3, (1, nr, 2, nz))):
            q[:, j0:j1 + 1, k0:k1 + 1] += noise * rng.standard_normal((ntheta, j1 - j0 + 1, k1 - k0 + 1))
    return q1, q2, q3


def annulus_particles(n, r0, r1, z0, z1, seed=0):
    """n positions uniform in area over r0 <= r <= r1, uniform in theta and z."""
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.uniform(r0 * r0, r1 * r1, n))
    th = rng.uniform(0.0, 2.0 * np.pi, n)
    z = rng.uniform(z0, z1, n)
    return r * np.cos(th), r * np.sin(th), z
