"""The VR2D axisymmetric pressure solve with a learned preconditioner.

Grid (the axisymmetric deck, r in [0, 5], z in [0, 15], 512 x 1024 cells) with
the radial faces clustered toward the ring radius r = 1 by a tanh map of
strength beta = 2: the index coordinate xi = A + B tanh(beta (r - 1) / 5)
runs uniformly from 0 to 1.  The network pools 4 x 4 between its four levels
(512 x 1024 down to 8 x 16), so its coarsest level sees the whole domain: with
2 x 2 pooling the coarsest level is 64 x 128 cells, a preconditioner of that
reach cannot act on the domain-wide modes, and the flexible CG stalled on
this grid.

Training data: (right-hand side, previous-step pressure, converged pressure)
triples from seeded synthetic sequences (seeds 2-21): a Gaussian-core ring
pressure low travelling along z with a slowly drifting radius, core size and
strength plus smooth seeded perturbations; the right-hand side of step t is
K applied to that step's pressure field, and the converged pressure is the
plain solver's answer (the direct DCT/radial-Thomas solve, which the Krylov
solves agree with to their tolerance).  What the preconditioner must undo is
the error of the warm start, e = p_t - p_{t-1}, whose residual is r = S e.
The network is applied with the symmetric Jacobi scaling, y = s D N(D r / s)
(D = diag(S)^-1/2, s the RMS of D r), which takes out the operator's strong
variation with the radius so that one translation-invariant network fits the
whole grid, and it is trained on the error in S's energy norm,
L = (y - e)' S (y - e) / e' S e, the norm CG minimises.  Half of each batch
is triple increments; a quarter random smooth fields and a quarter white
noise in the scaled variables (e = D w), so that the map also covers the
rougher errors a Krylov iteration leaves.

Everything runs on the GPU through the library (vr_k2d_*, vr_unet_*); torch
only holds device buffers.
"""
from __future__ import annotations

import os

import numpy as np

from .api import K2d, UNet

NR, NZ, RMAX, ZMAX = 512, 1024, 5.0, 15.0
BETA, RCLUST = 2.0, 1.0
CHANNELS = (16, 32, 48, 64)
POOL = 4  # 4 x 4 pooling: levels of 512 x 1024, 128 x 256, 32 x 64 and 8 x 16 cells
SEEDS = tuple(range(2, 22))
STEPS_PER_SEED = 1000
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "unet_vr2d_512x1024.npz")


def tanh_faces(nr: int = NR, rmax: float = RMAX, beta: float = BETA, rclust: float = RCLUST) -> np.ndarray:
    """nr + 1 radial faces, xi = A + B tanh(beta (r - rclust) / rmax) uniform."""
    t0 = np.tanh(beta * (0.0 - rclust) / rmax)
    t1 = np.tanh(beta * (rmax - rclust) / rmax)
    b = 1.0 / (t1 - t0)
    a = -b * t0
    xi = np.arange(nr + 1, dtype=np.float64) / nr
    r = rclust + rmax / beta * np.arctanh((xi - a) / b)
    r[0], r[-1] = 0.0, rmax
    return r


def cell_centres(faces, nz=NZ, zmax=ZMAX):
    rm = 0.5 * (faces[:-1] + faces[1:])
    zm = (np.arange(nz) + 0.5) * (zmax / nz)
    return rm, zm


class RingSequence:
    """Seeded pressure sequence p_t(r, z) of a travelling Gaussian-core ring."""

    def __init__(self, seed: int, faces, nz=NZ, zmax=ZMAX, nmodes=6):
        rng = np.random.default_rng(seed)
        self.rm, self.zm = cell_centres(faces, nz, zmax)
        self.R0 = rng.uniform(0.9, 1.1)
        self.z0 = rng.uniform(2.5, 4.0)
        self.U = rng.uniform(0.5, 1.5) * 2e-3      # z travel per step
        self.sig = rng.uniform(0.15, 0.3)
        self.amp = rng.uniform(0.5, 1.5)
        self.phase = rng.uniform(0, 2 * np.pi, 3)
        # smooth perturbation: a few separable cosine modes with slowly varying amplitude
        self.kr = rng.integers(1, 8, nmodes)
        self.kz = rng.integers(1, 16, nmodes)
        self.a0 = rng.normal(0.0, 0.05, nmodes)
        self.w = rng.uniform(0.002, 0.01, nmodes)
        self.rmax, self.zmax = faces[-1], zmax

    def pressure(self, t: int) -> np.ndarray:
        R = self.R0 * (1 + 0.05 * np.sin(1e-3 * t + self.phase[0]))
        s = self.sig * (1 + 0.1 * np.sin(7e-4 * t + self.phase[1]))
        A = self.amp * (1 + 0.1 * np.sin(5e-4 * t + self.phase[2]))
        zc = self.z0 + self.U * t
        r, z = self.rm[:, None], self.zm[None, :]
        p = -A * np.exp(-((r - R) ** 2 + (z - zc) ** 2) / (s * s))
        for a0, kr, kz, w in zip(self.a0, self.kr, self.kz, self.w):
            p = p + a0 * np.cos(w * t) * np.cos(np.pi * kr * r / self.rmax) * np.cos(np.pi * kz * z / self.zmax)
        return p


def make_solver(device: int = 0, nr: int = NR, nz: int = NZ) -> K2d:
    return K2d(tanh_faces(nr), nz, ZMAX, device=device)


def make_net(device: int = 0, nr: int = NR, nz: int = NZ, seed: int = 1, ch=CHANNELS, pool: int = POOL) -> UNet:
    return UNet(nr, nz, ch, seed=seed, device=device, pool=pool)


def save_weights(net: UNet, path: str = WEIGHTS, **meta) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, w=net.get_params(), ch=np.array(net.ch), nr=net.nr, nz=net.nz, pool=net.pool, **meta)


def load_weights(net: UNet, path: str = WEIGHTS) -> dict:
    d = np.load(path)
    assert tuple(d["ch"]) == net.ch and int(d["nr"]) == net.nr and int(d["nz"]) == net.nz
    assert int(d["pool"]) == net.pool
    net.set_params(d["w"])
    return {k: d[k] for k in d.files if k not in ("w",)}


def triple(k2d: K2d, seq: RingSequence, t: int):
    """(f_t, p_{t-1}, p_t): right-hand side, previous and converged pressure."""
    f = k2d.apply(seq.pressure(t))
    p = k2d.direct(f)
    p_prev = k2d.direct(k2d.apply(seq.pressure(t - 1))) if t > 0 else np.zeros_like(p)
    return f, p_prev, p


def train(net: UNet, k2d: K2d, steps: int, batch: int = 8, lr: float = 3e-3, seed: int = 0, log=None,
          lr_final: float = 3e-4):
    """Adam on batches of errors: half warm-start errors of the triple
    sequences, a quarter random smooth fields, a quarter scaled white noise."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(seed)
    seqs = [RingSequence(s, k2d.faces, k2d.nz, k2d.zmax) for s in SEEDS]
    n = k2d.nr * k2d.nz
    buf = torch.empty((batch, n), dtype=torch.float64, device=dev)
    rm, zm = cell_centres(k2d.faces, k2d.nz, k2d.zmax)
    dhalf = 1.0 / np.sqrt(k2d.diag())
    losses = []
    for it in range(steps):
        for b in range(batch):
            kind = b % 4
            if kind < 2:
                seq = seqs[rng.integers(len(seqs))]
                t = int(rng.integers(1, STEPS_PER_SEED))
                _, p_prev, p = triple(k2d, seq, t)
                e = p - p_prev
            elif kind == 2:
                kr = rng.integers(0, k2d.nr // 2, 8)
                kzz = rng.integers(0, k2d.nz // 2, 8)
                a = rng.normal(size=8) / (1.0 + kr + kzz)
                e = sum(ai * np.cos(np.pi * ki * rm[:, None] / k2d.faces[-1]) * np.cos(np.pi * kj * zm[None, :] / k2d.zmax)
                        for ai, ki, kj in zip(a, kr, kzz))
            else:
                e = rng.standard_normal((k2d.nr, k2d.nz)) * dhalf
            buf[b].copy_(torch.from_numpy(np.asfortranarray(e).ravel(order="F")))
        frac = it / max(1, steps - 1)
        lr_t = lr * (lr_final / lr) ** frac
        torch.cuda.synchronize()  # the library's streams do not wait for torch's
        loss = net.train_step(k2d, buf.data_ptr(), batch, lr_t)
        losses.append(loss)
        if log is not None and (it % 50 == 0 or it == steps - 1):
            log("step %d loss %.4e lr %.2e" % (it, loss, lr_t))
    return losses


def compare(k2d: K2d, net: UNet, f, x0=None, tol: float = 1e-10, maxit: int = 40000):
    """Plain CG, Jacobi CG, the flexible CG with the Jacobi steps alone and
    with the network between them, on one right-hand side:
    {method: (iterations, relres, ms, x)}; each stops after maxit iterations."""
    out = {}
    for m in ("cg", "pcg", "fcg_jacobi", "learned"):
        if m == "learned":
            k2d.set_preconditioner(net)
        x, it, rr, ms = k2d.solve(f, m, x0=x0, tol=tol, maxit=maxit)
        out[m] = (it, rr, ms, x)
    k2d.set_preconditioner(None)
    return out


def main(argv=None):
    """Train the VR2D preconditioner on the GPU and write its weights:
    python -m vring_b200.learned [--steps 800] [--batch 8] [--out path]
    (the committed weights came from the defaults), then compare the solvers
    on one triple of each of seeds 2, 7 and 21.  With --forward N it only
    runs N forward passes of an untrained network on a seeded random field
    (the case the convolution profiles are taken on) and exits; with
    --solve N it runs N iterations of the learned flexible CG with the
    committed weights on the triple of seed 2, step 500, and exits; with
    --compare it skips the training and compares the solvers with the
    committed weights."""
    import argparse
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=800)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--lr-final", type=float, default=3e-4)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--forward", type=int, default=0)
    ap.add_argument("--solve", type=int, default=0)
    ap.add_argument("--compare", action="store_true")
    a = ap.parse_args(argv)
    if a.solve:
        k = make_solver()
        net = make_net()
        load_weights(net)
        seq = RingSequence(2, k.faces, k.nz, k.zmax)
        f, p_prev, _ = triple(k, seq, 500)
        k.set_preconditioner(net)
        _, it, rr, ms = k.solve(f, "learned", x0=p_prev, tol=1e-30, maxit=a.solve)
        k.set_preconditioner(None)
        print("learned flexible CG: %d iterations, relres %.3e, %.2f ms" % (it, rr, ms))
        return
    if a.forward:
        net = make_net()
        x = np.random.default_rng(0).standard_normal((NR, NZ))
        for _ in range(a.forward):
            y = net.forward(x)
        print("forward passes %d, max|y| %.6g" % (a.forward, float(np.abs(y).max())))
        return
    k = make_solver()
    net = make_net()
    if a.compare:
        load_weights(net)
    else:
        t0 = time.time()
        train(net, k, a.steps, batch=a.batch, lr=a.lr, lr_final=a.lr_final,
              log=lambda s: print(s, "%.0fs" % (time.time() - t0), flush=True))
        save_weights(net, a.out, steps=a.steps, batch=a.batch, lr=a.lr, lr_final=a.lr_final)
    for seed, t in ((2, 500), (7, 250), (21, 900)):
        seq = RingSequence(seed, k.faces, k.nz, k.zmax)
        f, p_prev, p = triple(k, seq, t)
        for m, (it, rr, ms, x) in compare(k, net, f, x0=p_prev).items():
            print("seed %d t %d %-10s %6d iterations  relres %.2e  %8.1f ms  max|x - direct| / max|direct| %.2e"
                  % (seed, t, m, it, rr, ms, np.abs(x - p).max() / np.abs(p).max()), flush=True)


if __name__ == "__main__":
    main()
