"""Ensembles of independent vortex rings: the seeded ensemble workload, the
partition of rings across GPUs, and the sharded run.

Workload (64 rings drawn from numpy default_rng(1)): grids Nr in {64, 96, 128},
Ntheta in {32, 64}, Nz in {128, 256}; Re uniform in [500, 4000]; ring radius R
uniform in [0.8, 1.2]; core sigma / R uniform in [0.1, 0.3]; dt = 1e-3;
65,536 tracer particles per ring; the mixed precision form; r in [0, 4],
z in [0, 12] with the reference's z boundaries, the ring centred at z = 3.

Rings share nothing, so on N GPUs each rank takes a subset with no exchange
while stepping; the subsets are balanced by cell count (longest-processing-
time greedy: rings by decreasing cells, each to the least-loaded rank, ties
to the lower rank).  At the end rank 0 gathers one row of diagnostics per
ring (ring index, max |div u|, kinetic energy, live particles).
"""
from __future__ import annotations

import numpy as np

RMAX, ZMAX, DT, Z0 = 4.0, 12.0, 1e-3, 3.0
NPART = 65536


def ensemble_specs(n: int = 64, seed: int = 1) -> list[dict]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append(dict(index=i, nr=int(rng.choice([64, 96, 128])), nth=int(rng.choice([32, 64])),
                        nz=int(rng.choice([128, 256])), re=float(rng.uniform(500.0, 4000.0)),
                        R=float(rng.uniform(0.8, 1.2)), sr=float(rng.uniform(0.1, 0.3))))
    return out


def cells(spec: dict) -> int:
    return spec["nr"] * spec["nth"] * spec["nz"]


def partition(specs: list[dict], world: int) -> list[list[int]]:
    """Ring indices per rank, balanced by cell count (LPT greedy)."""
    order = sorted(range(len(specs)), key=lambda i: (-cells(specs[i]), i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += cells(specs[i])
    return [sorted(p) for p in parts]


def imbalance(specs: list[dict], parts: list[list[int]]) -> float:
    """max rank load / mean rank load."""
    loads = [sum(cells(specs[i]) for i in p) for p in parts]
    return max(loads) / (sum(loads) / len(loads))


def make_ring(spec: dict, precision: str = "mixed", device: int = 0, npart: int = NPART, seed: int | None = None):
    """A Run (and its attached tracer class) for one ensemble member."""
    from .api import Part, Run
    from .synthetic import annulus_particles, ring_fields
    s = spec
    seed = s["index"] if seed is None else seed
    run = Run(s["nth"], s["nr"], s["nz"], RMAX, ZMAX, DT, s["re"], 1.0, 1.0, precision=precision,
              theta_wavenumber="modified", device=device)
    q = ring_fields(s["nth"], s["nr"], s["nz"], RMAX, ZMAX, R=s["R"], sigma=s["sr"] * s["R"], gamma=1.0, z0=Z0,
                    noise=1e-4, seed=seed)
    for n, a in zip(("q1", "q2", "q3"), q):
        run.set(n, a)
    part = None
    if npart > 0:
        part = Part(run, 8, npart, 1)
        x, y, z = annulus_particles(npart, 0.5 * s["R"], 1.5 * s["R"], Z0 - 1.0, Z0 + 1.0, seed=seed)
        u = np.zeros((npart, 117), order="F")
        u[:, 0], u[:, 1], u[:, 2] = x, y, z
        part.set_state(u, np.zeros((npart, 3), order="F"), None, npart)
        part.attach(True)
    return run, part


def gather_rows(rows: list[tuple], rep) -> list[tuple] | None:
    """All ranks' diagnostic rows on rank 0 (sorted by ring index); None elsewhere."""
    if not rep.distributed:
        return sorted(rows)
    import torch.distributed as dist
    out = [None] * rep.world if rep.rank == 0 else None
    dist.gather_object(rows, out, dst=0)
    if rep.rank != 0:
        return None
    return sorted(r for part in out for r in part)
