"""Host logic of the ensemble workload: the seeded draw, the partition of
rings across ranks by cell count, and the sharded run on two gloo ranks on
the CPU (each rank steps its rings with the oracle standing in for the GPU
contexts, no exchange while stepping, one gather of per-ring diagnostics at
the end), which must give the rows a single process gives."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def test_ensemble_draw_and_partition():
    from vring_b200 import ensemble as E
    specs = E.ensemble_specs()
    assert len(specs) == 64
    assert {s["nr"] for s in specs} <= {64, 96, 128} and {s["nth"] for s in specs} <= {32, 64}
    assert {s["nz"] for s in specs} <= {128, 256}
    assert all(500 <= s["re"] <= 4000 and 0.8 <= s["R"] <= 1.2 and 0.1 <= s["sr"] <= 0.3 for s in specs)
    assert E.ensemble_specs() == specs                       # seeded
    for world in (1, 2, 3, 4, 8):
        parts = E.partition(specs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))                       # every ring exactly once
        assert E.imbalance(specs, parts) < 1.06, world       # LPT on 64 rings of 3 sizes classes
    # a single huge ring cannot be split: it takes a rank alone
    big = specs[:3] + [dict(specs[0], index=3, nr=1024, nth=256, nz=1024)]
    parts = E.partition(big, 2)
    assert [3] in parts


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rows_for(specs, idx):
    """Two RK3 steps of each ring (a small-grid stand-in of the same draw) on
    the oracle: (index, max |q3|, sum q2^2)."""
    from oracle import oracle as O
    from vring_b200.synthetic import ring_fields
    rows = []
    for i in idx:
        s = specs[i]
        nth, nr, nz = s["nth"] // 8, s["nr"] // 8, s["nz"] // 8
        o = O.Oracle(nth, nr, nz, 4.0, 12.0, 1e-3, s["re"], 1.0, 1.0, 1, 0, 1)
        q = ring_fields(nth, nr, nz, 4.0, 12.0, R=s["R"], sigma=s["sr"] * s["R"], z0=3.0, noise=1e-4, seed=i)
        for n, a in zip(("q1", "q2", "q3"), q):
            o.field(n)[...] = a
        o.iterate(2)
        rows.append((i, float(np.abs(o.field("q3")).max()), float((o.field("q2") ** 2).sum())))
        o.close()
    return rows


def _worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from vring_b200 import ensemble as E
    from vring_b200 import replicas
    rep = replicas.init("gloo", timeout_s=60.0)
    specs = E.ensemble_specs(12, seed=1)
    mine = E.partition(specs, rep.world)[rep.rank]
    rows = _rows_for(specs, mine)
    got = E.gather_rows(rows, rep)
    if rep.rank == 0:
        out["rows"] = got
    out[rank] = mine
    rep.close()


@pytest.mark.timeout(300)
def test_sharded_ensemble_on_two_gloo_ranks():
    from vring_b200 import ensemble as E
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    specs = E.ensemble_specs(12, seed=1)
    assert sorted(res[0] + res[1]) == list(range(12)) and not set(res[0]) & set(res[1])
    single = sorted(_rows_for(specs, range(12)))
    assert res["rows"] == single                 # bit-identical rows, gathered in ring order
