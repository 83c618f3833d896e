"""The multi-GPU path of the benchmark is independent replicas (one per GPU,
no exchange between them): the host logic around it -- process group, the
barrier around the timed region, the max over ranks of the timed duration and
the whole-job throughput -- runs here on two gloo ranks on the CPU.  Each rank
also advances its own oracle replica of a small ring, and the replicas agree
bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from vring_b200 import replicas
    from oracle import oracle as O
    from vring_b200.synthetic import ring_fields
    rep = replicas.init("gloo", timeout_s=60.0)
    assert rep.distributed and rep.world == world and rep.rank == rank
    o = O.Oracle(8, 16, 32, 4.0, 12.0, 2e-3, 1000.0, 1.0, 1.0, 1, 0, 0)
    for n, a in zip(("q1", "q2", "q3"), ring_fields(8, 16, 32, 4.0, 12.0, seed=0)):
        o.field(n)[...] = a
    rep.barrier()
    o.iterate(2)
    elapsed = 1.0 + rank          # stand-in for each rank's device-timed seconds
    tmax = rep.max_over_ranks(elapsed)
    out[rank] = (tmax, replicas.throughput(1000.0, rep.world, tmax),
                 float(np.abs(o.field("q3")).sum()))
    rep.close()


@pytest.mark.timeout(300)
def test_two_gloo_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    assert set(res) == {0, 1}
    for r in range(world):
        tmax, thr, chk = res[r]
        assert tmax == 2.0                      # the slowest rank's time on every rank
        assert thr == world * 1000.0 / 2.0      # whole-job units over the max time
    assert res[0][2] == res[1][2]               # independent replicas, same result


def test_single_process_needs_no_group(monkeypatch):
    from vring_b200 import replicas
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    rep = replicas.init("gloo")
    assert not rep.distributed and rep.world == 1
    assert rep.max_over_ranks(3.5) == 3.5
    rep.barrier()
    rep.close()
