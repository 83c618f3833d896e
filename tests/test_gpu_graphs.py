"""Substeps replayed as captured CUDA graphs give the same state, bit for bit,
and the same launch count as the kernels issued one by one."""
import numpy as np
import pytest

FIELDS = ("q1", "q2", "q3", "dq1", "dq2", "dq3", "ru1", "ru2", "ru3", "pres", "prg", "dph", "rhs")


def _run(V, precision, graphs):
    from vring_b200.synthetic import annulus_particles, ring_fields
    nth, nr, nz = 32, 64, 128
    run = V.Run(nth, nr, nz, 4.0, 12.0, 2e-3, 1000.0, 1.0, 1.0, precision=precision,
                theta_wavenumber="modified")
    run.set_graphs(graphs)
    for n, a in zip(("q1", "q2", "q3"), ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-4, seed=0)):
        run.set(n, a)
    npart = 2048
    part = V.Part(run, 8, npart, 1)
    u = np.zeros((npart, 117), order="F")
    u[:, 0], u[:, 1], u[:, 2] = annulus_particles(npart, 0.5, 1.5, 2.0, 4.0, seed=0)
    part.set_state(u, np.zeros((npart, 3), order="F"), None, npart)
    part.attach(True)
    n0 = run.launch_count
    run.iterate(4)
    run.substep(1)  # a single substep through the same path
    out = {n: run.get(n) for n in FIELDS}
    out["part"] = part.state()[0]
    out["launches"] = run.launch_count - n0
    part.attach(False)
    part.close()
    run.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_matches_launch_by_launch(precision):
    import vring_b200 as V
    a = _run(V, precision, True)
    b = _run(V, precision, False)
    assert a["launches"] == b["launches"]
    for k in FIELDS + ("part",):
        assert np.array_equal(a[k], b[k]), k
