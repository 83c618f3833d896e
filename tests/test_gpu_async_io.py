"""Asynchronous field transfers (vr_set_field_async / vr_get_field_async):
steps driven through them on two copy streams give the state the blocking
transfers give, bit for bit, and a float-stored field is refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_async_round_trips_match_blocking_transfers():
    import torch
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 32, 48, 96
    q = ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=2)
    names = ("q1", "q2", "q3")

    def make():
        r = V.Run(nth, nr, nz, 4.0, 12.0, 1e-3, 1500.0, 1.0, 1.0, theta_wavenumber="modified")
        for n, a in zip(names, q):
            r.set(n, a)
        return r

    ref = make()
    host = [np.array(a, order="F") for a in q]
    for _ in range(3):
        for n, a in zip(names, host):
            ref.set(n, a)
        ref.iterate(1)
        host = [ref.get(n) for n in names]
    run = make()
    pins = [torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).pin_memory() for a in q]
    h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()
    for st in range(3):
        # the set of a field waits for the previous get of the same field
        # (same host buffer) inside the library
        for p, n in zip(pins, names):
            run.set_async(n, p.data_ptr(), h2d.cuda_stream)
        run.iterate(1)
        for p, n in zip(pins, names):
            run.get_async(n, p.data_ptr(), d2h.cuda_stream)
    d2h.synchronize()
    run.sync()
    for p, a in zip(pins, host):
        assert np.array_equal(p.numpy().reshape(a.shape, order="F"), a)
    mixed = V.Run(nth, nr, nz, 4.0, 12.0, 1e-3, 1500.0, 1.0, 1.0, precision="mixed")
    with pytest.raises(V.VrError):
        mixed.get_async("ru1", pins[0].data_ptr(), d2h.cuda_stream)
    for r in (ref, run, mixed):
        r.close()


def test_pipelined_transfers_with_separate_buffers():
    # Inputs for every step in their own host buffers, queued before the
    # steps run, and one result buffer per step: the host->device copies run
    # ahead of the steps and the device->host copies behind them, through the
    # staging buffers.  Each result must be the step of its own input.
    import torch
    import vring_b200 as V
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 32, 48, 96
    names = ("q1", "q2", "q3")
    nsteps = 4
    inputs = [ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=10 + k) for k in range(nsteps)]

    def make():
        return V.Run(nth, nr, nz, 4.0, 12.0, 1e-3, 1500.0, 1.0, 1.0, theta_wavenumber="modified")

    ref = make()
    expect = []
    for qk in inputs:
        for n, a in zip(names, qk):
            ref.set(n, a)
        ref.iterate(1)
        expect.append([ref.get(n) for n in names])
    run = make()
    pin_in = [[torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).pin_memory() for a in qk]
              for qk in inputs]
    pin_out = [[torch.empty_like(p).pin_memory() for p in row] for row in pin_in]
    h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()
    for k in range(nsteps):
        for p, n in zip(pin_in[k], names):
            run.set_async(n, p.data_ptr(), h2d.cuda_stream)
        run.iterate(1)
        for p, n in zip(pin_out[k], names):
            run.get_async(n, p.data_ptr(), d2h.cuda_stream)
    d2h.synchronize()
    run.sync()
    for k in range(nsteps):
        for p, a in zip(pin_out[k], expect[k]):
            assert np.array_equal(p.numpy().reshape(a.shape, order="F"), a)
    for r in (ref, run):
        r.close()
