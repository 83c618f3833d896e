"""vr_solve_lap_thom_noalloc (no allocation, fixed device scratch) against
vr_solve_lap_thom through the C ABI, and each system against the oracle's
restatement of trithom.F90:6-29.

The two entry points run the same per-system Thomas recurrence, so the
results are expected to agree to rounding: the test tolerance is 1e-14
relative to the largest solution entry.  Because both launch the same kernel,
an error shared by both would pass that comparison, so every system is also
solved one at a time by the CPU oracle and compared at 1e-13 relative.  Two
calls in a row with different sizes check that the shared scratch carries
nothing from one call into the next.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(rng, n, nbatch):
    a = rng.uniform(-1.0, 1.0, (nbatch, n))
    c = rng.uniform(-1.0, 1.0, (nbatch, n))
    b = 2.5 + rng.uniform(0.0, 1.0, (nbatch, n))
    r = rng.uniform(-1.0, 1.0, (nbatch, n))
    return r, a, b, c


def _noalloc(r, a, b, c):
    import torch
    import vring_b200 as V
    nbatch, n = r.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    t = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (r, a, b, c)]
    sol = torch.empty_like(t[0])
    stream = torch.cuda.current_stream(dev)
    V.api.solve_lap_thom_noalloc(t[0].data_ptr(), sol.data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                                 t[3].data_ptr(), n, nbatch, stream.cuda_stream)
    stream.synchronize()
    return sol.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    import vring_b200 as V
    from oracle import oracle as O
    rng = np.random.default_rng(2024)
    for n, nbatch in ((64, 300), (257, 129)):
        r, a, b, c = _systems(rng, n, nbatch)
        ref = V.solve_lap_thom(r, a, b, c)
        got = _noalloc(r, a, b, c)
        tol = 1e-14 * np.abs(ref).max()
        assert np.abs(got - ref).max() <= tol, (n, nbatch, np.abs(got - ref).max())
        for k in range(nbatch):
            orc = O.solve_lap_thom(r[k], a[k], b[k], c[k])
            err = np.abs(got[k] - orc).max()
            assert err <= 1e-13 * np.abs(orc).max(), (n, nbatch, k, err)


def test_noalloc_rejects_more_than_its_scratch():
    import torch
    import vring_b200 as V
    n = 1024
    nbatch = V.api.THOM_NOALLOC_MAX // n + 1
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(V.VrError) as e:
        V.api.solve_lap_thom_noalloc(x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(),
                                     n, nbatch, 0)
    assert e.value.code == 11
