"""The learned preconditioner's network (vr_unet_*): the GPU forward pass and
gradients against the CPU restatement (oracle/unet_ref.py, FP64 with the
same BF16 rounding points), training through the project's own kernels,
and the trained network's effect on the VR2D Krylov solve.

Tolerances: forward output and every gradient within 5e-3 relative L2 of the
oracle's (the GPU accumulates in FP32; an FP32 sum that lands on the other
side of a BF16 rounding boundary changes that element by one BF16 ulp,
2^-8)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CH = (8, 16, 16, 24)
WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "vring_b200", "data",
                       "unet_vr2d_512x1024.npz")


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def test_forward_matches_oracle():
    import vring_b200 as V
    from oracle import unet_ref as U
    nr, nz = 32, 64
    net = V.UNet(nr, nz, CH, seed=5)
    assert net.nparams == U.nparams(CH)
    w = net.get_params()
    x = np.random.default_rng(0).standard_normal((nr, nz))
    s = np.sqrt(np.mean(x ** 2))
    y = net.forward(x)
    yo = s * U.forward(w, CH, x / s)
    print("forward rel L2 vs oracle %.2e" % _rel(y, yo))
    assert _rel(y, yo) <= 5e-3
    # homogeneous: N(3 x) = 3 N(x)
    assert _rel(net.forward(3 * x), 3 * y) <= 1e-12
    net.close()


@pytest.mark.parametrize("grid", [(32, 64), (64, 128)])
def test_tensor_core_forward_matches_cuda_core_forward_and_oracle(grid):
    """The tcgen05 implicit-GEMM convolutions against the CUDA-core ones and
    the oracle, on the network the preconditioner uses (16, 32, 48, 64)."""
    import vring_b200 as V
    from oracle import unet_ref as U
    nr, nz = grid
    ch = (16, 32, 48, 64)
    pool = 2 if nr < 64 else 4
    tc = V.UNet(nr, nz, ch, seed=9, pool=pool)
    cc = V.UNet(nr, nz, ch, seed=9, flags=V.UNet.CUDA_CORES, pool=pool)
    w = tc.get_params()
    assert np.array_equal(w, cc.get_params())
    x = np.random.default_rng(4).standard_normal((nr, nz))
    s = np.sqrt(np.mean(x ** 2))
    yt, yc = tc.forward(x), cc.forward(x)
    yo = s * U.forward(w, ch, x / s, F=pool)
    print("%s: tensor cores vs oracle %.2e, CUDA cores vs oracle %.2e, between %.2e"
          % (grid, _rel(yt, yo), _rel(yc, yo), _rel(yt, yc)))
    assert _rel(yt, yo) <= 5e-3 and _rel(yc, yo) <= 5e-3
    tc.close()
    cc.close()


@pytest.mark.parametrize("pool", [2, 4])
def test_gradients_match_oracle(pool):
    import vring_b200 as V
    from oracle import unet_ref as U
    nr, nz = (32, 64) if pool == 2 else (64, 128)
    net = V.UNet(nr, nz, CH, seed=6, pool=pool)
    w = net.get_params()
    rng = np.random.default_rng(1)
    x, g = rng.standard_normal((nr, nz)), rng.standard_normal((nr, nz))
    dw, dx = net.backward(x, g)
    dwo, dxo = U.backward(w, CH, x, g, F=pool)
    off = 0
    for i, (ci, co, _) in enumerate(U.layers(CH) + [(CH[0], 1, 0)]):
        n = ci * co * (9 if i < 14 else 1)
        e = _rel(dw[off:off + n], dwo[off:off + n])
        assert e <= 5e-3, (i, e)
        off += n
    print("dw rel L2 %.2e, dx rel L2 %.2e" % (_rel(dw, dwo), _rel(dx, dxo)))
    assert _rel(dx, dxo) <= 5e-3
    net.close()


def test_training_reduces_the_loss():
    import torch
    import vring_b200 as V
    from vring_b200 import learned as Lr
    nr, nz = 64, 128
    k = V.K2d(Lr.tanh_faces(nr), nz, 15.0)
    net = V.UNet(nr, nz, CH, seed=7)
    rng = np.random.default_rng(2)
    d = 1.0 / np.sqrt(k.diag()).ravel(order="F")
    e = torch.from_numpy(rng.standard_normal((4, nr * nz)) * d[None, :]).cuda()
    torch.cuda.synchronize()
    l0 = net.train_step(k, e.data_ptr(), 4, 3e-3)
    for _ in range(30):
        l1 = net.train_step(k, e.data_ptr(), 4, 3e-3)
    print("loss %.4e -> %.4e" % (l0, l1))
    assert np.isfinite(l1) and l1 < 0.5 * l0
    net.close()
    k.close()


@pytest.mark.timeout(600)
def test_training_on_solver_triples_cuts_iterations_small_grid():
    """Train the network from scratch on a 64 x 128 stretched grid with the
    project's kernels (residuals of the seeded triples, smooth and white
    residuals), then solve one triple: the learned flexible CG converges to
    the plain CG's field and needs fewer iterations than plain CG and than
    the same flexible CG with the Jacobi steps alone."""
    import vring_b200 as V
    from vring_b200 import learned as Lr
    nr, nz = 64, 128
    k = V.K2d(Lr.tanh_faces(nr), nz, Lr.ZMAX)
    net = V.UNet(nr, nz, Lr.CHANNELS, seed=1, pool=2)
    losses = Lr.train(net, k, 300, batch=4, lr=3e-3, lr_final=3e-4)
    print("loss %.3e -> %.3e" % (losses[0], np.mean(losses[-20:])))
    assert np.mean(losses[-20:]) < 0.5 * losses[0]
    seq = Lr.RingSequence(2, k.faces, nz, Lr.ZMAX)
    f, p_prev, p = Lr.triple(k, seq, 500)
    res = Lr.compare(k, net, f, x0=p_prev, tol=1e-10, maxit=4000)
    for m, (it, rr, ms, x) in res.items():
        print("%s: %d iterations, relres %.2e, %.1f ms, max|x - direct| / max|direct| %.2e"
              % (m, it, rr, ms, np.abs(x - p).max() / np.abs(p).max()))
        assert rr <= 1e-10
        assert np.abs(x - p).max() <= 1e-8 * np.abs(p).max()
    assert res["learned"][0] < res["cg"][0]
    assert res["learned"][0] < res["fcg_jacobi"][0]     # the network's own gain
    net.close()
    k.close()


@pytest.mark.timeout(900)
@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained weights committed")
def test_trained_network_cuts_vr2d_iterations_3x():
    """The committed network (trained on the GPU on the 512 x 1024 stretched
    grid) in the flexible CG against plain CG on a triple of seed 2: the same
    converged field, at least 3x fewer iterations, and fewer than the same
    flexible CG without the network."""
    import vring_b200 as V
    from vring_b200 import learned as Lr
    k = V.K2d(Lr.tanh_faces(Lr.NR), Lr.NZ, Lr.ZMAX)
    net = Lr.make_net()
    Lr.load_weights(net)
    seq = Lr.RingSequence(2, k.faces, Lr.NZ, Lr.ZMAX)
    f, p_prev, p = Lr.triple(k, seq, 500)
    res = Lr.compare(k, net, f, x0=p_prev, tol=1e-10, maxit=20000)
    for m, (it, rr, ms, x) in res.items():
        print("%s: %d iterations, relres %.2e, %.1f ms, max|x - direct| / max|direct| %.2e"
              % (m, it, rr, ms, np.abs(x - p).max() / np.abs(p).max()))
        assert rr <= 1e-10
        assert np.abs(x - p).max() <= 1e-8 * np.abs(p).max()
    assert res["cg"][0] >= 3 * res["learned"][0]
    assert res["learned"][0] < res["fcg_jacobi"][0]
    net.close()
    k.close()
