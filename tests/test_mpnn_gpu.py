"""Tensor-core (tcgen05) kernels of the learned preconditioner against CPU oracles.

* The GEMM tile, the building block of every layer: BF16 operands staged in
  shared memory, FP32 accumulators in tensor memory; it must equal the
  float64 product of the same BF16 values up to FP32 accumulation rounding.
* The network's forward pass against the float64 restatement with the same
  BF16 storage points (oracle/mpnn_ref.py), its weight gradients against CPU
  autograd in float64, one Adam step against an FP32 restatement, and the
  features of a training pair.
"""
import ctypes as C

import numpy as np
import pytest

import kfun3d_b200 as kf

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,K,N", [(128, 16, 16), (200, 32, 32), (128, 64, 80), (300, 80, 32),
                                      (1000, 128, 128), (77, 48, 64)])
def test_umma_tile_matches_cpu_product(rows, K, N):
    import torch
    L = kf.lib()
    g = torch.Generator().manual_seed(rows * 7 + K + N)
    X = torch.randn(rows, K, generator=g).to(torch.bfloat16)
    Wt = torch.randn(N, K, generator=g).to(torch.bfloat16)
    ref = X.double() @ Wt.double().T
    dX, dW = X.cuda(), Wt.cuda()
    dY = torch.full((rows, N), float("nan"), device="cuda")
    torch.cuda.synchronize()
    rc = L.kfun3d_umma_selftest(dX.data_ptr(), dW.data_ptr(), dY.data_ptr(), rows, K, N)
    assert rc == 0, kf.last_error()
    Y = dY.cpu().double()
    scale = X.double().abs() @ Wt.double().abs().T
    assert torch.all((Y - ref).abs() <= 1e-5 * scale + 1e-30), float(((Y - ref).abs() / scale).max())


# ---------------------------------------------------------------- the network

def _setup(box_mesh, n=6, seed=11):
    import torch
    from kfun3d_b200 import learned
    from oracle import mpnn_ref
    m = kf.Mesh(box_mesh(n, seed=seed))
    g_dev = learned.Graph(m)
    g_ref = mpnn_ref.Graph(m.view)
    rng = np.random.default_rng(seed)
    N = m.view.nnodes
    x0 = mpnn_ref.bf16_np(rng.standard_normal((N, 8)))
    tgt = (0.3 * rng.standard_normal((N, 4))).astype(np.float32)
    x0_d = torch.from_numpy(x0).to(torch.bfloat16).cuda()
    tgt_d = torch.from_numpy(tgt).cuda()
    return m, g_dev, g_ref, x0, tgt, x0_d, tgt_d


def test_forward_matches_oracle(box_mesh):
    from kfun3d_b200 import learned
    from oracle import mpnn_ref
    m, g_dev, g_ref, x0, tgt, x0_d, tgt_d = _setup(box_mesh)
    net = learned.Network(seed=5)
    th = net.params()
    out = net.forward(g_dev, x0_d).cpu().numpy().astype(np.float64)
    _, Ws = mpnn_ref.weights(th)
    ref = mpnn_ref.forward(Ws, g_ref, x0, rnd=True).numpy()
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    # same BF16 storage points; only FP32 accumulation order differs
    assert err < 1e-2, err


@pytest.mark.parametrize("n", [6, 14])
def test_fused_message_sum_is_bit_identical(box_mesh, n, monkeypatch):
    """Inference sums each node's messages inside the edge MLP's epilogue
    (tiles of whole nodes); the result equals the path that writes the
    messages to memory and sums them in the node MLP's gather, bit for bit."""
    from kfun3d_b200 import learned
    m, g_dev, g_ref, x0, tgt, x0_d, tgt_d = _setup(box_mesh, n=n, seed=17)
    net = learned.Network(seed=7)
    fused = net.forward(g_dev, x0_d).cpu().numpy()
    monkeypatch.setenv("KFUN3D_MPNN_FUSED", "0")
    g_plain = learned.Graph(m)
    plain = net.forward(g_plain, x0_d).cpu().numpy()
    assert np.array_equal(fused, plain)
    assert np.all(np.isfinite(fused)) and np.abs(fused).max() > 0


def test_gradient_matches_cpu_autograd(box_mesh):
    from kfun3d_b200 import learned
    from oracle import mpnn_ref
    m, g_dev, g_ref, x0, tgt, x0_d, tgt_d = _setup(box_mesh, n=7, seed=12)
    net = learned.Network(seed=6)
    # scale up the output layer (initialised small) so every layer carries gradient
    th = net.params()
    o, k, nr, off = learned.layer_shapes()[15]
    th[off:off + o * k] *= 10.0
    net.set_params(th)
    w = 1.0 / (4 * m.view.nnodes)
    net.zero_grad()
    loss = net.accumulate(g_dev, x0_d, tgt_d, w)
    g = net.grad().astype(np.float64)
    loss_ref, gr = mpnn_ref.loss_and_grad(th, g_ref, x0, tgt, w)
    assert abs(loss - loss_ref) <= 2e-2 * loss_ref, (loss, loss_ref)
    # BF16 activations and gradients against float64: overall and per layer
    cos = g @ gr / (np.linalg.norm(g) * np.linalg.norm(gr))
    assert cos > 0.999, cos
    assert np.linalg.norm(g - gr) / np.linalg.norm(gr) < 3e-2
    for L, (o, k, nr, off) in enumerate(learned.layer_shapes()):
        a, b = g[off:off + o * k], gr[off:off + o * k]
        assert np.linalg.norm(a - b) <= 0.1 * np.linalg.norm(b) + 1e-12, L
        # padding columns (after the ones feature) carry no gradient
        assert np.all(a.reshape(o, k)[:, nr + 1:] == 0.0), L


def test_adam_step_matches_oracle(box_mesh):
    from kfun3d_b200 import learned
    from oracle import mpnn_ref
    m, g_dev, g_ref, x0, tgt, x0_d, tgt_d = _setup(box_mesh, n=6, seed=13)
    net = learned.Network(seed=7)
    th = net.params()
    net.zero_grad()
    net.accumulate(g_dev, x0_d, tgt_d, 1.0 / (4 * m.view.nnodes))
    g = net.grad()
    net.adam_step(lr=1e-3)
    th1 = net.params()
    ref, _, _ = mpnn_ref.adam(th, np.zeros_like(th), np.zeros_like(th), g, 1, 1e-3)
    # the same FP32 operations in the same order, each rounded on its own
    bad = np.flatnonzero(th1 != ref)
    assert bad.size == 0, (bad[:5], th1[bad[:5]], ref[bad[:5]], g[bad[:5]])
    assert np.all(net.grad() == 0.0)   # cleared by the step


def test_training_reduces_loss(box_mesh):
    from kfun3d_b200 import learned
    m, g_dev, g_ref, x0, tgt, x0_d, tgt_d = _setup(box_mesh, n=6, seed=14)
    net = learned.Network(seed=8)
    w = 1.0 / (4 * m.view.nnodes)
    losses = []
    for it in range(60):
        losses.append(net.accumulate(g_dev, x0_d, tgt_d, w))
        net.adam_step(lr=3e-3)
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])


def test_pair_features_and_apply(box_mesh):
    import torch
    from kfun3d_b200 import learned
    from oracle import mpnn_ref
    m = kf.Mesh(box_mesh(6, seed=15))
    N = m.view.nnodes
    rng = np.random.default_rng(15)
    y = rng.standard_normal(4 * N) * 1e-3
    q = m.view.q.copy() + rng.uniform(-0.05, 0.05, 4 * N)
    x = y + rng.standard_normal(4 * N) * 1e-4
    yd, qd, xd = (torch.from_numpy(a).cuda() for a in (y, q, x))
    x0, tgt = learned.make_pair(yd, qd, xd)
    x0_ref, s = mpnn_ref.features(y, q)
    a = x0.float().cpu().numpy().astype(np.float64)
    # s is a device tree sum: at most one BF16 unit of difference
    assert np.all(np.abs(a - x0_ref) <= 2.0 ** -7 * np.abs(x0_ref) + 1e-30)
    assert np.allclose(tgt.cpu().numpy(), ((x - y) / s).reshape(-1, 4).astype(np.float32), rtol=1e-5, atol=1e-9)
    net = learned.Network(seed=9)
    g_dev = learned.Graph(m)
    z = net.apply(g_dev, yd, qd).cpu().numpy()
    out = net.forward(g_dev, x0).cpu().numpy().astype(np.float64).reshape(-1)
    assert np.allclose(z, y + s * out, rtol=1e-9, atol=1e-15)
