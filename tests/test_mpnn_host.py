"""Host-side checks of the learned preconditioner: the library's layer table
against the float64 oracle, the oracle's graph, and the oracle's gradient
against central differences (no GPU needed)."""
import numpy as np
import torch

import kfun3d_b200 as kf
from kfun3d_b200 import learned
from oracle import mpnn_ref


def test_layer_table_matches_oracle():
    assert learned.param_count() == mpnn_ref.NPARAM
    for L, (o, k, nr, off) in enumerate(learned.layer_shapes()):
        assert (o, k, nr) == mpnn_ref.SHAPES[L]
        assert off == mpnn_ref.OFFSETS[L]


def test_oracle_graph_structure(box_mesh):
    m = kf.Mesh(box_mesh(5, seed=4))
    g = mpnn_ref.Graph(m.view)
    assert g.R == 2 * m.view.nedges
    assert np.array_equal(g.rev[g.rev], np.arange(g.R))
    assert np.array_equal(g.rnode[g.rev], g.oth)
    owner = np.repeat(np.arange(g.N), np.diff(g.seg))
    assert np.array_equal(owner, g.rnode)
    # normals seen from the two ends are opposite
    ef = g.efeat.numpy()
    assert np.array_equal(ef[g.rev, :3], -ef[:, :3])


def test_oracle_gradient_against_differences(box_mesh):
    m = kf.Mesh(box_mesh(4, seed=5))
    g = mpnn_ref.Graph(m.view)
    rng = np.random.default_rng(0)
    th = mpnn_ref.bf16_np(0.2 * rng.standard_normal(mpnn_ref.NPARAM)).astype(np.float32)
    x0 = mpnn_ref.bf16_np(rng.standard_normal((g.N, 8)))
    tgt = rng.standard_normal((g.N, 4))
    _, grad = mpnn_ref.loss_and_grad(th, g, x0, tgt, 1.0)
    base = torch.from_numpy(th.astype(np.float64))

    def loss(v):
        Ws = [v[mpnn_ref.OFFSETS[L]:mpnn_ref.OFFSETS[L + 1]].view(o, k)
              for L, (o, k, _) in enumerate(mpnn_ref.SHAPES)]
        out = mpnn_ref.forward(Ws, g, x0, rnd=False)
        return float(((out - torch.from_numpy(tgt)) ** 2).sum())

    for idx in rng.choice(np.flatnonzero(grad), 12, replace=False):
        h = 1e-6
        vp, vm = base.clone(), base.clone()
        vp[idx] += h
        vm[idx] -= h
        fd = (loss(vp) - loss(vm)) / (2 * h)
        assert abs(fd - grad[idx]) <= 1e-4 * max(1.0, abs(grad[idx])), (idx, fd, grad[idx])
