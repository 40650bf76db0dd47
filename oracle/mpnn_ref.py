"""Test infrastructure only: float64 CPU restatement of the learned preconditioner.

The network has no reference counterpart; this module is its oracle.  It
restates, in PyTorch CPU float64 with autograd, the message-passing network
that ``kfun3d_b200/csrc/mpnn.cu`` evaluates and trains on tensor cores:

* directed edges are the node-incidence rows of the mesh, node by node, each
  node's rows in edge order (the order ``kfun3d_mpnn_graph_create`` builds);
* every linear map is ``X~ W~^T`` with ``X~ = [X, 1, 0 ...]`` (bias = the
  column of ``W~`` at index ``nreal``);
* ``rnd=True`` rounds to BF16 wherever the kernels store BF16 (edge
  features, node features, hidden activations, node states, messages and
  their sums), so the forward pass matches the kernels up to FP32
  accumulation order; ``rnd=False`` keeps float64 throughout, which is the
  function whose gradient the kernels' backward pass approximates.

The product never imports this module.
"""
import numpy as np
import torch

# (out, kin, nreal) per layer: enc1, enc2, [edge1, edge2, node1, node2] x 3, dec1, dec2
SHAPES = ([(32, 16, 8), (32, 48, 32)]
          + [(32, 80, 68), (32, 48, 32), (32, 80, 64), (32, 48, 32)] * 3
          + [(32, 48, 32), (16, 48, 32)])
OFFSETS = np.concatenate([[0], np.cumsum([o * k for o, k, _ in SHAPES])]).astype(np.int64)
NPARAM = int(OFFSETS[-1])
ENC1, DEC1 = 0, 14


def edge1(l):
    return 2 + 4 * l


def node1(l):
    return 4 + 4 * l


def bf16(x):
    """Round to BF16 (round to nearest even) through FP32, as the kernels do."""
    return x.to(torch.float32).to(torch.bfloat16).to(torch.float64)


def bf16_np(a):
    return bf16(torch.from_numpy(np.asarray(a, dtype=np.float64))).numpy()


class Graph:
    """Directed-edge graph of a GEOMETRY view (kfun3d_mpnn_graph_create)."""

    def __init__(self, view):
        N, E = view.nnodes, view.nedges
        n0 = view.n0.astype(np.int64)
        n1 = view.n1.astype(np.int64)
        cnt = np.bincount(n0, minlength=N) + np.bincount(n1, minlength=N)
        seg = np.zeros(N + 1, np.int64)
        seg[1:] = np.cumsum(cnt)
        pos = seg[:-1].copy()
        R = 2 * E
        rnode = np.zeros(R, np.int64)
        oth = np.zeros(R, np.int64)
        rev = np.zeros(R, np.int64)
        sgn = np.zeros(R)
        eid = np.zeros(R, np.int64)
        for e in range(E):
            a, b = n0[e], n1[e]
            ka = pos[a]; pos[a] += 1
            kb = pos[b]; pos[b] += 1
            rnode[ka], oth[ka], rev[ka], sgn[ka], eid[ka] = a, b, kb, 1.0, e
            rnode[kb], oth[kb], rev[kb], sgn[kb], eid[kb] = b, a, ka, -1.0, e
        amean = float(np.mean(view.area)) if E else 1.0
        ef = np.stack([sgn * view.xn[eid], sgn * view.yn[eid], sgn * view.zn[eid],
                       view.area[eid] / amean], axis=1)
        self.N, self.R = N, R
        self.seg, self.rnode, self.oth, self.rev = seg, rnode, oth, rev
        self.efeat = torch.from_numpy(bf16_np(ef))
        self.rnode_t = torch.from_numpy(rnode)
        self.oth_t = torch.from_numpy(oth)


def weights(theta, requires_grad=False):
    """BF16-rounded W~ matrices from the FP32 master vector."""
    th = bf16(torch.from_numpy(np.asarray(theta, dtype=np.float32).astype(np.float64)))
    th = th.clone().requires_grad_(requires_grad)
    Ws = [th[OFFSETS[L]:OFFSETS[L + 1]].view(o, k) for L, (o, k, _) in enumerate(SHAPES)]
    return th, Ws


def _aug(X, kin):
    """[X, 1, 0 ...] with kin columns."""
    n = X.shape[0]
    pad = torch.zeros(n, kin - X.shape[1], dtype=X.dtype)
    pad[:, 0] = 1.0
    return torch.cat([X, pad], dim=1)


def _mlp(X, W1, W2, rnd):
    H = torch.relu(_aug(X, W1.shape[1]) @ W1.T)
    if rnd:
        H = bf16(H)
    return _aug(H, W2.shape[1]) @ W2.T


def forward(Ws, g, x0, rnd=True):
    """out [N x 4] of the network for node features x0 [N x 8] (BF16 values)."""
    x0 = torch.as_tensor(x0, dtype=torch.float64)
    r = bf16 if rnd else (lambda t: t)
    h = r(_mlp(x0, Ws[0], Ws[1], rnd))
    seg = torch.from_numpy(g.seg)
    owner = torch.repeat_interleave(torch.arange(g.N), seg[1:] - seg[:-1])
    for l in range(3):
        Xe = torch.cat([h[g.rnode_t], h[g.oth_t], g.efeat], dim=1)
        m = r(_mlp(Xe, Ws[edge1(l)], Ws[edge1(l) + 1], rnd))
        agg = r(torch.zeros(g.N, 32, dtype=torch.float64).index_add(0, owner, m))
        Xn = torch.cat([h, agg], dim=1)
        h = r(h + _mlp(Xn, Ws[node1(l)], Ws[node1(l) + 1], rnd))
    out = _mlp(h, Ws[DEC1], Ws[DEC1 + 1], rnd)
    if rnd:
        out = out.to(torch.float32).to(torch.float64)
    return out[:, :4]


def loss_and_grad(theta, g, x0, target, weight):
    """weight * sum (N(x0) - target)^2 in float64 (no BF16 rounding of
    activations) and its gradient with respect to the BF16 weights."""
    th, Ws = weights(theta, requires_grad=True)
    out = forward(Ws, g, x0, rnd=False)
    t = torch.as_tensor(target, dtype=torch.float64)
    loss = weight * ((out - t) ** 2).sum()
    loss.backward()
    return float(loss.detach()), th.grad.numpy().copy()


def adam(theta, m, v, grad, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step in FP32 (the kernel's arithmetic), returns new (theta, m, v)."""
    f = np.float32
    theta, m, v, grad = (np.asarray(a, np.float32) for a in (theta, m, v, grad))
    b1f, b2f = f(b1), f(b2)
    c1 = f(1.0 - b1 ** step)          # formed in double, rounded once
    c2 = f(1.0 - b2 ** step)
    m2 = b1f * m + (f(1.0) - b1f) * grad
    v2 = b2f * v + ((f(1.0) - b2f) * grad) * grad
    th2 = theta - (f(lr) * (m2 / c1)) / (np.sqrt(v2 / c2) + f(eps))
    return th2.astype(np.float32), m2.astype(np.float32), v2.astype(np.float32)


def features(y, q):
    """x0 = BF16([y/s, q]) with s = RMS(y) (kfun3d_mpnn_make_pair)."""
    y = np.asarray(y, np.float64).reshape(-1, 4)
    q = np.asarray(q, np.float64).reshape(-1, 4)
    s = np.sqrt(np.sum(y * y) / y.size)
    s = s if s > 0 else 1.0
    inv = np.float32(1.0 / s)
    a = y.astype(np.float32) * inv
    x0 = np.concatenate([a.astype(np.float64), q.astype(np.float32).astype(np.float64)], axis=1)
    return bf16_np(x0), s
