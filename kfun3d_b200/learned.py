"""The learned right preconditioner: network handle, graphs and training.

Thin host layer over include/kfun3d_b200.h part 3.  Device memory for
features, targets and outputs is held in torch CUDA tensors and passed to the
library as raw pointers; every kernel (forward, backward, Adam, the pair
features) is the library's own.
"""
import ctypes as C

import numpy as np

from .api import lib, last_error


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed ({rc}): {last_error()}")


def param_count():
    return int(lib().kfun3d_mpnn_param_count())


def layer_shapes():
    """[(out, kin, nreal, offset)] of the network's 16 weight matrices."""
    L = lib()
    res = []
    for k in range(16):
        o, ki, nr, off = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(L.kfun3d_mpnn_layer_shape(k, C.byref(o), C.byref(ki), C.byref(nr), C.byref(off)), "layer_shape")
        res.append((o.value, ki.value, nr.value, off.value))
    return res


def _fptr(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Graph:
    """Directed-edge graph of a mesh on the device (kfun3d_mpnn_graph_create)."""

    def __init__(self, mesh):
        self.mesh = mesh            # keeps the GEOMETRY alive
        self.nnodes = mesh.view.nnodes
        self.h = lib().kfun3d_mpnn_graph_create(mesh.g)
        if not self.h:
            raise RuntimeError(f"kfun3d_mpnn_graph_create failed: {last_error()}")

    def close(self):
        if self.h:
            lib().kfun3d_mpnn_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Network:
    """Handle of one network on the current CUDA device."""

    def __init__(self, seed=0, params=None):
        self.h = lib().kfun3d_mpnn_create(int(seed))
        if not self.h:
            raise RuntimeError(f"kfun3d_mpnn_create failed: {last_error()}")
        if params is not None:
            self.set_params(params)

    def close(self):
        if self.h:
            lib().kfun3d_mpnn_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # parameters
    def params(self):
        a = np.zeros(param_count(), np.float32)
        _check(lib().kfun3d_mpnn_get_params(self.h, _fptr(a), a.size), "get_params")
        return a

    def set_params(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        _check(lib().kfun3d_mpnn_set_params(self.h, _fptr(a), a.size), "set_params")

    def grad(self):
        a = np.zeros(param_count(), np.float32)
        _check(lib().kfun3d_mpnn_get_grad(self.h, _fptr(a), a.size), "get_grad")
        return a

    def zero_grad(self):
        _check(lib().kfun3d_mpnn_zero_grad(self.h), "zero_grad")

    def save(self, path):
        np.save(path, self.params())

    @classmethod
    def load(cls, path):
        return cls(params=np.load(path))

    # device passes (torch CUDA tensors)
    def forward(self, graph, x0):
        import torch
        out = torch.empty((graph.nnodes, 4), dtype=torch.float32, device=x0.device)
        torch.cuda.synchronize()
        _check(lib().kfun3d_mpnn_forward(self.h, graph.h, x0.data_ptr(), out.data_ptr()), "forward")
        return out

    def accumulate(self, graph, x0, target, weight):
        import torch
        torch.cuda.synchronize()
        loss = C.c_double(0.0)
        _check(lib().kfun3d_mpnn_accumulate(self.h, graph.h, x0.data_ptr(), target.data_ptr(), float(weight),
                                            C.byref(loss)), "accumulate")
        return loss.value

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        _check(lib().kfun3d_mpnn_adam_step(self.h, float(lr), float(beta1), float(beta2), float(eps)), "adam_step")

    def apply(self, graph, y, q):
        """z = y + s N([y/s, q]) on FP64 CUDA tensors of 4 * nodes."""
        import torch
        z = torch.empty_like(y)
        torch.cuda.synchronize()
        _check(lib().kfun3d_mpnn_apply(self.h, graph.h, y.data_ptr(), q.data_ptr(), z.data_ptr()), "apply")
        return z


def make_pair(y, q, x=None):
    """(x0 BF16 [N x 8], target FP32 [N x 4] or None) from FP64 CUDA vectors."""
    import torch
    n = y.numel() // 4
    x0 = torch.empty((n, 8), dtype=torch.bfloat16, device=y.device)
    tgt = torch.empty((n, 4), dtype=torch.float32, device=y.device) if x is not None else None
    torch.cuda.synchronize()
    _check(lib().kfun3d_mpnn_make_pair(n, y.data_ptr(), q.data_ptr(), x.data_ptr() if x is not None else None,
                                       x0.data_ptr(), tgt.data_ptr() if tgt is not None else None), "make_pair")
    return x0, tgt


# ---------------------------------------------------------------- training

class Sample:
    """Pairs of one mesh kept on the device, with its graph."""

    def __init__(self, mesh, graph, x0, target, aoa, bump, stats):
        self.mesh, self.graph, self.x0, self.target = mesh, graph, x0, target
        self.aoa, self.bump, self.stats = aoa, bump, stats

    def __len__(self):
        return int(self.x0.shape[0])


def training_set(workdir, n_meshes=128, n=40, seed=0, stride=-3, cap=160, bump=(0.05, 0.15), aoa=(0.0, 6.0),
                 log=None, **params):
    """Seeded Kuhn-box meshes (n^3 nodes, bump height and angle of attack drawn
    uniformly from the given ranges), each solved from free stream by the
    ILU(0)-FGMRES solve writing training pairs on the GPU
    (kfun3d_collect_pairs).  The solver's device mirror of each mesh is
    released afterwards; its graph and pairs stay on the device."""
    import os
    from .api import Mesh, generate_mesh, set_aoa, get_aoa
    os.makedirs(workdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    p = dict(ts_max=20, stop_ratio=1e8)
    p.update(params)
    keep_aoa = get_aoa()
    out = []
    try:
        for i in range(n_meshes):
            b = float(rng.uniform(*bump))
            a = float(rng.uniform(*aoa))
            path = os.path.join(workdir, f"train_{n}_{seed}_{i}.msh")
            generate_mesh(path, n, bump_height=b, seed=int(rng.integers(1 << 31)))
            m = Mesh(path)
            os.remove(path)
            set_aoa(a)
            x0, tgt, st = m.collect_pairs(stride=stride, cap=cap, **p)
            g = Graph(m)
            m.release_device()
            out.append(Sample(m, g, x0, tgt, a, b, st))
            if log:
                log(f"mesh {i}: aoa {a:.2f} bump {b:.3f} pairs {len(x0)} its {st['gmres_its']}")
    finally:
        set_aoa(keep_aoa)
    return out


def train(net, data, steps, batch=8, lr=1e-3, seed=0, log=None, log_every=100, by_mesh=False):
    """Adam on the mean squared error over pairs: each step draws `batch`
    pairs at random (the kernels accumulate their gradients), then one Adam
    step.  by_mesh: the batch is `batch` different meshes, one pair drawn
    from each.  Returns the per-step loss."""
    rng = np.random.default_rng(seed)
    index = [(k, j) for k, s in enumerate(data) for j in range(len(s))]
    if not index:
        raise ValueError("no training pairs")
    meshes = [k for k, s in enumerate(data) if len(s)]
    losses = []
    for it in range(steps):
        if by_mesh:
            ks = rng.choice(len(meshes), size=min(batch, len(meshes)), replace=False)
            pick = [(meshes[k], int(rng.integers(len(data[meshes[k]])))) for k in ks]
        else:
            pick = [index[q] for q in rng.choice(len(index), size=min(batch, len(index)), replace=False)]
        loss = 0.0
        for k, j in pick:
            s = data[k]
            loss += net.accumulate(s.graph, s.x0[j], s.target[j], 1.0 / (len(pick) * 4 * s.graph.nnodes))
        net.adam_step(lr=lr)
        losses.append(loss)
        if log and (it % log_every == 0 or it == steps - 1):
            log(f"step {it}: loss {np.mean(losses[-log_every:]):.4e}")
    return losses


def zero_loss(data):
    """Loss of the zero correction (plain ILU(0)) over all pairs: the scale
    against which a trained loss is read."""
    tot, cnt = 0.0, 0
    for s in data:
        for j in range(len(s)):
            tot += float((s.target[j].double() ** 2).sum()) / (4 * s.graph.nnodes)
            cnt += 1
    return tot / max(cnt, 1)
