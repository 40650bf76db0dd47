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
