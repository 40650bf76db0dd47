"""ctypes mirror of include/kfun3d_b200.h.

Function names and argument meanings follow the reference's C entry points
(inc/core_kernel.h:6-22, inc/utils.h:15-28, src/main.c:19 Kernel); the extra
``kfun3d_*`` calls cover settings, the native mesh loader/generator, the
parameterised solve and device timing.
"""
import ctypes as C
import os

import numpy as np

from .geometry import GEOMETRY, GRADIENT, GeometryView

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libkfun3d_b200.so")

KFUN3D_MODE_EXACT = 0
KFUN3D_MODE_FAST = 1


class SolverParams(C.Structure):
    _fields_ = [("ts_max", C.c_int), ("stop_ratio", C.c_double), ("gmres_rtol", C.c_double),
                ("gmres_restart", C.c_int), ("gmres_max_it", C.c_int), ("cfl_init", C.c_double),
                ("cfl_max", C.c_double)]


class Step(C.Structure):
    _fields_ = [("step", C.c_int), ("gmres_its", C.c_int), ("cfl", C.c_double),
                ("fnorm", C.c_double), ("lift", C.c_double), ("drag", C.c_double),
                ("momn", C.c_double), ("seconds", C.c_double)]


class FlexStats(C.Structure):
    _fields_ = [("newton_steps", C.c_int), ("gmres_its", C.c_int), ("learned_its", C.c_int),
                ("fallback_solves", C.c_int), ("rejected_steps", C.c_int), ("disabled", C.c_int),
                ("pairs", C.c_int), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MeshSpec(C.Structure):
    _fields_ = [("n", C.c_uint), ("bump_height", C.c_double), ("bump_sigma", C.c_double),
                ("jitter", C.c_double), ("seed", C.c_ulonglong), ("permute", C.c_int)]


_lib = None


def lib():
    """Load the native library; raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C kfun3d_b200/csrc` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    P, D, G = C.POINTER, C.POINTER(C.c_double), C.POINTER(GEOMETRY)
    sig = {
        "ComputeA": (None, [G]),
        "ComputeTimeStep": (None, [C.c_double, G]),
        "ComputeFlux": (None, [G, D, P(GRADIENT), D]),
        "ComputeForces": (None, [G, D]),
        "ComputeNumericalILU": (None, [G]),
        "ComputeSparseTriangularSolve": (None, [G, D, D]),
        "Compute2ndNorm": (C.c_double, [C.c_size_t, D]),
        "ComputeAXPY": (None, [C.c_size_t, C.c_double, D, D]),
        "ComputeNewAXPY": (None, [C.c_size_t, C.c_double, D, D, D]),
        "Normalize": (C.c_double, [C.c_size_t, D]),
        "Kernel": (None, [G]),
        "CXX_Matrix_Init": (C.c_void_p, [C.c_size_t, C.c_size_t, C.c_uint, C.c_uint,
                                         P(C.c_uint), P(C.c_uint)]),
        "CXX_Matrix_Delete": (None, [C.c_void_p]),
        "CXX_METIS": (None, [C.c_uint, P(C.c_uint), C.c_void_p]),
        "CXX_Walk_Int": (None, [C.c_char_p, C.c_char_p, C.c_size_t, P(C.c_uint)]),
        "CXX_Walk_Double": (None, [C.c_char_p, C.c_char_p, C.c_size_t, D]),
        "kfun3d_gpu_last_status": (C.c_int, []),
        "kfun3d_gpu_last_error": (C.c_char_p, []),
        "kfun3d_clear_status": (None, []),
        "kfun3d_set_abort_on_error": (None, [C.c_int]),
        "kfun3d_set_aoa": (None, [C.c_double]),
        "kfun3d_get_aoa": (C.c_double, []),
        "kfun3d_get_freestream": (None, [D, D]),
        "kfun3d_set_mode": (None, [C.c_int]),
        "kfun3d_get_mode": (C.c_int, []),
        "kfun3d_set_precision": (None, [C.c_int]),
        "kfun3d_set_ilu_order": (None, [C.c_int]),
        "kfun3d_get_ilu_order": (C.c_int, []),
        "kfun3d_ilu_rank": (C.c_long, [G, C.POINTER(C.c_uint)]),
        "kfun3d_ilu_order_plan": (C.c_int, [G, C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_uint),
                                            C.POINTER(C.c_uint)]),
        "kfun3d_set_schwarz": (None, [C.c_uint]),
        "kfun3d_get_schwarz": (C.c_uint, []),
        "kfun3d_schwarz_partition": (C.c_int, [G, C.c_uint, C.POINTER(C.c_uint)]),
        "kfun3d_set_first_order": (None, [C.c_int]),
        "kfun3d_set_verbose": (None, [C.c_int]),
        "kfun3d_default_params": (None, [P(SolverParams)]),
        "kfun3d_solve": (C.c_int, [G, P(SolverParams), P(Step), C.c_int]),
        "kfun3d_setup_load": (G, [C.c_char_p]),
        "kfun3d_setup_free": (None, [G]),
        "kfun3d_initial_guess": (None, [G]),
        "kfun3d_mesh_generate": (C.c_int, [C.c_char_p, P(MeshSpec)]),
        "kfun3d_time_kernel": (C.c_double, [G, C.c_int, C.c_int]),
        "kfun3d_launch_count": (C.c_ulonglong, []),
        "kfun3d_reset_launch_count": (None, []),
        "kfun3d_device_release": (None, [G]),
        "kfun3d_check_bounded_wait": (C.c_int, []),
        "kfun3d_device_query": (C.c_long, [G, C.c_char_p]),
        "kfun3d_matrix_read": (C.c_long, [G, P(C.c_uint), P(C.c_uint), D]),
        "kfun3d_time_solve": (C.c_double, [G, P(SolverParams), C.c_int, P(Step), C.c_int, P(C.c_int)]),
        # learned preconditioner (include/kfun3d_b200.h, part 3)
        "kfun3d_mpnn_param_count": (C.c_size_t, []),
        "kfun3d_mpnn_layer_shape": (C.c_int, [C.c_int, P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_int)]),
        "kfun3d_mpnn_create": (C.c_void_p, [C.c_ulonglong]),
        "kfun3d_mpnn_free": (None, [C.c_void_p]),
        "kfun3d_mpnn_set_params": (C.c_int, [C.c_void_p, P(C.c_float), C.c_size_t]),
        "kfun3d_mpnn_get_params": (C.c_int, [C.c_void_p, P(C.c_float), C.c_size_t]),
        "kfun3d_mpnn_get_grad": (C.c_int, [C.c_void_p, P(C.c_float), C.c_size_t]),
        "kfun3d_mpnn_zero_grad": (C.c_int, [C.c_void_p]),
        "kfun3d_mpnn_graph_create": (C.c_void_p, [G]),
        "kfun3d_mpnn_graph_free": (None, [C.c_void_p]),
        "kfun3d_mpnn_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "kfun3d_mpnn_accumulate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                             P(C.c_double)]),
        "kfun3d_mpnn_adam_step": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double]),
        "kfun3d_mpnn_make_pair": (C.c_int, [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p]),
        "kfun3d_mpnn_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "kfun3d_umma_selftest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
        "kfun3d_time_learned_apply": (C.c_double, [G, C.c_void_p, C.c_int]),
        "kfun3d_solve_flexible": (C.c_int, [G, P(SolverParams), C.c_void_p, P(Step), C.c_int, P(FlexStats)]),
        "kfun3d_collect_pairs": (C.c_int, [G, P(SolverParams), C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                           P(FlexStats)]),
        "kfun3d_time_solve_flexible": (C.c_double, [G, P(SolverParams), C.c_void_p, C.c_int, P(Step), C.c_int,
                                                    P(C.c_int), P(FlexStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _d(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ---------------------------------------------------------------- settings

def set_aoa(deg):
    lib().kfun3d_set_aoa(float(deg))


def get_aoa():
    return lib().kfun3d_get_aoa()


def freestream():
    u, v = C.c_double(), C.c_double()
    lib().kfun3d_get_freestream(C.byref(u), C.byref(v))
    return u.value, v.value


def set_mode(mode):
    if isinstance(mode, str):
        mode = {"exact": KFUN3D_MODE_EXACT, "fast": KFUN3D_MODE_FAST}[mode]
    lib().kfun3d_set_mode(int(mode))


def get_mode():
    return lib().kfun3d_get_mode()


def set_precision(p):
    if isinstance(p, str):
        p = {"fp64": 0, "fp32": 1, "mixed": 1}[p]
    lib().kfun3d_set_precision(int(p))


def set_ilu_order(order):
    """Elimination order of ILU(0): 0 / "mesh" (the reference) or 1 / "spatial"
    (the block pattern renumbered by sweeps of the node coordinates; not a parity path)."""
    if isinstance(order, str):
        order = {"mesh": 0, "spatial": 1}[order]
    lib().kfun3d_set_ilu_order(int(order))


def get_ilu_order():
    return lib().kfun3d_get_ilu_order()


def set_schwarz(parts):
    """Additive Schwarz without overlap on one device: ILU(0) of each of `parts`
    subdomains (recursive coordinate bisection) on its own; 0 or 1 turns it off."""
    lib().kfun3d_set_schwarz(int(parts))


def get_schwarz():
    return lib().kfun3d_get_schwarz()


def set_first_order(on):
    lib().kfun3d_set_first_order(int(bool(on)))


def set_verbose(on):
    lib().kfun3d_set_verbose(int(bool(on)))


def last_status():
    return lib().kfun3d_gpu_last_status()


def last_error():
    return lib().kfun3d_gpu_last_error().decode()


def clear_status():
    lib().kfun3d_clear_status()


def set_abort_on_error(on):
    lib().kfun3d_set_abort_on_error(int(bool(on)))


def launch_count():
    return lib().kfun3d_launch_count()


def reset_launch_count():
    lib().kfun3d_reset_launch_count()


def default_params(**kw):
    p = SolverParams()
    lib().kfun3d_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


# ---------------------------------------------------------------- meshes

def generate_mesh(path, n, bump_height=0.1, bump_sigma=0.15, jitter=0.2, seed=0, permute=True):
    """Write the seeded Kuhn-box mesh of the benchmark configurations (uns3d .msh)."""
    spec = MeshSpec(n, bump_height, bump_sigma, jitter, seed, int(permute))
    rc = lib().kfun3d_mesh_generate(os.fsencode(path), C.byref(spec))
    if rc != 0:
        raise RuntimeError(f"kfun3d_mesh_generate failed ({rc})")
    return path


class Mesh:
    """A GEOMETRY loaded by the native loader (kfun3d_setup_load)."""

    def __init__(self, path):
        L = lib()
        self.path = path
        self.g = L.kfun3d_setup_load(os.fsencode(path))
        if not self.g:
            raise IOError(f"cannot load {path}: {last_error()}")
        self.view = GeometryView(self.g)
        self.view.owner = self   # the arrays live as long as the view

    @property
    def nnodes(self):
        return self.view.nnodes

    @property
    def nedges(self):
        return self.view.nedges

    def close(self):
        if getattr(self, "g", None):
            lib().kfun3d_setup_free(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset_state(self):
        """Free-stream initial guess for the current angle of attack."""
        lib().kfun3d_initial_guess(self.g)

    # ---- the reference's entry points
    def flux(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        gx, gy, gz, r = (np.zeros(self.view.dofs) for _ in range(4))
        grad = GRADIENT(_d(gx), _d(gy), _d(gz))
        lib().ComputeFlux(self.g, _d(q), C.byref(grad), _d(r))
        return (gx, gy, gz), r

    def timestep(self, cfl, q=None):
        if q is not None:
            self.view.q[:] = q
        lib().ComputeTimeStep(float(cfl), self.g)
        return self.view.cdt.copy()

    def fill(self, q=None, cdt=None):
        if q is not None:
            self.view.q[:] = q
        if cdt is not None:
            self.view.cdt[:] = cdt
        lib().ComputeA(self.g)

    def ilu(self):
        lib().ComputeNumericalILU(self.g)

    def sptrsv(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        lib().ComputeSparseTriangularSolve(self.g, _d(b), _d(x))
        return x

    def forces(self, q=None):
        if q is not None:
            self.view.q[:] = q
        out = np.zeros(3)
        lib().ComputeForces(self.g, _d(out))
        return out

    def kernel(self):
        """The reference's Kernel(): full solve with its constants, updates q."""
        lib().Kernel(self.g)

    def solve(self, **params):
        p = default_params(**params)
        hist = (Step * 64)()
        n = lib().kfun3d_solve(self.g, C.byref(p), hist, 64)
        if n < 0:
            raise RuntimeError(f"kfun3d_solve failed: {last_error()}")
        return [dict(step=h.step, gmres_its=h.gmres_its, cfl=h.cfl, fnorm=h.fnorm, lift=h.lift,
                     drag=h.drag, momn=h.momn, seconds=h.seconds) for h in hist[:n]]

    def ilu_rank(self):
        """Row of every node in the spatial ILU order (built on first use of order 1)."""
        rank = np.zeros(self.view.nnodes, dtype=np.uint32)
        if lib().kfun3d_ilu_rank(self.g, rank.ctypes.data_as(C.POINTER(C.c_uint))) < 0:
            raise RuntimeError(f"kfun3d_ilu_rank failed: {last_error()}")
        return rank.astype(np.int64)

    def schwarz_partition(self, parts):
        """Host-only: subdomain of every node for `parts` additive Schwarz subdomains."""
        part = np.zeros(self.view.nnodes, dtype=np.uint32)
        if lib().kfun3d_schwarz_partition(self.g, int(parts), part.ctypes.data_as(C.POINTER(C.c_uint))) != 0:
            raise RuntimeError(f"kfun3d_schwarz_partition failed: {last_error()}")
        return part.astype(np.int64)

    def ilu_order_plan(self, tiles=148):
        """Host-only preview of the spatial ILU(0) order (no GPU): (rank, levels of the
        lower sweep, levels of the upper sweep) of the renumbered pattern."""
        rank = np.zeros(self.view.nnodes, dtype=np.uint32)
        nl, nu = C.c_uint(0), C.c_uint(0)
        if lib().kfun3d_ilu_order_plan(self.g, int(tiles), rank.ctypes.data_as(C.POINTER(C.c_uint)),
                                       C.byref(nl), C.byref(nu)) != 0:
            raise RuntimeError(f"kfun3d_ilu_order_plan failed: {last_error()}")
        return rank.astype(np.int64), nl.value, nu.value

    def query(self, key):
        """Device path in use (kfun3d_device_query): "sptrsv_schedule", "lsq_terms_match",
        "visit_order_copies", "mgs_resident"."""
        v = lib().kfun3d_device_query(self.g, key.encode())
        if v < 0:
            raise RuntimeError(f"kfun3d_device_query({key}) failed: {last_error()}")
        return int(v)

    def time_kernel(self, which, reps=10):
        names = {"flux": 0, "timestep": 1, "fill": 2, "ilu": 3, "sptrsv": 4, "gmres_iter": 5,
                 "mgs": 6, "gradient": 7, "edge_flux": 8}
        w = names.get(which, which)
        ms = lib().kfun3d_time_kernel(self.g, int(w), int(reps))
        if ms < 0:
            raise RuntimeError(f"kfun3d_time_kernel failed: {last_error()}")
        return ms

    def matrix(self):
        """(ia, ja, blocks[nnz,4,4]) of the device matrix (Jacobian or factor)."""
        L = lib()
        nnz = L.kfun3d_matrix_read(self.g, None, None, None)
        ia = np.zeros(self.view.nnodes + 1, dtype=np.uint32)
        ja = np.zeros(nnz, dtype=np.uint32)
        blocks = np.zeros(nnz * 16)
        rc = L.kfun3d_matrix_read(self.g, ia.ctypes.data_as(C.POINTER(C.c_uint)),
                                  ja.ctypes.data_as(C.POINTER(C.c_uint)), _d(blocks))
        if rc < 0:
            raise RuntimeError(f"kfun3d_matrix_read failed: {last_error()}")
        return ia, ja, blocks.reshape(-1, 4, 4)

    def time_solve(self, reps=1, **params):
        """Mean device seconds per solve from the current state, and the last history."""
        p = default_params(**params)
        hist = (Step * 64)()
        ns = C.c_int(0)
        t = lib().kfun3d_time_solve(self.g, C.byref(p), int(reps), hist, 64, C.byref(ns))
        if t < 0:
            raise RuntimeError(f"kfun3d_time_solve failed: {last_error()}")
        steps = [dict(step=h.step, gmres_its=h.gmres_its, cfl=h.cfl, fnorm=h.fnorm, lift=h.lift,
                      drag=h.drag, momn=h.momn, seconds=h.seconds) for h in hist[:ns.value]]
        return t, steps

    def solve_flexible(self, net=None, **params):
        """FGMRES solve (ILU(0), or with `net` the learned preconditioner); updates q.
        Returns (history, stats)."""
        p = default_params(**params)
        hist = (Step * 64)()
        st = FlexStats()
        n = lib().kfun3d_solve_flexible(self.g, C.byref(p), net.h if net is not None else None, hist, 64,
                                        C.byref(st))
        if n < 0:
            raise RuntimeError(f"kfun3d_solve_flexible failed: {last_error()}")
        return _hist(hist, n), st.as_dict()

    def time_solve_flexible(self, net=None, reps=1, **params):
        """Mean device seconds per flexible solve from the current state (not updated)."""
        p = default_params(**params)
        hist = (Step * 64)()
        st = FlexStats()
        ns = C.c_int(0)
        t = lib().kfun3d_time_solve_flexible(self.g, C.byref(p), net.h if net is not None else None, int(reps),
                                             hist, 64, C.byref(ns), C.byref(st))
        if t < 0:
            raise RuntimeError(f"kfun3d_time_solve_flexible failed: {last_error()}")
        return t, _hist(hist, ns.value), st.as_dict()

    def time_learned_apply(self, net, reps=10):
        """Milliseconds of one application of the network on this mesh."""
        ms = lib().kfun3d_time_learned_apply(self.g, net.h, int(reps))
        if ms < 0:
            raise RuntimeError(f"kfun3d_time_learned_apply failed: {last_error()}")
        return ms

    def collect_pairs(self, stride=5, cap=64, **params):
        """Training pairs of the ILU(0)-FGMRES solve from the current state
        (q updated): (x0 BF16 [n, N, 8], target FP32 [n, N, 4], stats) on the GPU."""
        import torch
        N = self.view.nnodes
        x0 = torch.empty((cap, N, 8), dtype=torch.bfloat16, device="cuda")
        tgt = torch.empty((cap, N, 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        p = default_params(**params)
        st = FlexStats()
        n = lib().kfun3d_collect_pairs(self.g, C.byref(p), int(stride), x0.data_ptr(), tgt.data_ptr(), int(cap),
                                       C.byref(st))
        if n < 0:
            raise RuntimeError(f"kfun3d_collect_pairs failed: {last_error()}")
        if n < cap:
            x0, tgt = x0[:n].clone(), tgt[:n].clone()
        return x0, tgt, st.as_dict()

    def release_device(self):
        lib().kfun3d_device_release(self.g)


def _hist(hist, n):
    return [dict(step=h.step, gmres_its=h.gmres_its, cfl=h.cfl, fnorm=h.fnorm, lift=h.lift, drag=h.drag,
                 momn=h.momn, seconds=h.seconds) for h in hist[:n]]


def norm2(v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    return lib().Compute2ndNorm(v.size, _d(v))


def axpy(a, x, y):
    lib().ComputeAXPY(x.size, float(a), _d(x), _d(y))


def new_axpy(a, x, y):
    w = np.zeros_like(x)
    lib().ComputeNewAXPY(x.size, float(a), _d(x), _d(y), _d(w))
    return w


def normalize(x):
    return lib().Normalize(x.size, _d(x))
