"""Test infrastructure only: ctypes access to the C oracle (kfun3d_oracle.c).

The oracle restates the reference's kernels in plain C (built by
``make -C oracle port`` into ``oracle/_build/liboracle.so``).  It is the
checker for the CUDA path; the product never loads it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from kfun3d_b200.geometry import GEOMETRY

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")


class Phys(C.Structure):
    _fields_ = [("u", C.c_double), ("v", C.c_double)]


class Params(C.Structure):
    _fields_ = [("ts_max", C.c_int), ("stop_ratio", C.c_double),
                ("gmres_rtol", C.c_double), ("gmres_restart", C.c_int),
                ("gmres_max_it", C.c_int), ("cfl_init", C.c_double),
                ("cfl_max", C.c_double), ("first_order", C.c_int),
                ("precision", C.c_int)]


class Step(C.Structure):
    _fields_ = [("step", C.c_int), ("gmres_its", C.c_int), ("cfl", C.c_double),
                ("fnorm", C.c_double), ("lift", C.c_double), ("drag", C.c_double),
                ("momn", C.c_double)]


class BSR(C.Structure):
    _fields_ = [("n", C.c_size_t), ("nnz", C.c_size_t),
                ("ia", C.POINTER(C.c_uint32)), ("ja", C.POINTER(C.c_uint32)),
                ("diag", C.POINTER(C.c_uint32)), ("a", C.POINTER(C.c_double)),
                ("af", C.POINTER(C.c_float)), ("lslot", C.POINTER(C.c_double)),
                ("lpos", C.POINTER(C.c_uint32)), ("last_lower", C.POINTER(C.c_uint32))]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, G, D = C.POINTER, C.POINTER(GEOMETRY), C.POINTER(C.c_double)
        L.orc_phys_from_aoa.restype = Phys
        L.orc_phys_from_aoa.argtypes = [C.c_double]
        L.orc_flux.argtypes = [G, Phys, D, D, D, D, D, C.c_int]
        L.orc_timestep.argtypes = [G, C.c_double, D, D]
        L.orc_forces.argtypes = [G, Phys, D, D]
        L.orc_bsr_create.restype = P(BSR)
        L.orc_bsr_create.argtypes = [G]
        L.orc_bsr_free.argtypes = [P(BSR)]
        L.orc_fill.argtypes = [P(BSR), G, Phys, D, D]
        L.orc_ilu.argtypes = [P(BSR)]
        L.orc_sptrsv.argtypes = [P(BSR), D, D]
        L.orc_round_f32.argtypes = [P(BSR)]
        L.orc_ilu_f32.argtypes = [P(BSR)]
        L.orc_sptrsv_f32.argtypes = [P(BSR), D, D]
        L.orc_inv4.argtypes = [D, D]
        L.orc_norm2.restype = C.c_double
        L.orc_norm2.argtypes = [C.c_size_t, D]
        L.orc_solve.restype = C.c_int
        L.orc_solve.argtypes = [G, Phys, D, P(Params), P(Step), C.c_int]
        _lib = L
    return _lib


def dptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def phys(aoa_deg):
    return lib().orc_phys_from_aoa(aoa_deg)


def flux(gptr, aoa, q, first_order=False):
    dofs = q.size
    q = np.ascontiguousarray(q, dtype=np.float64)
    gx, gy, gz, r = (np.zeros(dofs) for _ in range(4))
    lib().orc_flux(gptr, phys(aoa), dptr(q), dptr(gx), dptr(gy), dptr(gz), dptr(r),
                   int(first_order))
    return (gx, gy, gz), r


def timestep(gptr, nnodes, cfl, q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    cdt = np.zeros(nnodes)
    lib().orc_timestep(gptr, cfl, dptr(q), dptr(cdt))
    return cdt


def forces(gptr, aoa, q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros(3)
    lib().orc_forces(gptr, phys(aoa), dptr(q), dptr(out))
    return out


class Matrix:
    """The oracle's BSR with the reference's ILU slot state."""

    def __init__(self, gptr):
        self.gptr = gptr
        self.m = lib().orc_bsr_create(gptr)
        c = self.m.contents
        self.n, self.nnz = int(c.n), int(c.nnz)

    def __del__(self):
        try:
            lib().orc_bsr_free(self.m)
        except Exception:
            pass

    def pattern(self):
        c = self.m.contents
        ia = np.ctypeslib.as_array(c.ia, shape=(self.n + 1,)).copy()
        ja = np.ctypeslib.as_array(c.ja, shape=(self.nnz,)).copy()
        d = np.ctypeslib.as_array(c.diag, shape=(self.n,)).copy()
        return ia, ja, d

    def blocks(self):
        return np.ctypeslib.as_array(self.m.contents.a, shape=(self.nnz * 16,)).copy().reshape(-1, 4, 4)

    def blocks_f32(self):
        return np.ctypeslib.as_array(self.m.contents.af, shape=(self.nnz * 16,)).copy().reshape(-1, 4, 4)

    def drop_coupling(self, cross):
        """Set to zero the blocks flagged in `cross` (one flag per block of the
        pattern), in place: the matrix an additive Schwarz preconditioner
        without overlap factors."""
        a = np.ctypeslib.as_array(self.m.contents.a, shape=(self.nnz * 16,)).reshape(-1, 16)
        a[np.asarray(cross, dtype=bool)] = 0.0

    def fill(self, aoa, q, cdt):
        q = np.ascontiguousarray(q, dtype=np.float64)
        cdt = np.ascontiguousarray(cdt, dtype=np.float64)
        lib().orc_fill(self.m, self.gptr, phys(aoa), dptr(q), dptr(cdt))

    def ilu(self):
        lib().orc_ilu(self.m)

    def ilu_f32(self):
        lib().orc_round_f32(self.m)
        lib().orc_ilu_f32(self.m)

    def sptrsv(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        lib().orc_sptrsv(self.m, dptr(b), dptr(x))
        return x

    def sptrsv_f32(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        lib().orc_sptrsv_f32(self.m, dptr(b), dptr(x))
        return x


def default_params(**kw):
    p = dict(ts_max=15, stop_ratio=1e7, gmres_rtol=0.01, gmres_restart=30,
             gmres_max_it=10000, cfl_init=50.0, cfl_max=100000.0, first_order=0,
             precision=0)
    p.update(kw)
    return Params(**p)


def solve(gptr, aoa, q, **params):
    """Newton/GMRES solve from state q (updated in place); list of step dicts."""
    assert q.dtype == np.float64 and q.flags.c_contiguous
    p = default_params(**params)
    hist = (Step * 64)()
    n = lib().orc_solve(gptr, phys(aoa), dptr(q), C.byref(p), hist, 64)
    return [dict(step=h.step, gmres_its=h.gmres_its, cfl=h.cfl, fnorm=h.fnorm,
                 lift=h.lift, drag=h.drag, momn=h.momn) for h in hist[:n]]
