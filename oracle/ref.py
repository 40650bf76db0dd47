"""Test infrastructure only: ctypes access to the reference itself.

``oracle/_ref/libkfun3d_ref.so`` is the reference compiled from its own
sources by ``oracle/Makefile`` (target ``ref``).  This module calls its C entry
points (inc/core_kernel.h:6-22, inc/utils.h:15-28, src/mesh.c:22 Setup) and the
harness in ``oracle/ref_harness.c``.  Only tests, ``smoke()`` and the CPU
baseline of ``bench.py`` use it, and only as the checker.
"""
import ctypes as C
import os

import numpy as np

from kfun3d_b200.geometry import GEOMETRY, GRADIENT, GeometryView

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libkfun3d_ref.so")


class RefParams(C.Structure):
    _fields_ = [("ts_max", C.c_int), ("stop_ratio", C.c_double),
                ("gmres_rtol", C.c_double), ("gmres_restart", C.c_int),
                ("gmres_max_it", C.c_int), ("cfl_init", C.c_double),
                ("cfl_max", C.c_double)]


class RefStep(C.Structure):
    _fields_ = [("step", C.c_int), ("gmres_its", C.c_int), ("cfl", C.c_double),
                ("fnorm", C.c_double), ("lift", C.c_double), ("drag", C.c_double),
                ("momn", C.c_double)]


def default_params(**kw):
    """src/kernel.c:12-22 defaults."""
    p = dict(ts_max=15, stop_ratio=1e7, gmres_rtol=0.01, gmres_restart=30,
             gmres_max_it=10000, cfl_init=50.0, cfl_max=100000.0)
    p.update(kw)
    return RefParams(**p)


def available():
    return os.path.exists(LIB_PATH)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle ref`")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.ref_setup.restype = P(GEOMETRY)
        L.ref_setup.argtypes = [C.c_char_p, C.c_int]
        L.ref_free.argtypes = [P(GEOMETRY)]
        L.ref_set_aoa.argtypes = [C.c_double]
        L.ref_get_uv.argtypes = [P(C.c_double), P(C.c_double)]
        L.ref_solve.restype = C.c_int
        L.ref_solve.argtypes = [P(GEOMETRY), P(RefParams), P(RefStep), C.c_int]
        L.ComputeFlux.argtypes = [P(GEOMETRY), P(C.c_double), P(GRADIENT), P(C.c_double)]
        L.ComputeTimeStep.argtypes = [C.c_double, P(GEOMETRY)]
        L.ComputeA.argtypes = [P(GEOMETRY)]
        L.ComputeNumericalILU.argtypes = [P(GEOMETRY)]
        L.ComputeSparseTriangularSolve.argtypes = [P(GEOMETRY), P(C.c_double), P(C.c_double)]
        L.ComputeForces.argtypes = [P(GEOMETRY), P(C.c_double)]
        L.Compute2ndNorm.restype = C.c_double
        L.Compute2ndNorm.argtypes = [C.c_size_t, P(C.c_double)]
        L.ref_matrix_rows.restype = C.c_size_t
        L.ref_matrix_rows.argtypes = [C.c_void_p]
        L.ref_matrix_bsr.argtypes = [C.c_void_p] + [P(P(C.c_uint32))] * 3 + [P(P(C.c_double))]
        L.ref_matrix_levels.argtypes = [C.c_void_p, P(C.c_uint32), P(C.c_uint32)]
        _lib = L
    return _lib


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class RefMesh:
    """A GEOMETRY built by the reference's own Setup (src/mesh.c:22-154)."""

    def __init__(self, path, aoa_deg=3.0, threads=1):
        L = lib()
        L.ref_set_aoa(aoa_deg)
        self.aoa = aoa_deg
        self.g = L.ref_setup(os.fsencode(path), threads)
        self.view = GeometryView(self.g)
        self.view.owner = self

    def close(self):
        if self.g:
            lib().ref_free(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _aoa(self):
        lib().ref_set_aoa(self.aoa)

    def flux(self, q):
        self._aoa()
        v = self.view
        q = np.ascontiguousarray(q, dtype=np.float64)
        gx, gy, gz, r = (np.zeros(v.dofs) for _ in range(4))
        grad = GRADIENT(dptr(gx), dptr(gy), dptr(gz))
        lib().ComputeFlux(self.g, dptr(q), C.byref(grad), dptr(r))
        return (gx, gy, gz), r

    def timestep(self, cfl, q):
        self._aoa()
        self.view.q[:] = q
        lib().ComputeTimeStep(cfl, self.g)
        return self.view.cdt.copy()

    def fill(self, q, cdt):
        """ComputeA at state q with diagonal cdt; returns (ia, ja, diag, blocks)."""
        self._aoa()
        self.view.q[:] = q
        self.view.cdt[:] = cdt
        lib().ComputeA(self.g)
        return self.bsr()

    def ilu(self):
        lib().ComputeNumericalILU(self.g)
        return self.bsr()

    def bsr(self):
        L = lib()
        n = L.ref_matrix_rows(self.view.matrix)
        ia, ja, d = (C.POINTER(C.c_uint32)() for _ in range(3))
        a = C.POINTER(C.c_double)()
        L.ref_matrix_bsr(self.view.matrix, C.byref(ia), C.byref(ja), C.byref(d), C.byref(a))
        ia_np = np.ctypeslib.as_array(ia, shape=(n + 1,)).copy()
        nnz = int(ia_np[-1])
        ja_np = np.ctypeslib.as_array(ja, shape=(nnz,)).copy()
        d_np = np.ctypeslib.as_array(d, shape=(n,)).copy()
        a_np = np.ctypeslib.as_array(a, shape=(nnz * 16,)).copy().reshape(nnz, 4, 4)
        return ia_np, ja_np, d_np, a_np

    def levels(self):
        nl, nu = C.c_uint32(), C.c_uint32()
        lib().ref_matrix_levels(self.view.matrix, C.byref(nl), C.byref(nu))
        return nl.value, nu.value

    def sptrsv(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        lib().ComputeSparseTriangularSolve(self.g, dptr(b), dptr(x))
        return x

    def forces(self, q):
        self._aoa()
        self.view.q[:] = q
        out = np.zeros(3)
        lib().ComputeForces(self.g, dptr(out))
        return out

    def solve(self, **params):
        """Newton/GMRES driver of src/kernel.c:47-232 (harness, parameterised).

        Starts from the state currently in ``view.q``; returns a list of dicts.
        """
        self._aoa()
        p = default_params(**params)
        hist = (RefStep * 64)()
        n = lib().ref_solve(self.g, C.byref(p), hist, 64)
        return [dict(step=h.step, gmres_its=h.gmres_its, cfl=h.cfl, fnorm=h.fnorm,
                     lift=h.lift, drag=h.drag, momn=h.momn) for h in hist[:n]]
