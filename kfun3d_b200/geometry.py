"""ctypes mirror of the reference's GEOMETRY struct (inc/geometry.h:1-107).

The drop-in C-ABI takes ``GEOMETRY *`` exactly as the reference's kernels do
(inc/core_kernel.h:6-22), so the layout here must match the C header field for
field: ``unsigned long int`` is 64-bit, pointers are host pointers.  Helpers
return zero-copy numpy views of the arrays a GEOMETRY points to.
"""
import ctypes as C

import numpy as np

c_u32p = C.POINTER(C.c_uint32)
c_f64p = C.POINTER(C.c_double)


class XYZN(C.Structure):  # struct xyzn: unit normal + area per edge
    _fields_ = [("x0", c_f64p), ("x1", c_f64p), ("x2", c_f64p), ("x3", c_f64p)]


class XYZ(C.Structure):  # struct xyz (also GRADIENT)
    _fields_ = [("x0", c_f64p), ("x1", c_f64p), ("x2", c_f64p)]


GRADIENT = XYZ


class Edge(C.Structure):
    _fields_ = [("n0", c_u32p), ("n1", c_u32p)]


class Face(C.Structure):
    _fields_ = [("n0", c_u32p), ("n1", c_u32p), ("n2", c_u32p)]


class Weights(C.Structure):
    _fields_ = [("w0", C.POINTER(XYZ)), ("w1", C.POINTER(XYZ))]


class ETbl(C.Structure):
    _fields_ = [("sz", C.c_ulong), ("eptr", C.POINTER(Edge)),
                ("xyzn", C.POINTER(XYZN)), ("w", C.POINTER(Weights))]


class NTbl(C.Structure):
    _fields_ = [("sz", C.c_ulong), ("xyz", C.POINTER(XYZ)),
                ("part", c_u32p), ("cdt", c_f64p)]


class STbl(C.Structure):
    _fields_ = [("sz", C.c_ulong), ("i", c_u32p)]


class BNTbl(C.Structure):
    _fields_ = [("sz", C.c_ulong), ("nptr", c_u32p), ("xyz", C.POINTER(XYZ))]


class BFTbl(C.Structure):
    _fields_ = [("sz", C.c_ulong), ("fptr", C.POINTER(Face))]


class BTbl(C.Structure):
    _fields_ = [("s", C.POINTER(BNTbl)), ("f", C.POINTER(BNTbl)),
                ("fc", C.POINTER(BFTbl))]


class CTbl(C.Structure):
    _fields_ = [("b", C.c_uint), ("b2", C.c_uint), ("sz", C.c_ulong)]


class QTbl(C.Structure):
    _fields_ = [("q", c_f64p)]


class GEOMETRY(C.Structure):
    _fields_ = [("e", C.POINTER(ETbl)), ("n", C.POINTER(NTbl)),
                ("b", C.POINTER(BTbl)), ("c", C.POINTER(CTbl)),
                ("s", C.POINTER(STbl)), ("t", C.POINTER(STbl)),
                ("q", C.POINTER(QTbl)), ("matrix", C.c_void_p)]


def _view(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    ctype = C.c_double if dtype == np.float64 else C.c_uint32
    arr = C.cast(ptr, C.POINTER(ctype * n)).contents
    return np.frombuffer(arr, dtype=dtype)


class GeometryView:
    """Zero-copy numpy views of the arrays behind a ``GEOMETRY *``.

    ``gptr`` is a ``POINTER(GEOMETRY)``; the views stay valid as long as the
    GEOMETRY they were taken from is alive.
    """

    def __init__(self, gptr):
        self.ptr = gptr
        g = gptr.contents
        e, n, b, c = g.e.contents, g.n.contents, g.b.contents, g.c.contents
        self.nnodes = int(n.sz)
        self.nedges = int(e.sz)
        self.bsz = int(c.b)
        self.dofs = int(c.sz)
        E, N = self.nedges, self.nnodes
        self.n0 = _view(e.eptr.contents.n0, E, np.uint32)
        self.n1 = _view(e.eptr.contents.n1, E, np.uint32)
        xn = e.xyzn.contents
        self.xn = _view(xn.x0, E, np.float64)
        self.yn = _view(xn.x1, E, np.float64)
        self.zn = _view(xn.x2, E, np.float64)
        self.area = _view(xn.x3, E, np.float64)
        w = e.w.contents
        self.w0 = [_view(getattr(w.w0.contents, k), E, np.float64) for k in ("x0", "x1", "x2")]
        self.w1 = [_view(getattr(w.w1.contents, k), E, np.float64) for k in ("x0", "x1", "x2")]
        self.xyz = [_view(getattr(n.xyz.contents, k), N, np.float64) for k in ("x0", "x1", "x2")]
        self.part = _view(n.part, N, np.uint32)
        self.cdt = _view(n.cdt, N, np.float64)
        s, f, fc = b.s.contents, b.f.contents, b.fc.contents
        self.ns = int(s.sz)
        self.nf = int(f.sz)
        self.nfaces = int(fc.sz)
        self.s_nodes = _view(s.nptr, self.ns, np.uint32)
        self.s_xyz = [_view(getattr(s.xyz.contents, k), self.ns, np.float64) for k in ("x0", "x1", "x2")]
        self.f_nodes = _view(f.nptr, self.nf, np.uint32)
        self.f_xyz = [_view(getattr(f.xyz.contents, k), self.nf, np.float64) for k in ("x0", "x1", "x2")]
        fp = fc.fptr.contents
        self.faces = [_view(getattr(fp, k), self.nfaces, np.uint32) for k in ("n0", "n1", "n2")]
        st = g.s.contents
        self.nthreads = int(st.sz)
        self.ie = _view(st.i, self.nthreads + 1, np.uint32)
        tt = g.t.contents
        self.ncolors = int(tt.sz)
        self.colors = _view(tt.i, self.ncolors + 1, np.uint32)
        self.q = _view(g.q.contents.q, self.dofs, np.float64)
        self.matrix = g.matrix
