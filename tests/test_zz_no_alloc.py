"""The allocation-free triangular solve, checked against the existing entry point.

kfun3d_sptrsv_device_noalloc exists for callers that cannot allocate device
memory: a framework that owns every device allocation (its own pooled
allocator, or all device memory sized at start-up) and forbids libraries from
calling cudaMalloc afterwards.  It takes the caller's device arrays and keeps
its only working memory (per-row completion flags) in a fixed file-scope
device array.  These tests run it twice in a row on the same factor, in both
precisions of the factor, and require the result to equal
ComputeSparseTriangularSolve's: exactly in exact mode, within the fast mode's
1e-9 solve tolerance in fast mode.  They also check its refusals (no factor,
misaligned pointers, the spatial ILU order, a precision changed after
factoring, more rows than the fixed array holds).  The file runs last (file
name) so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import MESH_A, seeded_state
import kfun3d_b200 as kf
from kfun3d_b200.geometry import GEOMETRY
from oracle import port

pytestmark = pytest.mark.gpu

KFUN3D_ERR_ARG = 4


def noalloc_fn():
    L = kf.lib()
    f = L.kfun3d_sptrsv_device_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(GEOMETRY), C.c_void_p, C.c_void_p]
    return f


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("mode,tol", [("exact", 0.0), ("fast", 1e-9)])
def test_noalloc_matches_existing_entry_point(box_mesh, mode, tol, precision):
    import torch
    kf.set_mode(mode)
    kf.set_precision(precision)
    kf.set_ilu_order(0)
    kf.set_aoa(3.06)
    try:
        for path in (MESH_A, box_mesh(12, seed=7)):
            m = kf.Mesh(path)
            v = m.view
            q = seeded_state(v.q.copy(), 5)
            cdt = port.timestep(m.g, v.nnodes, 40.0, q)
            m.fill(q, cdt)
            m.ilu()
            f = noalloc_fn()
            for call in range(2):
                b = np.random.default_rng(100 + call).standard_normal(v.dofs)
                x_ref = m.sptrsv(b)
                db = torch.from_numpy(b).to("cuda")
                dx = torch.full_like(db, float("nan"))
                rc = f(m.g, db.data_ptr(), dx.data_ptr())
                assert rc == 0, kf.last_error()
                x = dx.cpu().numpy()
                if tol == 0.0:
                    assert np.array_equal(x, x_ref), (path, call)
                else:
                    assert np.max(np.abs(x - x_ref)) <= tol * np.max(np.abs(x_ref)), (path, call)
            m.close()
    finally:
        kf.set_mode("exact")
        kf.set_precision(0)
        kf.set_aoa(3.0)


def test_noalloc_rejects_bad_arguments(box_mesh):
    import torch
    kf.set_mode("exact")
    kf.set_precision(0)
    kf.set_abort_on_error(False)
    try:
        m = kf.Mesh(MESH_A)
        f = noalloc_fn()
        # no factor on the device yet
        assert f(m.g, 0, 0) == KFUN3D_ERR_ARG
        assert "ComputeNumericalILU" in kf.last_error()
        m.fill()
        m.ilu()
        db = torch.zeros(m.view.dofs + 2, dtype=torch.float64, device="cuda")
        # misaligned device pointer
        assert f(m.g, db.data_ptr() + 8, db.data_ptr()) == KFUN3D_ERR_ARG
        # factor computed in FP64, FP32 now set
        kf.set_precision(1)
        assert f(m.g, db.data_ptr(), db.data_ptr() + 8 * 4 * 2) == KFUN3D_ERR_ARG
        assert "precision" in kf.last_error()
        kf.set_precision(0)
        m.close()
        # the spatial ILU(0) order is refused
        m = kf.Mesh(box_mesh(10, seed=2))
        kf.set_ilu_order(1)
        m.fill()
        m.ilu()
        dx = torch.zeros(m.view.dofs, dtype=torch.float64, device="cuda")
        assert f(m.g, db.data_ptr(), dx.data_ptr()) == KFUN3D_ERR_ARG
        assert "spatial" in kf.last_error()
        kf.set_ilu_order(0)
        m.close()
        # more rows than the fixed flag array holds (129^3 = 2,146,689 > 2,097,152),
        # refused from the host pattern alone
        m = kf.Mesh(box_mesh(129, seed=1))
        assert f(m.g, db.data_ptr(), dx.data_ptr()) == KFUN3D_ERR_ARG
        assert "2,097,152" in kf.last_error()
        m.close()
        kf.clear_status()
    finally:
        kf.set_ilu_order(0)
        kf.set_precision(0)
        kf.set_abort_on_error(True)
