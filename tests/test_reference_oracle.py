"""The C oracle against the reference itself (oracle/_ref), kernel by kernel.

Skipped where the reference build is absent.  On seeded meshes and states the
oracle's residual, gradients, time step, Jacobian, ILU(0) factor (two
consecutive Newton steps, so the persistent-slot behaviour is exercised),
triangular solves and forces are bit-identical to the reference's.
"""
import numpy as np
import pytest

from conftest import seeded_state
from oracle import port, ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("n,seed,aoa", [(6, 1, 3.06), (12, 5, 4.5), (9, 2, 0.0)])
def test_kernels_bit_identical(box_mesh, n, seed, aoa):
    m = ref.RefMesh(box_mesh(n, seed=seed), aoa, 1)
    v = m.view
    q = seeded_state(v.q.copy(), seed)
    (g1, r1) = m.flux(q)
    (g2, r2) = port.flux(m.g, aoa, q)
    assert np.array_equal(r1, r2)
    assert all(np.array_equal(a, b) for a, b in zip(g1, g2))
    c1 = m.timestep(123.0, q)
    c2 = port.timestep(m.g, v.nnodes, 123.0, q)
    assert np.array_equal(c1, c2)
    M = port.Matrix(m.g)
    for step in range(2):
        qs = q + step * 0.01
        _, _, _, A1 = m.fill(qs, c1)
        M.fill(aoa, qs, c1)
        assert np.array_equal(A1, M.blocks())
        _, _, _, F1 = m.ilu()
        M.ilu()
        assert np.array_equal(F1, M.blocks())
        b = np.random.default_rng(seed + step).standard_normal(v.dofs)
        assert np.array_equal(m.sptrsv(b), M.sptrsv(b))
    assert np.array_equal(m.forces(q), port.forces(m.g, aoa, q))


def test_first_order_mode_is_zero_gradient_flux(box_mesh):
    m = ref.RefMesh(box_mesh(6, seed=1), 3.0, 1)
    q = seeded_state(m.view.q.copy(), 4)
    (g, r) = port.flux(m.g, 3.0, q, first_order=True)
    assert all(np.all(x == 0) for x in g)
    (g2, r2) = port.flux(m.g, 3.0, q)
    assert not np.array_equal(r, r2)


def test_fp32_preconditioner_close_to_fp64(box_mesh):
    m = ref.RefMesh(box_mesh(8, seed=2), 3.0, 1)
    v = m.view
    q = seeded_state(v.q.copy(), 3)
    cdt = port.timestep(m.g, v.nnodes, 50.0, q)
    M = port.Matrix(m.g)
    M.fill(3.0, q, cdt)
    M.ilu_f32()
    M2 = port.Matrix(m.g)
    M2.fill(3.0, q, cdt)
    M2.ilu()
    b = np.random.default_rng(0).standard_normal(v.dofs)
    x32, x64 = M.sptrsv_f32(b), M2.sptrsv(b)
    assert np.max(np.abs(x32 - x64)) / np.max(np.abs(x64)) < 1e-4
