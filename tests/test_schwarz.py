"""Additive Schwarz without overlap on one device (kfun3d_set_schwarz).

* the subdomains are the recursive coordinate bisection restated below
  (host only, no GPU);
* with the blocks that couple two subdomains removed, the device's ILU(0)
  factor and triangular solves equal the oracle's (matrix/ilu.cpp:49-136,
  matrix/sptrsv.cpp:34-73) run on the same matrix with the same blocks set
  to zero: bit for bit in FP64, within 1e-5 in FP32, in the mesh's
  numbering and in the spatial order;
* the factor is block-Jacobi: every removed block stays exactly zero and a
  triangular solve of a right-hand side that lives in one subdomain stays
  in it;
* a solve with subdomains converges to the state without them (the
  Jacobian-vector products do not change, only the preconditioner).
"""
import numpy as np
import pytest

import kfun3d_b200 as kf
from oracle import port
from conftest import seeded_state
from test_ilu_order import Renumbered, _from_spatial, _to_spatial


@pytest.fixture(autouse=True)
def _settings():
    aoa, mode = kf.get_aoa(), kf.get_mode()
    kf.set_aoa(3.06)
    kf.set_precision(0)
    kf.set_ilu_order(0)
    kf.set_schwarz(0)
    yield
    kf.set_schwarz(0)
    kf.set_ilu_order(0)
    kf.set_precision(0)
    kf.set_mode(mode)
    kf.set_aoa(aoa)


def rcb(xyz, parts):
    """Recursive coordinate bisection: a set of n nodes going to p parts is cut
    across the longest side of its bounding box, the floor(n * floor(p/2) / p)
    nodes lowest in that coordinate (ties by node index) going to the first
    floor(p/2) parts."""
    part = np.zeros(xyz[0].size, dtype=np.int64)

    def split(idx, p0, np_):
        if np_ <= 1 or idx.size <= 1:
            part[idx] = p0
            return
        ext = [c[idx].max() - c[idx].min() for c in xyz]
        ax = 0
        for d in (1, 2):
            if ext[d] > ext[ax]:
                ax = d
        nl = np_ // 2
        cut = idx.size * nl // np_
        o = idx[np.lexsort((idx, xyz[ax][idx]))]
        split(o[:cut], p0, nl)
        split(o[cut:], p0 + nl, np_ - nl)

    split(np.arange(xyz[0].size), 0, parts)
    return part


def cross_blocks(ia, ja, part_row):
    rows = np.repeat(np.arange(ia.size - 1), np.diff(ia.astype(np.int64)))
    return part_row[rows] != part_row[ja.astype(np.int64)]


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_partition_is_rcb(box_mesh, parts):
    m = kf.Mesh(box_mesh(11, seed=41))
    part = m.schwarz_partition(parts)
    assert np.array_equal(part, rcb([c.copy() for c in m.view.xyz], parts))
    sizes = np.bincount(part, minlength=parts)
    assert sizes.size == parts and sizes.min() > 0
    assert sizes.max() - sizes.min() <= 2


def test_setting_round_trip():
    kf.set_schwarz(4)
    assert kf.get_schwarz() == 4
    kf.set_schwarz(1)
    assert kf.get_schwarz() == 0


def _filled(path, seed):
    m = kf.Mesh(path)
    v = m.view
    q = seeded_state(v.q.copy(), seed)
    cdt = port.timestep(m.g, v.nnodes, 40.0, q)
    return m, q, cdt


@pytest.mark.gpu
@pytest.mark.parametrize("parts", [2, 5])
def test_exact_block_jacobi_mesh_order(box_mesh, parts):
    kf.set_mode("exact")
    m, q, cdt = _filled(box_mesh(12, seed=42), 42)
    v = m.view
    part = m.schwarz_partition(parts)
    kf.set_schwarz(parts)
    M = port.Matrix(m.g)
    ia, ja, _ = M.pattern()
    cross = cross_blocks(ia, ja, part)
    assert cross.any()
    b = np.random.default_rng(42).standard_normal(v.dofs)
    for prec in (0, 1):
        kf.set_precision(prec)
        m.fill(q, cdt)
        M.fill(3.06, q, cdt)
        M.drop_coupling(cross)
        m.ilu()
        if prec == 0:
            M.ilu()
            _, _, f = m.matrix()
            assert np.array_equal(f, M.blocks())
            assert not f[cross].any()
            assert np.array_equal(m.sptrsv(b), M.sptrsv(b))
        else:
            M.ilu_f32()
            x = M.sptrsv_f32(b)
            assert np.max(np.abs(m.sptrsv(b) - x)) / np.max(np.abs(x)) < 1e-5
    assert kf.last_status() == 0
    # a right-hand side inside subdomain 0 gives a solution inside it
    kf.set_precision(0)
    m.fill(q, cdt)
    m.ilu()
    b0 = b.reshape(-1, 4).copy()
    b0[part != 0] = 0.0
    x0 = m.sptrsv(b0.reshape(-1)).reshape(-1, 4)
    assert not x0[part != 0].any()
    assert x0[part == 0].any()


@pytest.mark.gpu
def test_exact_block_jacobi_spatial_order(box_mesh):
    kf.set_mode("exact")
    m, q, cdt = _filled(box_mesh(13, seed=43), 43)
    v = m.view
    parts = 4
    part = m.schwarz_partition(parts)
    kf.set_ilu_order(1)
    kf.set_schwarz(parts)
    m.fill(q, cdt)
    m.ilu()
    rank = m.ilu_rank()
    M = port.Matrix(m.g)
    M.fill(3.06, q, cdt)
    R = Renumbered(M, rank, v.n0, v.n1)
    part_row = np.empty_like(part)
    part_row[rank] = part
    cross = cross_blocks(R.ia, R.ja, part_row)
    assert cross.any()
    R.a.reshape(-1, 16)[cross] = 0.0
    R.ilu()
    b = np.random.default_rng(43).standard_normal(v.dofs)
    x = _from_spatial(R.sptrsv(_to_spatial(b, rank)), rank)
    assert np.array_equal(m.sptrsv(b), x)
    assert kf.last_status() == 0


@pytest.mark.gpu
def test_solve_with_subdomains_converges_to_the_same_state(box_mesh):
    kf.set_mode("fast")
    kf.set_precision(1)
    kf.set_ilu_order(1)
    m = kf.Mesh(box_mesh(22, seed=33))
    q0 = m.view.q.copy()
    out = {}
    for parts in (0, 8):
        kf.set_schwarz(parts)
        m.view.q[:] = q0
        h = m.solve(ts_max=20, stop_ratio=1e8)
        assert kf.last_status() == 0
        assert h[0]["fnorm"] / h[-1]["fnorm"] >= 1e8, parts
        out[parts] = (sum(s["gmres_its"] for s in h), np.array([h[-1][k] for k in ("lift", "drag", "momn")]),
                      m.view.q.copy())
    (its0, f0, qa), (its8, f8, qb) = out[0], out[8]
    # the subdomains only weaken the preconditioner; the state is the same
    assert its8 > its0, (its0, its8)
    assert np.allclose(f0, f8, rtol=1e-6, atol=0)
    assert float(np.max(np.abs(qa - qb)) / np.max(np.abs(qa))) < 1e-6
