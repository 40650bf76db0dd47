"""CUDA path against the oracle (and the reference's golden history), on the GPU.

Exact mode must be bit-identical to the oracle, which is bit-identical to the
reference at one OpenMP thread.  Fast mode (FMA, tree reductions) is held to
1e-12 relative (max-norm) for the residual, gradients, time step and Jacobian,
1e-9 for the ILU factor and triangular solves, and to the converged-force
tolerance of 1e-10 for whole solves.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, MESH_A, seeded_state
import kfun3d_b200 as kf
from oracle import port

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def defaults():
    kf.set_abort_on_error(True)
    kf.set_mode("exact")
    kf.set_precision(0)
    kf.set_first_order(False)
    kf.set_aoa(3.0)
    kf.set_verbose(False)
    yield
    kf.set_mode("exact")
    kf.set_precision(0)
    kf.set_first_order(False)
    kf.set_aoa(3.0)


def meshes(box_mesh):
    return [(MESH_A, 3.0, 7), (box_mesh(10, seed=3), 3.06, 11), (box_mesh(17, seed=5), 4.5, 2)]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_exact_kernels_bit_identical(box_mesh):
    for path, aoa, seed in meshes(box_mesh):
        kf.set_aoa(aoa)
        m = kf.Mesh(path)
        # the least-squares terms recomputed on the device from per-node
        # coefficients made there equal the stored (reference) ones bit for bit
        assert m.query("lsq_terms_match") == 1, path
        assert m.query("sptrsv_schedule") == 8, path
        v = m.view
        q = seeded_state(v.q.copy(), seed)
        (g1, r1) = m.flux(q)
        (g2, r2) = port.flux(m.g, aoa, q)
        assert np.array_equal(r1, r2), path
        assert all(np.array_equal(a, b) for a, b in zip(g1, g2))
        c1 = m.timestep(37.5, q)
        c2 = port.timestep(m.g, v.nnodes, 37.5, q)
        assert np.array_equal(c1, c2)
        M = port.Matrix(m.g)
        for step in range(2):   # two Newton steps: persistent L slots carried over
            qs = q + 0.01 * step
            m.fill(qs, c1)
            M.fill(aoa, qs, c1)
            ia, ja, A = m.matrix()
            assert np.array_equal(A, M.blocks()), (path, step)
            m.ilu()
            M.ilu()
            _, _, F = m.matrix()
            assert np.array_equal(F, M.blocks()), (path, step)
            b = np.random.default_rng(seed + step).standard_normal(v.dofs)
            assert np.array_equal(m.sptrsv(b), M.sptrsv(b))
        assert np.array_equal(m.forces(q), port.forces(m.g, aoa, q))
        assert kf.last_status() == 0


def test_exact_first_order_flux(box_mesh):
    kf.set_first_order(True)
    m = kf.Mesh(box_mesh(10, seed=3))
    q = seeded_state(m.view.q.copy(), 5)
    (g1, r1) = m.flux(q)
    (_, r2) = port.flux(m.g, 3.0, q, first_order=True)
    assert np.array_equal(r1, r2)
    assert all(np.all(x == 0) for x in g1)


def test_exact_solve_meshA_matches_reference_history():
    """The whole-solve history check: every step's residual norm, CFL, GMRES
    count and forces equal the reference's (tolerance 1e-10 relative; exact mode
    achieves equality)."""
    gold = json.load(open(os.path.join(GOLDEN, "meshA_history.json")))["steps"]
    m = kf.Mesh(MESH_A)
    hist = m.solve()
    assert len(hist) == len(gold)
    for h, w in zip(hist, gold):
        assert h["gmres_its"] == w["gmres_its"]
        for k in ("cfl", "fnorm", "lift", "drag", "momn"):
            assert abs(h[k] - float(w[k])) <= 1e-10 * abs(float(w[k])), (h["step"], k)
            assert repr(h[k]) == w[k], (h["step"], k, h[k], w[k])
    # final state equals the oracle's
    m2 = kf.Mesh(MESH_A)
    q = m2.view.q.copy()
    port.solve(m2.g, 3.0, q)
    assert np.array_equal(m.view.q, q)


@pytest.mark.parametrize("path", ["meshA", "box12"])
def test_exact_solve_with_visit_order_copies(box_mesh, path, monkeypatch):
    """With the node data in a Morton visit order (the residual's visit-order
    copies, and the matrix-free product forming the shifted state and its
    visit-order copy in one pass) the exact-mode solve is the mesh order's,
    step for step and bit for bit."""
    mesh = MESH_A if path == "meshA" else box_mesh(12, seed=41)
    kf.set_aoa(3.0 if path == "meshA" else 3.06)
    out = {}
    for order in ("natural", "morton"):
        monkeypatch.setenv("KFUN3D_NODE_ORDER", order)
        m = kf.Mesh(mesh)
        assert m.query("visit_order_copies") == (1 if order == "morton" else 0)
        out[order] = (m.solve(ts_max=4), m.view.q.copy())
        m.close()
    (h0, q0), (h1, q1) = out["natural"], out["morton"]
    assert len(h0) == len(h1)
    for a, b in zip(h0, h1):
        for k in ("gmres_its", "cfl", "fnorm", "lift", "drag", "momn"):
            assert a[k] == b[k], (path, a["step"], k)
    assert np.array_equal(q0, q1)
    assert kf.last_status() == 0


def test_exact_kernel_entry_point_box(box_mesh):
    """Kernel() (the reference's constants) equals the oracle's solve."""
    kf.set_aoa(3.06)
    p = box_mesh(10, seed=3)
    m = kf.Mesh(p)
    m.kernel()
    m2 = kf.Mesh(p)
    q = m2.view.q.copy()
    port.solve(m2.g, 3.06, q)
    assert np.array_equal(m.view.q, q)


def test_fast_kernels_close(box_mesh):
    kf.set_mode("fast")
    for path, aoa, seed in meshes(box_mesh):
        kf.set_aoa(aoa)
        m = kf.Mesh(path)
        v = m.view
        q = seeded_state(v.q.copy(), seed)
        (g1, r1) = m.flux(q)
        (g2, r2) = port.flux(m.g, aoa, q)
        assert rel(r1, r2) < 1e-12
        assert max(rel(a, b) for a, b in zip(g1, g2)) < 1e-12
        c1 = m.timestep(37.5, q)
        c2 = port.timestep(m.g, v.nnodes, 37.5, q)
        assert rel(c1, c2) < 1e-12
        M = port.Matrix(m.g)
        m.fill(q, c2)
        M.fill(aoa, q, c2)
        _, _, A = m.matrix()
        assert rel(A, M.blocks()) < 1e-12
        m.ilu()
        M.ilu()
        _, _, F = m.matrix()
        assert rel(F, M.blocks()) < 1e-9
        b = np.random.default_rng(seed).standard_normal(v.dofs)
        assert rel(m.sptrsv(b), M.sptrsv(b)) < 1e-9


def test_fast_solve_meshA_forces():
    gold = json.load(open(os.path.join(GOLDEN, "meshA_history.json")))["steps"]
    kf.set_mode("fast")
    m = kf.Mesh(MESH_A)
    hist = m.solve()
    last, want = hist[-1], gold[-1]
    for k in ("lift", "drag", "momn"):
        assert abs(last[k] - float(want[k])) <= 1e-10 * abs(float(want[k]))
    assert hist[0]["gmres_its"] == gold[0]["gmres_its"]


def test_mixed_precision_solve(box_mesh):
    kf.set_mode("fast")
    kf.set_aoa(3.06)
    p = box_mesh(12, seed=2)
    m64 = kf.Mesh(p)
    h64 = m64.solve(ts_max=20, stop_ratio=1e8)
    kf.set_precision(1)
    m32 = kf.Mesh(p)
    h32 = m32.solve(ts_max=20, stop_ratio=1e8)
    assert h32[-1]["fnorm"] / h32[0]["fnorm"] <= 1.0e-8 + 1e-20
    for k in ("lift", "drag", "momn"):
        assert abs(h32[-1][k] - h64[-1][k]) <= 1e-8 * abs(h64[-1][k])
    assert rel(m32.view.q, m64.view.q) < 1e-8


def test_fp32_preconditioner_close_to_oracle(box_mesh):
    kf.set_precision(1)
    m = kf.Mesh(box_mesh(10, seed=3))
    v = m.view
    q = seeded_state(v.q.copy(), 3)
    cdt = port.timestep(m.g, v.nnodes, 50.0, q)
    m.fill(q, cdt)
    M = port.Matrix(m.g)
    M.fill(3.0, q, cdt)
    M.ilu_f32()   # rounds the FP64 blocks first
    m.ilu()
    b = np.random.default_rng(1).standard_normal(v.dofs)
    assert rel(m.sptrsv(b), M.sptrsv_f32(b)) < 1e-5


def test_blas_entry_points():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(12345)
    y = rng.standard_normal(12345)
    s = 0.0
    for t in x:
        s += t * t
    assert kf.api.norm2(x) == np.sqrt(s)
    y2 = y.copy()
    kf.api.axpy(-0.75, x, y2)
    assert np.array_equal(y2, -0.75 * x + y)
    assert np.array_equal(kf.api.new_axpy(2.5, x, y), 2.5 * x + y)
    z = x.copy()
    nrm = kf.api.normalize(z)
    assert nrm == np.sqrt(s)
    assert np.array_equal(z, x * (1.0 / nrm))


@pytest.mark.parametrize("schedule", ["packed", "packed:32", "levels", "syncfree", "persistent", "pdl", "pdl4", "mono",
                                      "mono:8", "mono:4", "mono:16:1", "mono:8:3"])
def test_exact_sptrsv_every_schedule(box_mesh, schedule, monkeypatch):
    """Every triangular-solve schedule (chosen when the device mirror is built;
    for the persistent sweep also lanes per row and CTAs per SM) gives the
    oracle's solve bit for bit in exact mode, FP64 and FP32."""
    parts = schedule.split(":")
    monkeypatch.setenv("KFUN3D_SPTRSV", parts[0])
    if parts[0] == "packed":
        # chunks of 64 rows (256 threads) or 32 rows (128 threads) a CTA; FP64
        # factors through the packed kernels too (by default they take pdl4)
        monkeypatch.setenv("KFUN3D_PK_ROWS", f"{parts[1]},{parts[1]}" if len(parts) > 1 else "64,64")
        monkeypatch.setenv("KFUN3D_PK_FP64", "1")
    elif len(parts) > 1:
        monkeypatch.setenv("KFUN3D_SPTRSV_LANES", parts[1])
    if len(parts) > 2:
        monkeypatch.setenv("KFUN3D_SPTRSV_CTAS", parts[2])
    kf.set_mode("exact")
    kf.set_aoa(3.06)
    m = kf.Mesh(box_mesh(12, seed=31))
    v = m.view
    q = seeded_state(v.q.copy(), 31)
    cdt = port.timestep(m.g, v.nnodes, 40.0, q)
    M = port.Matrix(m.g)
    b = np.random.default_rng(31).standard_normal(v.dofs)
    for prec in (0, 1):
        kf.set_precision(prec)
        m.fill(q, cdt)
        M.fill(3.06, q, cdt)
        m.ilu()
        if prec == 0:
            M.ilu()
            assert np.array_equal(m.sptrsv(b), M.sptrsv(b)), schedule
        else:
            M.ilu_f32()
            assert rel(m.sptrsv(b), M.sptrsv_f32(b)) < 1e-5, schedule
    kf.set_precision(0)
    assert kf.last_status() == 0


@pytest.mark.parametrize("order", ["natural", "morton"])
def test_exact_kernels_any_node_order(box_mesh, order, monkeypatch):
    """The order in which node-centric kernels visit nodes (and the storage
    order of the edge arrays that follows it) leaves every result
    bit-identical to the oracle, through the factor and the triangular
    solves: each node's sums still run over its edges in edge order."""
    monkeypatch.setenv("KFUN3D_NODE_ORDER", order)
    kf.set_mode("exact")
    kf.set_precision(0)
    kf.set_aoa(3.06)
    for path in (box_mesh(12, seed=41), MESH_A):
        m = kf.Mesh(path)
        # the incidence lists, edge storage and visit-order copies built on
        # the device equal the host's sequential build element for element
        assert m.query("lists_match_host") == 1, (order, path)
        assert m.query("visit_order_copies") == (1 if order == "morton" else 0), (order, path)
        v = m.view
        q = seeded_state(v.q.copy(), 41)
        (g1, r1) = m.flux(q)
        (g2, r2) = port.flux(m.g, 3.06, q)
        assert np.array_equal(r1, r2) and all(np.array_equal(a, b) for a, b in zip(g1, g2)), (order, path)
        c1 = m.timestep(37.5, q)
        assert np.array_equal(c1, port.timestep(m.g, v.nnodes, 37.5, q))
        M = port.Matrix(m.g)
        m.fill(q, c1)
        M.fill(3.06, q, c1)
        assert np.array_equal(m.matrix()[2], M.blocks()), (order, path)
        m.ilu()
        M.ilu()
        assert np.array_equal(m.matrix()[2], M.blocks()), (order, path)
        b = np.random.default_rng(42).standard_normal(v.dofs)
        assert np.array_equal(m.sptrsv(b), M.sptrsv(b)), (order, path)
    assert kf.last_status() == 0


def test_exact_factor_on_a_mesh_built_by_the_threaded_host_paths(box_mesh):
    """42^3 (74,088 rows) runs the host-side set-up (incidence lists, visit
    order, level descriptors) on several host threads, and the block pattern
    with its many-CTA scans on the device; factor and solves must still equal
    the oracle's bit for bit."""
    kf.set_mode("exact")
    kf.set_precision(0)
    kf.set_aoa(3.06)
    m = kf.Mesh(box_mesh(42, seed=13))
    v = m.view
    q = seeded_state(v.q.copy(), 13)
    cdt = port.timestep(m.g, v.nnodes, 40.0, q)
    M = port.Matrix(m.g)
    for step in range(2):
        m.fill(q, cdt)
        M.fill(3.06, q, cdt)
        m.ilu()
        M.ilu()
        assert np.array_equal(m.matrix()[2], M.blocks()), step
        b = np.random.default_rng(13 + step).standard_normal(v.dofs)
        assert np.array_equal(m.sptrsv(b), M.sptrsv(b)), step
    assert kf.last_status() == 0


def test_block_pattern_built_on_the_device_equals_the_host_build(box_mesh):
    """The block pattern, transpose map, persistent L slots, last-touched
    lower blocks, level lists and ILU(0) product lists that the device builds
    (setup_device.cu) equal kf_build_pattern's on the host, element for
    element, in the mesh numbering and in the spatial renumbering; meshes from
    one scan block to several, randomly and regularly numbered."""
    kf.set_aoa(3.06)
    for path in (MESH_A, box_mesh(10, seed=3), box_mesh(42, seed=13), box_mesh(23, seed=7, permute=False)):
        kf.set_ilu_order(0)
        m = kf.Mesh(path)
        assert m.query("pattern_matches_host") == 1, path
        assert m.query("lists_match_host") == 1, path
        with pytest.raises(RuntimeError):   # not built yet: the query answers -1
            m.query("spatial_pattern_matches_host")
        kf.clear_status()
        kf.set_ilu_order(1)
        m.flux(m.view.q.copy())    # the first entry point in the spatial order builds it
        assert m.query("spatial_pattern_matches_host") == 1, path
        assert m.query("pattern_matches_host") == 1, path
        assert m.query("pattern_us") > 0 and m.query("setup_us") >= m.query("pattern_us")
    kf.set_ilu_order(0)
    assert kf.last_status() == 0
