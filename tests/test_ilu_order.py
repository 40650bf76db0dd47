"""ILU(0) in a spatial elimination order (slab sweeps; tiles, one sweep or
Morton on request).

* through the renumbering code with the identity permutation the factor, the
  triangular solves and a whole exact-mode solve are bit-identical to the
  mesh order: the renumbering adds nothing of its own;
* with each of those permutations the device computes P^T (LU)^-1 P b where LU is
  the reference's ILU(0) (matrix/ilu.cpp:49-136, persistent L slots included)
  of the renumbered matrix P A P^T: checked bit for bit against the oracle's
  ILU(0) and triangular solve run on the renumbered pattern and blocks;
* on a randomly numbered mesh the spatial order converges to the same state
  in fewer GMRES iterations.
"""
import ctypes as C

import numpy as np
import pytest

import kfun3d_b200 as kf
from oracle import port
from conftest import seeded_state

P = dict(ts_max=20, stop_ratio=1e8)


@pytest.fixture(autouse=True)
def _settings(monkeypatch):
    aoa, mode = kf.get_aoa(), kf.get_mode()
    kf.set_aoa(3.06)
    kf.set_precision(0)
    kf.set_ilu_order(0)
    monkeypatch.delenv("KFUN3D_ILU_PERM", raising=False)
    monkeypatch.delenv("KFUN3D_SPTRSV", raising=False)
    yield
    kf.set_ilu_order(0)
    kf.set_precision(0)
    kf.set_mode(mode)
    kf.set_aoa(aoa)


def sweep_rank(xyz):
    """Position of every node in ascending x + y + z, ties in node order (the
    order kfun3d_set_ilu_order(1) builds)."""
    key = (xyz[0] + xyz[1]) + xyz[2]
    order = np.argsort(key, kind="stable")
    rank = np.empty(key.size, dtype=np.int64)
    rank[order] = np.arange(key.size)
    return rank


def morton_rank(xyz):
    """Position of every node in the Morton order of its coordinates: 21 bits
    per axis over the bounding box, ties in node order (the order built with
    KFUN3D_ILU_PERM=morton)."""
    N = xyz[0].size
    key = np.zeros(N, dtype=np.uint64)
    for d, c in enumerate(xyz):
        lo, hi = c.min(), c.max()
        span = hi - lo if hi > lo else 1.0
        b = np.minimum(2097151.0, np.maximum(0.0, (c - lo) / span * 2097151.0)).astype(np.uint64)
        v = np.zeros(N, dtype=np.uint64)
        for bit in range(21):
            v |= ((b >> np.uint64(bit)) & np.uint64(1)) << np.uint64(3 * bit)
        key |= v << np.uint64(d)
    order = np.argsort(key, kind="stable")
    rank = np.empty(N, dtype=np.int64)
    rank[order] = np.arange(N)
    return rank


class Renumbered:
    """The oracle's BSR of P A P^T: the pattern built as orc_bsr_create builds
    it from the renumbered edge list, the blocks of a filled oracle matrix
    moved to their renumbered places, and the persistent L slots as a fill
    from a fresh state leaves them (the last lower block of each row in its
    row's first slot)."""

    def __init__(self, M, rank, n0, n1):
        N = M.n
        ia0, ja0, _ = M.pattern()
        A0 = M.blocks().reshape(-1, 16)
        r0, r1 = rank[n0.astype(np.int64)], rank[n1.astype(np.int64)]
        rows = np.concatenate([np.arange(N), r0, r1])
        cols = np.concatenate([np.arange(N), r1, r0])
        o = np.lexsort((cols, rows))
        rows, cols = rows[o], cols[o]
        self.ia = np.zeros(N + 1, dtype=np.uint32)
        self.ia[1:] = np.cumsum(np.bincount(rows, minlength=N))
        self.ja = cols.astype(np.uint32)
        key = rows * N + cols
        self.diag = np.searchsorted(key, np.arange(N) * N + np.arange(N)).astype(np.uint32)
        self.lpos = np.zeros(N + 1, dtype=np.uint32)
        self.lpos[1:] = np.cumsum(self.diag - self.ia[:-1])
        i0 = np.repeat(np.arange(N), np.diff(ia0.astype(np.int64)))
        dst = np.searchsorted(key, rank[i0] * N + rank[ja0.astype(np.int64)])
        self.a = np.zeros((key.size, 16))
        self.a[dst] = A0
        self.a = self.a.reshape(-1)
        self.af = np.zeros(self.a.size, dtype=np.float32)
        ll = np.full(N, -1, dtype=np.int64)
        for a, b in zip(r0, r1):
            if b < a:
                ll[a] = b
            if a < b:
                ll[b] = a
        self.last_lower = np.full(N, 0xFFFFFFFF, dtype=np.uint32)
        self.lslot = np.zeros(int(self.lpos[N]) * 16 + 16)
        for i in np.nonzero(ll >= 0)[0]:
            j = int(np.searchsorted(key, i * N + ll[i]))
            self.last_lower[i] = j
            self.lslot[16 * int(self.lpos[i]):16 * int(self.lpos[i]) + 16] = self.a[16 * j:16 * j + 16]
        u32 = C.POINTER(C.c_uint32)
        self.bsr = port.BSR(N, key.size, self.ia.ctypes.data_as(u32), self.ja.ctypes.data_as(u32),
                            self.diag.ctypes.data_as(u32), port.dptr(self.a),
                            self.af.ctypes.data_as(C.POINTER(C.c_float)), port.dptr(self.lslot),
                            self.lpos.ctypes.data_as(u32), self.last_lower.ctypes.data_as(u32))

    def ilu(self):
        port.lib().orc_ilu(C.byref(self.bsr))

    def ilu_f32(self):
        port.lib().orc_round_f32(C.byref(self.bsr))
        port.lib().orc_ilu_f32(C.byref(self.bsr))

    def sptrsv(self, b, f32=False):
        x = np.zeros_like(b)
        fn = port.lib().orc_sptrsv_f32 if f32 else port.lib().orc_sptrsv
        fn(C.byref(self.bsr), port.dptr(np.ascontiguousarray(b)), port.dptr(x))
        return x


def _to_spatial(v, rank):
    out = np.empty_like(v.reshape(-1, 4))
    out[rank] = v.reshape(-1, 4)
    return out.reshape(-1)


def _from_spatial(v, rank):
    return v.reshape(-1, 4)[rank].reshape(-1)


def test_renumbered_helper_with_identity_is_the_oracle(box_mesh):
    """The renumbered oracle matrix with the identity permutation factors and
    solves exactly as the oracle's own matrix does (no GPU)."""
    m = kf.Mesh(box_mesh(7, seed=34))
    v = m.view
    q = seeded_state(v.q.copy(), 34)
    cdt = port.timestep(m.g, v.nnodes, 29.0, q)
    M = port.Matrix(m.g)
    M.fill(3.06, q, cdt)
    R = Renumbered(M, np.arange(v.nnodes), v.n0, v.n1)
    assert np.array_equal(R.a.reshape(-1, 4, 4), M.blocks())
    M.ilu()
    R.ilu()
    b = np.random.default_rng(9).standard_normal(v.dofs)
    assert np.array_equal(M.sptrsv(b), R.sptrsv(b))


def _depth(n0, n1, rank):
    """Number of level sets of the lower triangle of the pattern renumbered by
    `rank`: depth(i) = 1 + max depth of its lower neighbours (the definition of
    matrix/init.cpp:194-232), restated with Python loops."""
    N = rank.size
    a, b = rank[n0.astype(np.int64)], rank[n1.astype(np.int64)]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    o = np.argsort(hi, kind="stable")
    ptr = np.zeros(N + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(np.bincount(hi[o], minlength=N))
    low = lo[o].tolist()
    depth = [1] * N
    for i in range(N):
        if ptr[i] < ptr[i + 1]:
            depth[i] = 1 + max(depth[j] for j in low[ptr[i]:ptr[i + 1]])
    return max(depth)


@pytest.mark.parametrize("perm", ["identity", "slabs", "sweep", "tiles", "morton"])
def test_plan_on_the_host(box_mesh, perm, monkeypatch):
    """kfun3d_ilu_order_plan (no GPU): every order is a permutation, the sweep
    and Morton orders are the ones restated above, and the level counts of
    both triangular sweeps are those of the renumbered pattern."""
    if perm != "slabs":
        monkeypatch.setenv("KFUN3D_ILU_PERM", perm)
    m = kf.Mesh(box_mesh(11, seed=36))
    v = m.view
    rank, nl, nu = m.ilu_order_plan(tiles=16)
    N = v.nnodes
    assert np.array_equal(np.sort(rank), np.arange(N))
    xyz = [c.copy() for c in v.xyz]
    if perm == "identity":
        assert np.array_equal(rank, np.arange(N))
    if perm == "sweep":
        assert np.array_equal(rank, sweep_rank(xyz))
    if perm == "morton":
        assert np.array_equal(rank, morton_rank(xyz))
    assert nl == _depth(v.n0, v.n1, rank)
    assert nu == _depth(v.n0, v.n1, N - 1 - rank)


@pytest.mark.parametrize("perm", ["sweep", "morton"])
def test_plan_threaded_sort_on_a_large_mesh(box_mesh, perm, monkeypatch):
    """42^3 (74,088 nodes) sorts on several host threads (chunks sorted, then
    merged pairwise, ties by node index); the order must still be exactly the
    stable sort restated above."""
    monkeypatch.setenv("KFUN3D_ILU_PERM", perm)
    m = kf.Mesh(box_mesh(42, seed=13))
    rank, _, _ = m.ilu_order_plan()
    xyz = [c.copy() for c in m.view.xyz]
    assert np.array_equal(rank, sweep_rank(xyz) if perm == "sweep" else morton_rank(xyz))


def test_plan_slab_sweeps_have_fewer_levels(box_mesh, monkeypatch):
    m = kf.Mesh(box_mesh(20, seed=37))
    _, nl_slabs, _ = m.ilu_order_plan()
    monkeypatch.setenv("KFUN3D_ILU_PERM", "sweep")
    _, nl_sweep, _ = m.ilu_order_plan()
    monkeypatch.setenv("KFUN3D_ILU_PERM", "identity")
    _, nl_mesh, _ = m.ilu_order_plan()
    # a sweep orders the mesh like a lattice (about 3n levels); four slabs,
    # each swept from both faces, cut that several times
    assert nl_slabs < nl_sweep / 2, (nl_slabs, nl_sweep, nl_mesh)


@pytest.mark.gpu
def test_identity_renumbering_is_the_mesh_order(box_mesh, monkeypatch):
    """Set 1 built with the identity permutation: bit-identical factor,
    triangular solves and solve history."""
    kf.set_mode("exact")
    path = box_mesh(9, seed=31)
    ref = kf.Mesh(path)
    monkeypatch.setenv("KFUN3D_ILU_PERM", "identity")
    m = kf.Mesh(path)
    q = seeded_state(ref.view.q.copy(), 31)
    cdt = ref.timestep(41.0, q)
    for prec in (0, 1):
        kf.set_precision(prec)
        for step in range(2):
            qs = q + 0.01 * step
            kf.set_ilu_order(0)
            ref.fill(qs, cdt)
            ref.ilu()
            b = np.random.default_rng(step).standard_normal(ref.view.dofs)
            x0 = ref.sptrsv(b)
            kf.set_ilu_order(1)
            m.fill(qs, cdt)
            m.ilu()
            x1 = m.sptrsv(b)
            assert np.array_equal(x0, x1), (prec, step)
    kf.set_precision(0)
    kf.set_ilu_order(0)
    ref.reset_state()
    h0 = ref.solve(**P)
    kf.set_ilu_order(1)
    m.reset_state()
    h1 = m.solve(**P)
    assert [s["gmres_its"] for s in h0] == [s["gmres_its"] for s in h1]
    assert [s["fnorm"] for s in h0] == [s["fnorm"] for s in h1]
    assert np.array_equal(ref.view.q, m.view.q)
    assert kf.last_status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("perm", ["slabs", "tiles", "sweep", "morton"])
def test_spatial_factor_is_the_renumbered_reference_factor(box_mesh, prec, perm, monkeypatch):
    kf.set_mode("exact")
    kf.set_precision(prec)
    aoa = 3.06
    if perm != "slabs":
        monkeypatch.setenv("KFUN3D_ILU_PERM", perm)
    m = kf.Mesh(box_mesh(8, seed=32))
    v = m.view
    q = seeded_state(v.q.copy(), 32)
    cdt = m.timestep(29.0, q)
    kf.set_ilu_order(1)
    m.fill(q, cdt)
    m.ilu()
    b = np.random.default_rng(5).standard_normal(v.dofs)
    x = m.sptrsv(b)
    rank = m.ilu_rank()
    xyz = [c.copy() for c in v.xyz]
    assert np.array_equal(np.sort(rank), np.arange(v.nnodes))
    assert not np.array_equal(rank, np.arange(v.nnodes))
    if perm == "sweep":
        assert np.array_equal(rank, sweep_rank(xyz))
    if perm == "morton":
        assert np.array_equal(rank, morton_rank(xyz))
    M = port.Matrix(m.g)
    M.fill(aoa, q, cdt)
    R = Renumbered(M, rank, v.n0, v.n1)
    if prec == 0:
        R.ilu()
        y = _from_spatial(R.sptrsv(_to_spatial(b, rank)), rank)
        assert np.array_equal(x, y)
    else:
        R.ilu_f32()
        y = _from_spatial(R.sptrsv(_to_spatial(b, rank), f32=True), rank)
        assert float(np.max(np.abs(x - y)) / np.max(np.abs(y))) < 1e-5
    # the mesh-order factor is a different preconditioner
    kf.set_ilu_order(0)
    m.fill(q, cdt)
    m.ilu()
    assert not np.allclose(m.sptrsv(b), x, rtol=1e-3)
    # with the spatial order active the raw block and allocation-free readers refuse
    kf.set_ilu_order(1)
    m.fill(q, cdt)
    m.ilu()
    with pytest.raises(RuntimeError):
        m.matrix()
    kf.clear_status()
    assert kf.last_status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("perm", ["slabs", "tiles"])
@pytest.mark.parametrize("n", [13, 30])
def test_spatial_sweep_every_schedule(box_mesh, n, perm, monkeypatch):
    """The packed level launches (default for the spatial order; chunks of 64
    and of 32 rows), one launch per level with four lanes per row and with
    sixteen, the persistent sweep and the sync-free sweep give bit-identical
    triangular solves on the spatial factor (exact mode)."""
    kf.set_mode("exact")
    if perm != "slabs":
        monkeypatch.setenv("KFUN3D_ILU_PERM", perm)
    path = box_mesh(n, seed=35)
    out = {}
    monkeypatch.setenv("KFUN3D_PK_FP64", "1")   # FP64 factors through the packed kernels too
    for sched in ["packed", "packed:32", "pdl4", "pdl", "mono", "syncfree"]:
        monkeypatch.delenv("KFUN3D_PK_ROWS", raising=False)
        if sched == "packed":
            monkeypatch.delenv("KFUN3D_SPTRSV", raising=False)
        else:
            monkeypatch.setenv("KFUN3D_SPTRSV", sched.split(":")[0])
            if ":" in sched:
                monkeypatch.setenv("KFUN3D_PK_ROWS", "32,32")
            else:
                monkeypatch.setenv("KFUN3D_PK_ROWS", "64,64")
        kf.set_ilu_order(0)
        m = kf.Mesh(path)
        q = seeded_state(m.view.q.copy(), 35)
        cdt = m.timestep(33.0, q)
        kf.set_ilu_order(1)
        for prec in (0, 1):
            kf.set_precision(prec)
            m.fill(q, cdt)
            m.ilu()
            b = np.random.default_rng(prec).standard_normal(m.view.dofs)
            out[sched, prec] = m.sptrsv(b)
            assert kf.last_status() == 0, (sched, prec)
        m.close()
    for (sched, prec), x in out.items():
        assert np.array_equal(x, out["packed", prec]), (sched, prec)


@pytest.mark.gpu
def test_spatial_order_fewer_iterations_same_state(box_mesh):
    kf.set_mode("fast")
    kf.set_precision(1)
    path = box_mesh(22, seed=33)
    m = kf.Mesh(path)
    q0 = m.view.q.copy()
    h0 = m.solve(**P)
    qa = m.view.q.copy()
    kf.set_ilu_order(1)
    m.view.q[:] = q0
    h1 = m.solve(**P)
    qb = m.view.q.copy()
    its0, its1 = sum(s["gmres_its"] for s in h0), sum(s["gmres_its"] for s in h1)
    assert h1[0]["fnorm"] / h1[-1]["fnorm"] >= 1e8
    assert its1 < 0.9 * its0, (its0, its1)
    f0 = np.array([h0[-1]["lift"], h0[-1]["drag"], h0[-1]["momn"]])
    f1 = np.array([h1[-1]["lift"], h1[-1]["drag"], h1[-1]["momn"]])
    assert np.allclose(f0, f1, rtol=1e-6, atol=0)
    assert float(np.max(np.abs(qa - qb)) / np.max(np.abs(qa))) < 1e-6
    # the flexible form follows the same order
    m.view.q[:] = q0
    hf, st = m.solve_flexible(**P)
    assert [s["gmres_its"] for s in hf] == [s["gmres_its"] for s in h1]
