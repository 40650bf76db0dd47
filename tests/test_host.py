"""Host-side parts of the product: the native .msh generator/loader and the C ABI.

No compute calls here (no GPU on this machine); the GPU paths are in
test_gpu_*.py.
"""
import os
import re

import numpy as np
import pytest

from conftest import MESH_A, ROOT
import kfun3d_b200 as kf
from oracle import ref


def kuhn_counts(n):
    E = 3 * n * n * (n - 1) + 3 * n * (n - 1) ** 2 + (n - 1) ** 3
    return n ** 3, E, 2 * (n - 1) ** 2, n * n, 5 * 2 * (n - 1) ** 2


@pytest.mark.parametrize("n", [4, 7, 25])
def test_generator_counts_and_closure(box_mesh, n):
    m = kf.Mesh(box_mesh(n, seed=1))
    v = m.view
    N, E, F, Ns, _ = kuhn_counts(n)
    assert (v.nnodes, v.nedges, v.nfaces, v.ns) == (N, E, F, Ns)
    assert v.nf == n ** 3 - (n - 2) ** 3 - (n - 2) ** 2
    # closure of every median-dual control volume
    S = np.zeros((N, 3))
    sv = np.stack([v.xn * v.area, v.yn * v.area, v.zn * v.area], 1)
    np.add.at(S, v.n0, sv)
    np.add.at(S, v.n1, -sv)
    np.add.at(S, v.s_nodes, np.stack(v.s_xyz, 1))
    np.add.at(S, v.f_nodes, np.stack(v.f_xyz, 1))
    assert np.abs(S).max() < 1e-14
    # edges sorted by n0, n0 < n1, unit normals oriented n0 -> n1
    assert np.all(np.diff(v.n0.astype(np.int64)) >= 0)
    assert np.all(v.n0 < v.n1)
    assert np.allclose(v.xn ** 2 + v.yn ** 2 + v.zn ** 2, 1.0)
    X = np.stack(v.xyz, 1)
    d = X[v.n1] - X[v.n0]
    assert np.all((sv * d).sum(1) > 0)


def test_generator_seed_changes_mesh(box_mesh):
    a = kf.Mesh(box_mesh(6, seed=1)).view
    b = kf.Mesh(box_mesh(6, seed=2)).view
    assert not np.array_equal(a.n0, b.n0)


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("n,seed", [(5, 0), (11, 9), (42, 13)])
def test_loader_bit_identical_to_reference_setup(box_mesh, n, seed):
    """42^3 (74,088 nodes) takes the loader's multi-threaded paths (index
    sort, least-squares weights), which must give the same bits."""
    p = box_mesh(n, seed=seed)
    a = kf.Mesh(p).view
    b = ref.RefMesh(p, 3.0, 1).view
    for name in ("n0", "n1", "xn", "yn", "zn", "area", "colors", "s_nodes", "f_nodes", "q"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    for k in range(3):
        assert np.array_equal(a.w0[k], b.w0[k]) and np.array_equal(a.w1[k], b.w1[k])
        assert np.array_equal(a.faces[k], b.faces[k])
        assert np.array_equal(a.xyz[k], b.xyz[k])


def test_loader_rejects_truncated_file(tmp_path):
    data = open(MESH_A, "rb").read()
    p = tmp_path / "bad.msh"
    p.write_bytes(data[:-8])
    with pytest.raises(IOError):
        kf.Mesh(str(p))
    assert kf.last_status() == 5
    kf.clear_status()


def header_functions():
    names = set()
    for h in ("kfun3d_b200.h",):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name not in ("if", "sizeof", "defined"):
                names.add(name)
    return names


def test_library_exports_every_declared_symbol():
    L = kf.lib()
    names = header_functions()
    assert "ComputeFlux" in names and "Kernel" in names and len(names) > 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_settings_roundtrip():
    kf.set_aoa(4.5)
    u, v = kf.freestream()
    assert u == np.cos(4.5 / (180 / np.pi)) and v == np.sin(4.5 / (180 / np.pi))
    kf.set_aoa(3.0)
    kf.set_mode("fast")
    assert kf.get_mode() == 1
    kf.set_mode("exact")
    assert kf.get_mode() == 0
    kf.set_ilu_order("spatial")
    assert kf.get_ilu_order() == 1
    kf.set_ilu_order(0)
    assert kf.get_ilu_order() == 0


def test_matrix_handle_pattern_matches_reference(box_mesh):
    p = box_mesh(7, seed=4)
    m = kf.Mesh(p)
    import ctypes as C
    L = kf.lib()
    nnz = L.kfun3d_matrix_read(m.g, None, None, None)
    ia = np.zeros(m.nnodes + 1, dtype=np.uint32)
    ja = np.zeros(nnz, dtype=np.uint32)
    L.kfun3d_matrix_read(m.g, ia.ctypes.data_as(C.POINTER(C.c_uint)), ja.ctypes.data_as(C.POINTER(C.c_uint)), None)
    from oracle import port
    ia2, ja2, _ = port.Matrix(m.g).pattern()
    assert np.array_equal(ia, ia2) and np.array_equal(ja, ja2)
