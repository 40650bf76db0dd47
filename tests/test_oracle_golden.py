"""The C oracle against the golden fixtures produced by the reference itself.

Fixtures (tests/golden/, made by make_golden.py from oracle/_ref): the
known-answer history of the unmodified reference on its own mesh A, digests
of the reference's kernels on mesh A at a seeded state, and the reference's
solve on the seeded 10^3 Kuhn box.  Every comparison is bit-exact.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, MESH_A, seeded_state
import kfun3d_b200 as kf
from oracle import port


def digest(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64)) + 0.0
    return hashlib.sha256(a.tobytes()).hexdigest()


def load(name):
    with open(os.path.join(GOLDEN, name)) as fh:
        return json.load(fh)


def check_history(got, want):
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert g["gmres_its"] == w["gmres_its"]
        for k in ("cfl", "fnorm", "lift", "drag", "momn"):
            assert repr(float(g[k])) == w[k], (g["step"], k, g[k], w[k])


def test_oracle_meshA_known_answer():
    """Bit-identical to the reference binary's printed history (8 steps)."""
    m = kf.Mesh(MESH_A)
    q = m.view.q.copy()
    hist = port.solve(m.g, 3.0, q)
    check_history(hist, load("meshA_history.json")["steps"])


def test_oracle_meshA_kernels():
    gold = load("meshA_kernels.json")
    m = kf.Mesh(MESH_A)
    v = m.view
    q = seeded_state(v.q.copy(), gold["seed"])
    (gx, gy, gz), r = port.flux(m.g, gold["aoa"], q)
    assert digest(r) == gold["r"]
    assert [digest(gx), digest(gy), digest(gz)] == [gold["gx"], gold["gy"], gold["gz"]]
    cdt = port.timestep(m.g, v.nnodes, gold["cfl"], q)
    assert digest(cdt) == gold["cdt"]
    M = port.Matrix(m.g)
    M.fill(gold["aoa"], q, cdt)
    assert digest(M.blocks()) == gold["A"]
    M.ilu()
    assert digest(M.blocks()) == gold["F"]
    b = np.random.default_rng(gold["seed"] + 1).standard_normal(v.dofs)
    assert digest(M.sptrsv(b)) == gold["x"]
    f = port.forces(m.g, gold["aoa"], q)
    assert [repr(float(t)) for t in f] == gold["forces"]


def test_loader_matches_reference_setup_digests():
    gold = load("meshA_kernels.json")["setup"]
    v = kf.Mesh(MESH_A).view
    assert digest(v.n0.astype(np.float64)) == gold["n0"]
    assert digest(v.n1.astype(np.float64)) == gold["n1"]
    assert [digest(w) for w in v.w0] == gold["w0"]
    assert [digest(w) for w in v.w1] == gold["w1"]
    assert [digest(f.astype(np.float64)) for f in v.faces] == gold["faces"]
    assert [int(c) for c in v.colors] == gold["colors"]


def test_generator_is_reproducible_and_oracle_matches_box10(box_mesh):
    gold = load("box10_history.json")
    p = box_mesh(10, seed=3)
    with open(p, "rb") as fh:
        assert hashlib.sha256(fh.read()).hexdigest() == gold["mesh_sha256"]
    kf.set_aoa(3.06)
    try:
        m = kf.Mesh(p)
        q = m.view.q.copy()
        hist = port.solve(m.g, 3.06, q, ts_max=20, stop_ratio=1e8)
        check_history(hist, gold["steps"])
        kd = gold["kernels"]
        qs = seeded_state(m.view.q.copy(), kd["seed"])
        (_, _, _), r = port.flux(m.g, 3.06, qs)
        assert digest(r) == kd["r"]
    finally:
        kf.set_aoa(3.0)


def test_generator_writes_the_config_fixture_meshes_and_oracle_matches_box25(box_mesh):
    """The 25^3 (seed 0) and 70^3 (seed 1) meshes of the config fixtures are
    what the generator writes today; the oracle repeats the reference's 25^3
    history (first 8 Newton steps, bit for bit)."""
    for name, n, seed in (("box25_history.json", 25, 0), ("box70_forces.json", 70, 1)):
        path = os.path.join(GOLDEN, name)
        if not os.path.exists(path):
            continue
        gold = json.load(open(path))
        with open(box_mesh(n, seed=seed, bump=0.1), "rb") as fh:
            assert hashlib.sha256(fh.read()).hexdigest() == gold["mesh_sha256"], name
    gold = load("box25_history.json")
    kf.set_aoa(3.06)
    try:
        m = kf.Mesh(box_mesh(25, seed=0, bump=0.1))
        q = m.view.q.copy()
        hist = port.solve(m.g, 3.06, q, ts_max=8, stop_ratio=1e30)
        check_history(hist, gold["steps"][:8])
    finally:
        kf.set_aoa(3.0)
