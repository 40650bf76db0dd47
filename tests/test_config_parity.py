"""Parity at the benchmark configurations' sizes, against the reference's own runs.

Fixtures (tests/golden/make_golden.py, the reference compiled from its sources
at one OpenMP thread, src/kernel.c:47-232 through the harness):

* box25_history.json -- the plain FP64 CPU-runnable workload's mesh (25^3,
  seed 0, bump 0.1, AoA 3.06), 20 Newton steps of the second-order solve (the
  reference has no first-order flux).  Exact mode must reproduce every step
  (residual norm, CFL, GMRES count, lift, drag, moment) bit for bit.
* box70_forces.json -- the 70^3 mesh (seed 1, bump 0.1, AoA 3.06) solved on
  to a 1e-11 drop, so the history holds the forces at the 1e-8 stop and at the
  tighter stop.  Fast-mode FP64 (FMA, tree reductions: not bit-identical) must
  give the reference's converged forces within 1e-10 relative; the FP32
  preconditioner, with ILU(0) in the mesh's or the spatial elimination order,
  within 1e-8.  Stopping both at a 1e-11 drop separates the form's own error
  from the slack a 1e-8 stop leaves; the forces at the 1e-8 stop are checked
  against the reference's 1e-8 stop as well.
"""
import hashlib
import json
import os

import pytest

from conftest import GOLDEN
import kfun3d_b200 as kf

pytestmark = pytest.mark.gpu


def fixture(name):
    return json.load(open(os.path.join(GOLDEN, name)))


def sha256(path):
    with open(path, "rb") as fh:
        return hashlib.sha256(fh.read()).hexdigest()


def stop_index(steps, ratio):
    """Index of the step at which the reference stops for this drop
    (round(|r0| / |r|) >= ratio on the pre-update norm, src/kernel.c:214)."""
    f0 = float(steps[0]["fnorm"])
    for k, s in enumerate(steps):
        if round(f0 / float(s["fnorm"])) >= ratio:
            return k
    raise AssertionError("the fixture never reaches this drop")


@pytest.fixture(autouse=True)
def defaults():
    kf.set_abort_on_error(True)
    kf.set_first_order(False)
    kf.set_verbose(False)
    yield
    kf.set_mode("exact")
    kf.set_precision(0)
    kf.set_ilu_order(0)
    kf.set_aoa(3.0)


def test_exact_box25_history_is_the_reference(box_mesh):
    gold = fixture("box25_history.json")
    path = box_mesh(25, seed=0, bump=0.1)
    assert sha256(path) == gold["mesh_sha256"], "the generator no longer writes the fixture's mesh"
    kf.set_mode("exact")
    kf.set_precision(0)
    kf.set_ilu_order(0)
    kf.set_aoa(gold["params"]["aoa"])
    m = kf.Mesh(path)
    hist = m.solve(ts_max=gold["params"]["ts_max"], stop_ratio=gold["params"]["stop_ratio"])
    assert len(hist) == len(gold["steps"])
    for h, w in zip(hist, gold["steps"]):
        assert h["gmres_its"] == w["gmres_its"], h["step"]
        for k in ("cfl", "fnorm", "lift", "drag", "momn"):
            assert repr(h[k]) == w[k], (h["step"], k, h[k], w[k])
    m.close()


FORMS = [
    # (name, mode, precision, ILU(0) order, tolerance of the converged forces)
    ("fp64", "fast", 0, 0, 1e-10),
    ("mixed", "fast", 1, 0, 1e-8),
    ("mixed_spatial", "fast", 1, 1, 1e-8),
]


@pytest.mark.parametrize("name,mode,prec,order,tol", FORMS)
def test_box70_forces_against_the_reference(box_mesh, name, mode, prec, order, tol):
    gold = fixture("box70_forces.json")
    steps = gold["steps"]
    path = box_mesh(70, seed=1, bump=0.1)
    assert sha256(path) == gold["mesh_sha256"], "the generator no longer writes the fixture's mesh"
    kf.set_mode(mode)
    kf.set_precision(prec)
    kf.set_ilu_order(order)
    kf.set_aoa(gold["params"]["aoa"])
    m = kf.Mesh(path)
    q0 = m.view.q.copy()
    report = {}
    for ratio in (1e8, gold["params"]["stop_ratio"]):
        m.view.q[:] = q0
        hist = m.solve(ts_max=gold["params"]["ts_max"], stop_ratio=ratio)
        want = steps[stop_index(steps, ratio)]
        err = max(abs(hist[-1][k] - float(want[k])) / abs(float(want[k])) for k in ("lift", "drag", "momn"))
        report[ratio] = (len(hist), sum(h["gmres_its"] for h in hist), err)
        if ratio > 1e8 or name == "fp64":
            assert err <= tol, (name, ratio, report)
    m.close()
    print(name, report)
