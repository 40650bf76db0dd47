"""The drop-in itself: the reference's own host driver linked against the library.

oracle/_ref/kfun3d_dropin.out is the reference's src/main.c, src/mesh.c and
set-up sources (compiled unmodified from the reference tree by `make -C oracle
dropin`) linked against kfun3d_b200/_lib/libkfun3d_b200.so in place of the
reference's kernel and matrix sources (src/flux.c, fill.c, ..., kernel.c,
matrix/*.cpp).  Run as the reference is run (`-m A -t 1`, src/main.c:23-59),
its per-step report must equal the reference binary's known-answer output
(tests/golden/meshA_history.json) at the printed precision (%g,
src/kernel.c:208-212), GMRES iteration counts included.
"""
import json
import os
import re
import shutil
import subprocess

import pytest

from conftest import GOLDEN, MESH_A, ROOT

DROPIN = os.path.join(ROOT, "oracle", "_ref", "kfun3d_dropin.out")
ANSI = re.compile(r"\x1b\[[0-9;]*m")


def run_dropin(tmp_path, threads):
    if not os.path.exists(DROPIN):
        pytest.fail(f"{DROPIN} missing: build it with `make -C oracle ref dropin` where the reference sources are")
    os.makedirs(tmp_path / "mesh", exist_ok=True)
    shutil.copy(MESH_A, tmp_path / "mesh" / "uns3dA.msh")
    return subprocess.run([DROPIN, "-m", "A", "-t", str(threads)], cwd=tmp_path, capture_output=True,
                          text=True, timeout=300)


def report(stdout):
    """(gmres_its, 'STEP: ... NORM: ...', 'LIFT: ... MOMN: ...') per Newton step."""
    steps, its = [], None
    lines = [ANSI.sub("", l).strip() for l in stdout.splitlines()]
    for k, line in enumerate(lines):
        if "TOTAL ITERATIONS" in line:
            its = int(line.split()[-1])
        elif line.startswith("STEP:"):
            steps.append((its, line, lines[k + 1]))
    return steps


@pytest.mark.gpu
def test_reference_driver_through_the_library(tmp_path):
    p = run_dropin(tmp_path, 1)
    assert p.returncode == 0, p.stderr[-2000:]
    got = report(p.stdout)
    gold = json.load(open(os.path.join(GOLDEN, "meshA_history.json")))["steps"]
    want = [(s["gmres_its"],
             "STEP: %d CFL: %g NORM: %g" % (s["step"], float(s["cfl"]), float(s["fnorm"])),
             "LIFT: %g DRAG: %g MOMN: %g" % (float(s["lift"]), float(s["drag"]), float(s["momn"])))
            for s in gold]
    assert got == want, "\n".join(f"{g}\n{w}" for g, w in zip(got, want))


@pytest.mark.gpu
def test_reference_driver_refuses_a_threaded_geometry(tmp_path):
    """Setup at two threads replicates cut edges (src/subdomains.c); the
    library refuses that GEOMETRY and, like the reference's asserts, ends the
    process with a message instead of printing nothing."""
    p = run_dropin(tmp_path, 2)
    assert p.returncode != 0
    assert "more than one OpenMP thread" in p.stderr
    assert "STEP:" not in p.stdout
