"""Host-side pieces of bench.py (no GPU): the reference's own iteration count
read from its committed full runs, and the stand-alone mesh generator that
the reference arm uses instead of the CUDA library."""
import hashlib
import json
import os
import subprocess
import sys

from conftest import GOLDEN, ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_reference_count_from_the_70cube_fixture():
    rc = bench.reference_count(bench.CONFIGS[1])
    steps = json.load(open(os.path.join(GOLDEN, "box70_forces.json")))["steps"]
    # the reference stops at the first step whose pre-update norm is 1e8 below the first
    f0 = float(steps[0]["fnorm"])
    k = next(i for i, s in enumerate(steps) if round(f0 / float(s["fnorm"])) >= 1e8)
    assert rc["newton_steps"] == k + 1
    assert rc["gmres_its"] == sum(s["gmres_its"] for s in steps[:k + 1])
    assert rc["threads"] == 1


def test_standalone_generator_writes_the_library_mesh(tmp_path):
    import kfun3d_b200 as kf
    exe = bench.MESHGEN
    assert os.path.exists(exe), "build kfun3d_b200/csrc first"
    a, b = tmp_path / "a.msh", tmp_path / "b.msh"
    subprocess.run([exe, str(a), "9", "0.12", "4"], check=True)
    kf.generate_mesh(str(b), 9, bump_height=0.12, seed=4)
    assert hashlib.sha256(a.read_bytes()).digest() == hashlib.sha256(b.read_bytes()).digest()
