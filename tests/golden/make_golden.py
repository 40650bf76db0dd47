"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference sources (the path in REF below):
    make -C oracle ref port && make -C kfun3d_b200/csrc
    python tests/golden/make_golden.py                 # the fast fixtures below
    python tests/golden/make_golden.py --configs       # box25 / box70 (about 20 min, one core)
    python tests/golden/make_golden.py --ref-count T   # box120 count (about 30 min on T threads)

Fixtures:
  uns3dA.msh            the reference's own mesh (mesh/uns3dA.msh, MIT licence),
                        the only mesh the reference ships.
  meshA_history.json    known-answer run: the reference built unmodified from its
                        sources (oracle/_ref/kfun3d_hist.out, whose per-step report
                        prints %.17g) on mesh A at one thread.
  meshA_kernels.json    per-kernel digests of the reference's own kernels
                        (oracle/_ref/libkfun3d_ref.so) on mesh A at a seeded state.
  box10_history.json    reference solve on the seeded 10^3 Kuhn-box mesh that
                        kfun3d_mesh_generate writes (AoA 3.06, 1e-8 drop).
  box25_history.json    reference solve on the 25^3 mesh of the plain FP64
                        CPU-runnable workload (seed 0, bump 0.1, AoA 3.06, 20
                        Newton steps, second order: the reference has no
                        first-order flux), one thread, every value %.17g.
  box70_forces.json     reference solve on the 70^3 mesh (seed 1, bump 0.1, AoA
                        3.06) at one thread, run on to a 1e-11 drop so that the
                        forces at the 1e-8 stop and at the tighter stop are both
                        in the history.
  box120_reference_count.json
                        the reference's own Newton steps, GMRES iterations and
                        wall time to the 1e-8 drop on the 120^3 held-out mesh
                        (seed 4, bump 0.12, AoA 4.5) at T OpenMP threads: the
                        iteration count the CPU baseline extrapolates to.
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import ref  # noqa: E402
import kfun3d_b200 as kf  # noqa: E402

REF = "/root/reference"
GOLD = os.path.join(ROOT, "tests", "golden")


def digest(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64)) + 0.0   # -0.0 -> 0.0
    return hashlib.sha256(a.tobytes()).hexdigest()


def seeded_state(q0, seed):
    rng = np.random.default_rng(seed)
    return q0 + rng.uniform(-0.05, 0.05, q0.shape)


def history_from_binary():
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "mesh"))
        os.symlink(os.path.join(REF, "mesh", "uns3dA.msh"), os.path.join(d, "mesh", "uns3dA.msh"))
        out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "kfun3d_hist.out"), "-m", "A", "-t", "1"],
                             cwd=d, capture_output=True, text=True, check=True).stdout
    steps, its = [], None
    for line in out.splitlines():
        line = line.replace("\x1b[36m", "").replace("\x1b[0m", "")
        if "TOTAL ITERATIONS" in line:
            its = int(line.split()[-1])
        elif line.startswith("STEP:"):
            t = line.split()
            steps.append(dict(step=int(t[1]), cfl=float(t[3]), fnorm=float(t[5]), gmres_its=its))
        elif line.startswith("LIFT:"):
            t = line.split()
            steps[-1].update(lift=float(t[1]), drag=float(t[3]), momn=float(t[5]))
    return steps


def kernel_digests(path, aoa, seed):
    m = ref.RefMesh(path, aoa, 1)
    v = m.view
    q = seeded_state(v.q.copy(), seed)
    (gx, gy, gz), r = m.flux(q)
    cdt = m.timestep(37.5, q)
    _, _, _, A = m.fill(q, cdt)
    _, _, _, F = m.ilu()
    b = np.random.default_rng(seed + 1).standard_normal(v.dofs)
    x = m.sptrsv(b)
    f = m.forces(q)
    out = dict(seed=seed, aoa=aoa, cfl=37.5,
               setup=dict(n0=digest(v.n0.astype(np.float64)), n1=digest(v.n1.astype(np.float64)),
                          w0=[digest(w) for w in v.w0], w1=[digest(w) for w in v.w1],
                          faces=[digest(f_.astype(np.float64)) for f_ in v.faces],
                          colors=[int(c) for c in v.colors]),
               r=digest(r), gx=digest(gx), gy=digest(gy), gz=digest(gz), cdt=digest(cdt),
               A=digest(A), F=digest(F), x=digest(x), forces=[repr(float(t)) for t in f],
               samples=dict(r=[repr(float(t)) for t in r[::997]], F=[repr(float(t)) for t in F.ravel()[::4999]]))
    m.close()
    return out


def main():
    hist = history_from_binary()
    with open(os.path.join(GOLD, "meshA_history.json"), "w") as fh:
        json.dump(dict(source="oracle/_ref/kfun3d_hist.out -m A -t 1 (reference, unmodified sources)",
                       steps=[{k: (repr(v) if isinstance(v, float) else v) for k, v in s.items()} for s in hist]),
                  fh, indent=1)
    with open(os.path.join(GOLD, "meshA_kernels.json"), "w") as fh:
        json.dump(kernel_digests(os.path.join(REF, "mesh", "uns3dA.msh"), 3.0, 7), fh, indent=1)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "box10.msh")
        kf.generate_mesh(p, 10, seed=3)
        m = ref.RefMesh(p, 3.06, 1)
        h = m.solve(ts_max=20, stop_ratio=1e8)
        kd = kernel_digests(p, 3.06, 11)
        with open(p, "rb") as fh:
            mesh_digest = hashlib.sha256(fh.read()).hexdigest()
    with open(os.path.join(GOLD, "box10_history.json"), "w") as fh:
        json.dump(dict(source="oracle/_ref/libkfun3d_ref.so ref_solve, kfun3d_mesh_generate(n=10, seed=3)",
                       mesh_sha256=mesh_digest, params=dict(aoa=3.06, ts_max=20, stop_ratio=1e8),
                       steps=[{k: (repr(v) if isinstance(v, float) else v) for k, v in s.items()} for s in h],
                       kernels=kd), fh, indent=1)
    print("golden fixtures written to", GOLD)


def _mesh(d, n, seed, bump):
    p = os.path.join(d, f"box{n}.msh")
    kf.generate_mesh(p, n, bump_height=bump, seed=seed)
    with open(p, "rb") as fh:
        return p, hashlib.sha256(fh.read()).hexdigest()


def _steps(h):
    return [{k: (repr(v) if isinstance(v, float) else v) for k, v in s.items()} for s in h]


def config_fixtures():
    """box25_history.json and box70_forces.json (one thread, the deterministic
    reference path: src/kernel.c:47-232 through the harness's ref_solve)."""
    import time
    with tempfile.TemporaryDirectory() as d:
        p, sha = _mesh(d, 25, 0, 0.1)
        m = ref.RefMesh(p, 3.06, 1)
        params = dict(ts_max=20, stop_ratio=1e30)
        t0 = time.perf_counter()
        h = m.solve(**params)
        dt = time.perf_counter() - t0
        m.close()
        with open(os.path.join(GOLD, "box25_history.json"), "w") as fh:
            json.dump(dict(source="oracle/_ref/libkfun3d_ref.so ref_solve at 1 thread, "
                                  "kfun3d_mesh_generate(n=25, seed=0, bump_height=0.1)",
                           mesh_sha256=sha, params=dict(aoa=3.06, **params), seconds=dt,
                           steps=_steps(h)), fh, indent=1)
        print("box25:", len(h), "steps", sum(s["gmres_its"] for s in h), "its", f"{dt:.1f} s", flush=True)
        p, sha = _mesh(d, 70, 1, 0.1)
        m = ref.RefMesh(p, 3.06, 1)
        params = dict(ts_max=40, stop_ratio=1e11)
        t0 = time.perf_counter()
        h = m.solve(**params)
        dt = time.perf_counter() - t0
        m.close()
        with open(os.path.join(GOLD, "box70_forces.json"), "w") as fh:
            json.dump(dict(source="oracle/_ref/libkfun3d_ref.so ref_solve at 1 thread, "
                                  "kfun3d_mesh_generate(n=70, seed=1, bump_height=0.1)",
                           mesh_sha256=sha, params=dict(aoa=3.06, **params), seconds=dt,
                           steps=_steps(h)), fh, indent=1)
        print("box70:", len(h), "steps", sum(s["gmres_its"] for s in h), "its", f"{dt:.1f} s", flush=True)


def reference_count(threads):
    """box120_reference_count.json: the reference's full solve at `threads`
    OpenMP threads (its ILU(0) is then a racing Chow-Patel sweep,
    matrix/ilu.cpp:49-97, so the count belongs to this thread count)."""
    import platform
    import time
    with tempfile.TemporaryDirectory() as d:
        p, sha = _mesh(d, 120, 4, 0.12)
        t0 = time.perf_counter()
        m = ref.RefMesh(p, 4.5, threads)
        t_setup = time.perf_counter() - t0
        params = dict(ts_max=20, stop_ratio=1e8)
        t0 = time.perf_counter()
        h = m.solve(**params)
        dt = time.perf_counter() - t0
        m.close()
    cpu = platform.processor() or platform.machine()
    try:
        with open("/proc/cpuinfo") as fh:
            cpu = next(l.split(":", 1)[1].strip() for l in fh if l.startswith("model name"))
    except (OSError, StopIteration):
        pass
    out = dict(source=f"oracle/_ref/libkfun3d_ref.so ref_solve at {threads} threads, "
                      "kfun3d_mesh_generate(n=120, seed=4, bump_height=0.12)",
               command=f"python tests/golden/make_golden.py --ref-count {threads}",
               mesh_sha256=sha, params=dict(aoa=4.5, **params), threads=threads, cpu=cpu,
               setup_seconds=t_setup, solve_seconds=dt, newton_steps=len(h),
               gmres_its=sum(s["gmres_its"] for s in h), steps=_steps(h))
    with open(os.path.join(GOLD, "box120_reference_count.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("box120:", out["newton_steps"], "steps", out["gmres_its"], "its", f"{dt:.1f} s", flush=True)


if __name__ == "__main__":
    if "--configs" in sys.argv:
        config_fixtures()
    elif "--ref-count" in sys.argv:
        reference_count(int(sys.argv[sys.argv.index("--ref-count") + 1]))
    else:
        main()
