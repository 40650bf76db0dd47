#!/usr/bin/env python
"""One-line benchmark of the kfun3d_b200 hot path (pseudo-transient Newton-Krylov).

Workload (N = 1): the config-4 comparison -- the 120^3 seeded Kuhn-box mesh
(1,728,000 nodes, 11,923,919 edges, bump 0.12, angle of attack 4.5, both
held out of the network's training set, jitter 0.2h, random numbering),
second-order residual, SER CFL from 50, at most 20 Newton steps, stopped at a
1e-8 drop of the residual norm.  A step is one solve from the free-stream
state in the mixed-precision + learned form (FP32 Jacobian blocks, ILU(0) in
the spatial elimination order and FP32 triangular solves; FP64 residual,
norms, CFL, Gram-Schmidt and Givens; flexible GMRES(30) with the trained
network as right preconditioner and its fallback).  `comparison` holds, on
the same mesh, the plain FP64 solve (the reference's method: FP64, ILU(0) in
the mesh's numbering), the same mixed solve without the network, the mixed
solve in the mesh's numbering, and the wall forces' relative error against
FP64, with the ladder between them (FP64 in the spatial order, FP32 in the
spatial order without the network) so that the ordering, the precision and
the network each show their own gain.  The metric is seconds to the 1e-8 drop
(lower is better), with flux edges/s and the other kernel throughputs beside
it.  --config 1 runs the 70^3 plain FP64 solve instead.

value    device-resident: state and mesh already in HBM, CUDA events on the
         solver's stream around each solve, max over ranks.
e2e      the same solve through the C ABI with host buffers
         (kfun3d_solve_flexible / kfun3d_solve: state uploaded, solved, state
         and time step downloaded), wall clock.
roofline the kernel family with the largest share of one GMRES iteration,
         algorithmic bytes (per-kernel formulas below) / its CUDA-event time,
         against MEASURED_PEAKS.json's HBM copy bandwidth.
cpu_baseline / --impl reference: the reference itself (oracle/_ref, built from
         its own sources) on all host cores, timed on a bounded sample (its
         first Newton step(s)) and extrapolated by GMRES iterations to the
         reference's own iteration count, taken from a full run of the
         reference committed under tests/golden/ (make_golden.py).  The
         reference arm never loads the CUDA library: its mesh comes from the
         stand-alone generator program kfun3d_meshgen.

Multi-GPU: replicas (one independent mesh per GPU, no collective on the data
path); `scaling` is weak.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to 1e-8 residual drop: mixed+learned vs plain FP64 on 1 B200; flux edges/s"

CONFIGS = {
    0: dict(workload="config0: 25^3 Kuhn box, first-order flux, FP64 exact arithmetic, 20 Newton steps",
            n=25, seed=0, bump=0.1, aoa=3.06, precision=0, mode="exact", first_order=True,
            ts_max=20, stop_ratio=1e30),
    1: dict(workload="config1: 70^3 Kuhn box, second-order flux, plain FP64, solve to 1e-8 drop",
            n=70, seed=1, bump=0.1, aoa=3.06, precision=0, mode="fast", first_order=False,
            ts_max=20, stop_ratio=1e8, ref_count=("box70_forces.json", 1e8)),
    2: dict(workload="config2: 70^3 Kuhn box, FP32 Jacobian/ILU(0)/SpTRSV, FP64 residual and GMRES, to 1e-8 drop",
            n=70, seed=1, bump=0.1, aoa=3.06, precision=1, mode="fast", first_order=False,
            ts_max=20, stop_ratio=1e8),
    4: dict(workload="config4: 120^3 Kuhn box (bump 0.12, AoA 4.5, held out of training), mixed precision + "
                     "spatial ILU(0) + learned FGMRES against plain FP64, to 1e-8 drop",
            n=120, seed=4, bump=0.12, aoa=4.5, precision=1, mode="fast", first_order=False,
            ts_max=20, stop_ratio=1e8, learned=True, ilu_order=1, ref_ts=1,
            ref_count=("box120_reference_count.json", 1e8)),
}
WEIGHTS = os.path.join(ROOT, "kfun3d_b200", "weights", "mpnn_box40.npy")
GOLDEN = os.path.join(ROOT, "tests", "golden")
MESHGEN = os.path.join(ROOT, "kfun3d_b200", "_lib", "kfun3d_meshgen")
DEFAULT_CONFIG = 4


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- algorithmic bytes
def alg_bytes(N, E, Fs, Ns, Nf, nnzb, prec, j=15):
    """Per-call algorithmic bytes of each kernel family (f64 = 8 B, u32 = 4 B;
    node arrays counted once per pass; w = 8 for FP64 blocks, 4 for FP32)."""
    w = 4 if prec else 8
    b = {}
    b["gradient"] = 56 * E + 128 * N
    b["edge_flux"] = 40 * E + 184 * N + 12 * Fs + 28 * Nf
    b["flux"] = b["gradient"] + b["edge_flux"]                       # 96E + 312N + 12Fs + 28Nf
    b["timestep"] = 40 * E + 40 * N + 28 * (Ns + Nf)
    b["fill"] = (296 * E + 168 * N if not prec else 168 * E + 104 * N) + 28 * (Ns + Nf)
    b["ilu"] = nnzb * (32 * w + 4) + 8 * (N + 1)
    b["sptrsv"] = nnzb * (16 * w + 4) + 8 * (N + 1) + 96 * N
    # Gram-Schmidt at Arnoldi index j: the j+1 basis vectors read once, the new
    # vector read and written once (the kernel keeps it on chip; classical MGS
    # would move (5(j+1)+3)*32N re-reading and re-writing it per projection)
    b["mgs"] = (j + 3) * 32 * N
    b["gmres_iter"] = b["flux"] + 296 * N + b["sptrsv"] + b["mgs"]
    return b


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpus):
        self.gpus = gpus
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", ",".join(str(g) for g in self.gpus), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception as e:   # no nvidia-smi: report no clock data
            log("clock sampler unavailable:", e)
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            t = [x.strip() for x in line.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                mx = max(mx, float(t[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if t[5 + k].lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- distributed plumbing
class Dist:
    def __init__(self, gpus):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            import datetime
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist
            self.backend = backend

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


def cuda_sync():
    try:
        import torch
        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except Exception:
        pass


# ---------------------------------------------------------------- the reference on the host cores
class CStdoutToStderr:
    """Routes C-level stdout (the reference prints METIS statistics) to stderr,
    so this script's stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_count(cfg):
    """The reference's own GMRES iteration count (and Newton steps) to the
    workload's drop, from a full run of oracle/_ref committed as a fixture
    (tests/golden/make_golden.py records the command and thread count), or
    None when the workload has none."""
    spec = cfg.get("ref_count")
    if not spec:
        return None
    path = os.path.join(GOLDEN, spec[0])
    if not os.path.exists(path):
        return None
    d = json.load(open(path))
    f0, its, steps = None, 0, 0
    for st in d["steps"]:
        fn = float(st["fnorm"])
        f0 = fn if f0 is None else f0
        its += int(st["gmres_its"])
        steps += 1
        if round(f0 / fn) >= spec[1]:
            break
    out = {"gmres_its": its, "newton_steps": steps, "threads": d.get("threads", 1),
           "fixture": f"tests/golden/{spec[0]}"}
    if "solve_seconds" in d and d.get("newton_steps") == steps:
        out["full_run_seconds"] = d["solve_seconds"]
        out["cpu"] = d.get("cpu")
    return out


def reference_sample(path, cfg, total_its, threads):
    """Time the reference (oracle/_ref) on a bounded sample of the solve: its
    first Newton steps (two, one at 120^3) on the same mesh and settings, at `threads` OpenMP
    threads.  Seconds to the 1e-8 drop are extrapolated by GMRES iterations:
    sample_time * total_its / sample_its (the per-iteration work of this solver
    is the same at every step)."""
    from oracle import ref
    m = ref.RefMesh(path, cfg["aoa"], threads)
    v = m.view
    q0 = v.q.copy()
    # ComputeFlux throughput (edges/s): a few calls
    t0 = time.perf_counter()
    nflux = 3
    for _ in range(nflux):
        m.flux(q0)
    t_flux = (time.perf_counter() - t0) / nflux
    t0 = time.perf_counter()
    hist = m.solve(ts_max=cfg.get("ref_ts", 2), stop_ratio=cfg["stop_ratio"])
    t_sample = time.perf_counter() - t0
    its = sum(h["gmres_its"] for h in hist)
    m.close()
    return dict(seconds=t_sample * total_its / max(its, 1), sample_seconds=t_sample, sample_its=its,
                flux_edges_per_s=v.nedges / t_flux)


def run_reference_arm(args, cfg):
    # Under torchrun only rank 0 times the reference; the other ranks have no work.
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libkfun3d_ref.so was not built"}))
        return
    path = mesh_path(cfg)
    threads = host_cores()
    rc = reference_count(cfg)
    if args.ref_total_its:
        total_its, its_src = args.ref_total_its, "given on the command line"
    elif rc:
        total_its = rc["gmres_its"]
        its_src = (f"the reference's own count at {rc['threads']} thread(s), full run in {rc['fixture']}")
    else:
        print(json.dumps({"impl": "reference", "unavailable": "no reference iteration count for this workload"}))
        return
    # Warm-up: one untimed ComputeFlux pass per requested warm-up step (page-in
    # of the mesh and OpenMP thread start); each timed step is a full sample.
    if args.warmup:
        with CStdoutToStderr():
            m = ref.RefMesh(path, cfg["aoa"], threads)
            for _ in range(args.warmup):
                m.flux(m.view.q.copy())
            m.close()
    vals = []
    t_all = time.perf_counter()
    with CStdoutToStderr():
        for _ in range(args.steps):
            vals.append(reference_sample(path, cfg, total_its, threads))
    wall = time.perf_counter() - t_all
    value = statistics.mean(v["seconds"] for v in vals)
    sample = (f"first {cfg.get('ref_ts', 2)} Newton step(s) ({vals[-1]['sample_its']} GMRES iterations, "
              f"{vals[-1]['sample_seconds']:.2f} s) of the workload at {threads} threads, extrapolated to "
              f"{total_its} GMRES iterations ({its_src})")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": cfg["workload"], "threads": threads},
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "reference",
                             "sample": sample, "flux_edges_per_s": vals[-1]["flux_edges_per_s"],
                             "reference_gmres_its": total_its, "sample_gmres_its": vals[-1]["sample_its"],
                             "reference_full_run": rc},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- the GPU arm
def mesh_path(cfg):
    """The workload's mesh file, written on first use by the stand-alone
    generator program (kfun3d_meshgen: host code only, so the reference arm
    never loads the CUDA library)."""
    d = os.environ.get("KFUN3D_MESH_DIR", os.path.join(tempfile.gettempdir(), "kfun3d_meshes"))
    os.makedirs(d, exist_ok=True)
    p = os.path.join(d, f"box{cfg['n']}_s{cfg['seed']}_b{cfg['bump']}.msh")
    if not os.path.exists(p):
        tmp = p + f".{os.getpid()}.tmp"
        if not os.path.exists(MESHGEN):
            raise SystemExit(f"{MESHGEN} missing: run `make -C kfun3d_b200/csrc`")
        subprocess.run([MESHGEN, tmp, str(cfg["n"]), repr(cfg["bump"]), str(cfg["seed"])], check=True)
        os.replace(tmp, p)
    return p


def configure(kf, cfg):
    kf.set_mode(cfg["mode"])
    kf.set_precision(cfg["precision"])
    kf.set_ilu_order(cfg.get("ilu_order", 0))
    kf.set_first_order(cfg["first_order"])
    kf.set_aoa(cfg["aoa"])
    kf.set_verbose(False)


def run_gpu_arm(args, cfg):
    dist = Dist(list(range(args.gpus)))
    import torch
    if torch.cuda.is_available():
        torch.cuda.set_device(dist.local)
        torch.zeros(1, device="cuda")   # the context exists before the set-up's timers start
    import kfun3d_b200 as kf
    configure(kf, cfg)
    path = mesh_path(cfg)
    m = kf.Mesh(path)
    v = m.view
    N, E = v.nnodes, v.nedges
    params = dict(ts_max=cfg["ts_max"], stop_ratio=cfg["stop_ratio"])
    net = None
    if cfg.get("learned"):
        from kfun3d_b200 import learned
        if not os.path.exists(WEIGHTS):
            raise SystemExit(f"trained network missing: {WEIGHTS} (python -m kfun3d_b200.train_mpnn)")
        net = learned.Network.load(WEIGHTS)

    def timed(reps):
        """Mean device seconds of `reps` solves of the workload's form from free stream."""
        if net is not None:
            return m.time_solve_flexible(net=net, reps=reps, **params)
        t, h = m.time_solve(reps=reps, **params)
        return t, h, None

    # warm-up (uploads the mesh, builds the device mirror)
    timed(args.warmup)
    cuda_sync()
    dist.barrier()
    cuda_sync()
    sampler = ClockSampler([dist.local]) if dist.rank == 0 else None
    if sampler:
        sampler.start()
    kf.reset_launch_count()
    t_wall = time.perf_counter()
    t_solve, hist, fstats = timed(args.steps)
    cuda_sync()
    launches = kf.launch_count()
    dist.barrier()
    cuda_sync()
    wall = time.perf_counter() - t_wall
    clocks = sampler.stop() if sampler else None
    value = dist.max(t_solve)
    gmres_its = sum(h["gmres_its"] for h in hist)
    drop = hist[-1]["fnorm"] / hist[0]["fnorm"] if hist else float("nan")

    # end to end through the C ABI, host buffers
    q0 = v.q.copy()
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        v.q[:] = q0
        t0 = time.perf_counter()
        if net is not None:
            m.solve_flexible(net=net, **params)
        else:
            m.solve(**params)
        e2e.append(time.perf_counter() - t0)
    v.q[:] = q0
    e2e_value = dist.max(statistics.mean(e2e))

    # the learned form against plain FP64 (the reference's method: FP64, ILU(0)
    # in the mesh's numbering), one solve each, and the ladder between them so
    # that each form's own gain shows: FP64 with ILU(0) in the spatial order
    # (the ordering's gain), FP32 preconditioner in the spatial order without
    # the network (the precision's gain), then the network (its gain); and
    # plain GMRES in mixed precision in the mesh's numbering
    comparison = None
    if net is not None:
        f_ours = [hist[-1][k] for k in ("lift", "drag", "momn")]

        def warm(fn):
            """One untimed solve of the form first (its CUDA graphs captured,
            as the headline's are in its warm-up), then the timed one."""
            fn()
            return fn()
        t_ilu, h_ilu, st_ilu = warm(lambda: m.time_solve_flexible(net=None, reps=1, **params))
        kf.set_precision(0)
        t_sp64, h_sp64 = warm(lambda: m.time_solve(reps=1, **params))
        kf.set_precision(cfg["precision"])
        kf.set_ilu_order(0)
        t_mesh, h_mesh = warm(lambda: m.time_solve(reps=1, **params))
        kf.set_precision(0)
        t_plain, h_plain = warm(lambda: m.time_solve(reps=1, **params))
        kf.set_precision(cfg["precision"])
        kf.set_ilu_order(cfg.get("ilu_order", 0))
        f_plain = [h_plain[-1][k] for k in ("lift", "drag", "momn")]
        its = lambda h: sum(x["gmres_its"] for x in h)   # noqa: E731
        comparison = {
            "plain_fp64_s": t_plain, "plain_fp64_gmres_its": its(h_plain),
            "plain_fp64_newton_steps": len(h_plain),
            "speedup_vs_plain_fp64": t_plain / value,
            "fp64_spatial_gmres_s": t_sp64, "fp64_spatial_gmres_its": its(h_sp64),
            "mixed_spatial_fgmres_no_network_s": t_ilu, "mixed_spatial_fgmres_no_network_its": st_ilu["gmres_its"],
            "mixed_mesh_order_gmres_s": t_mesh, "mixed_mesh_order_gmres_its": its(h_mesh),
            "gain_ordering": t_plain / t_sp64,
            "gain_precision": t_sp64 / t_ilu,
            "gain_network": t_ilu / value,
            "ilu_order": "spatial (slab sweeps)" if cfg.get("ilu_order", 0) else "mesh numbering",
            "learned_stats": fstats,
            "forces_rel_err_vs_fp64": max(abs(a - b) / abs(b) for a, b in zip(f_ours, f_plain)),
        }

    # per-kernel live timing (CUDA events on the solver's stream)
    peak, peak_kind = peaks()
    Fs, Ns, Nf = v.nfaces, v.ns, v.nf
    nnzb = N + 2 * E
    B = alg_bytes(N, E, Fs, Ns, Nf, nnzb, cfg["precision"])
    t = {}
    for name in ("flux", "gradient", "edge_flux", "timestep", "fill", "sptrsv", "mgs", "gmres_iter"):
        t[name] = m.time_kernel(name, 20 if name not in ("gmres_iter",) else 10)
    t["ilu"] = max(m.time_kernel("ilu", 3) - t["fill"], 1e-6)
    kernels = {k: {"ms": round(t[k], 5), "gbs": round(B[k] / (t[k] * 1e-3) / 1e9, 1),
                   "frac": round(B[k] / (t[k] * 1e-3) / 1e9 / peak, 4)} for k in t}
    # the plain form's Jacobian fill, ILU(0) and triangular solves (FP64 blocks,
    # the mesh's numbering); flux and time step are FP64 in every form
    kernels_fp64 = None
    if cfg["precision"] or cfg.get("ilu_order", 0):
        kf.set_precision(0)
        kf.set_ilu_order(0)
        B64 = alg_bytes(N, E, Fs, Ns, Nf, nnzb, 0)
        t64 = {k: m.time_kernel(k, 20) for k in ("fill", "sptrsv")}
        t64["ilu"] = max(m.time_kernel("ilu", 3) - t64["fill"], 1e-6)
        kf.set_precision(cfg["precision"])
        kf.set_ilu_order(cfg.get("ilu_order", 0))
        kernels_fp64 = {k: {"ms": round(t64[k], 5), "gbs": round(B64[k] / (t64[k] * 1e-3) / 1e9, 1),
                            "frac": round(B64[k] / (t64[k] * 1e-3) / 1e9 / peak, 4)} for k in t64}
        kernels_fp64["fill_edges_per_s"] = E / (t64["fill"] * 1e-3)
    share = {k: t[k] for k in ("flux", "sptrsv", "mgs")}
    dominant = max(share, key=share.get)
    traffic = None
    tp = os.path.join(ROOT, "profiles", f"traffic_config{args.config}.json")
    if os.path.exists(tp):
        # measured DRAM bytes per call, per kernel family and ILU(0) order
        key = dominant + ("@spatial" if cfg.get("ilu_order", 0) else "")
        traffic = json.load(open(tp)).get(key)
    achieved = B[dominant] / (t[dominant] * 1e-3) / 1e9
    roofline = {"kernel": dominant, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "peak_kind": peak_kind, "algorithmic_bytes": B[dominant]}

    # set-up (outside the timed region): the device mirror, its block pattern
    # built on the device, the spatial order's set, against the same pattern
    # built on the host threads (checked equal element for element)
    setup = None
    if dist.rank == 0:
        us = lambda k: round(m.query(k) / 1e6, 4)   # noqa: E731
        setup = {"mirror_s": us("setup_us"), "pattern_on_device_s": us("pattern_us"),
                 "spatial_order_s": us("spatial_setup_us")}
        setup["pattern_matches_host"] = m.query("pattern_matches_host") == 1
        setup["pattern_on_host_threads_s"] = us("host_pattern_us")
        setup["host_threads"] = min(32, os.cpu_count() or 1)   # the host build's thread count

    cpu = None
    if dist.rank == 0 and args.gpus == 1 and not args.no_cpu_baseline:
        from oracle import ref
        rc = reference_count(cfg)
        if ref.available() and rc:
            threads = host_cores()
            with CStdoutToStderr():
                s = reference_sample(path, cfg, rc["gmres_its"], threads)
            cpu = {"value": s["seconds"], "unit": "s", "cores": threads, "kind": "reference",
                   "sample": (f"reference (oracle/_ref) first {cfg.get('ref_ts', 2)} Newton step(s) of this workload: "
                              f"{s['sample_its']} GMRES iterations in {s['sample_seconds']:.2f} s at "
                              f"{threads} threads, extrapolated to the reference's own {rc['gmres_its']} GMRES "
                              f"iterations to the 1e-8 drop (full run at {rc['threads']} thread(s), "
                              f"{rc['fixture']}; FP64, ILU(0) in the mesh's numbering)"),
                   "reference_gmres_its": rc["gmres_its"], "gpu_gmres_its": gmres_its,
                   "flux_edges_per_s": s["flux_edges_per_s"]}
    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if cfg["precision"] == 0 else "f64/f32",
            "data": "synthetic (seeded Kuhn-box mesh generated on the box)",
            "config": {"workload": cfg["workload"], "nodes": N, "edges": E, "nnz_blocks": nnzb,
                       "newton_steps": len(hist), "gmres_its": gmres_its, "residual_drop": drop,
                       "mode": cfg["mode"], "precision": "fp64" if cfg["precision"] == 0 else "fp32-precond",
                       "parallelism": f"replicas x{args.gpus}",
                       "l2": "working set (matrix + vectors) larger than the 126 MB L2"},
            "e2e": {"value": e2e_value, "unit": "s", "h2d_bytes_per_step": 32 * N,
                    "d2h_bytes_per_step": 32 * N + 8 * N},
            "roofline": roofline,
            "kernels": kernels,
            "kernels_fp64": kernels_fp64,
            "flux_edges_per_s": E / (t["flux"] * 1e-3),
            "fill_edges_per_s": E / (t["fill"] * 1e-3),
            "gmres_iterations_per_s": gmres_its / value,
            "gpu_launches": int(launches),
            "comparison": comparison,
            "setup": setup,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "wall_s": wall,
        }
        print(json.dumps(line))
    m.close()
    dist.close()


def run_network_probe(args, cfg, kf, m):
    """--kernel mpnn_apply: one application of the shipped network on the
    workload's mesh (k_mlp_fwd), `reps` times; --kernel mpnn_train: pairs from
    one solve on the mesh, then `reps` Adam steps of the library's training
    loop (k_mlp_fwd, k_mlp_bwd, k_adam), batch 8."""
    from kfun3d_b200 import learned
    if args.kernel == "mpnn_apply":
        net = learned.Network.load(WEIGHTS)
        ms = m.time_learned_apply(net, args.reps)
        net.close()
        return {"kernel": args.kernel, "config": cfg["workload"], "ms": ms}
    import time
    x0, tgt, st = m.collect_pairs(stride=2, cap=16, ts_max=cfg["ts_max"], stop_ratio=cfg["stop_ratio"])
    g = learned.Graph(m)
    net = learned.Network(seed=0)
    data = [learned.Sample(m, g, x0, tgt, cfg["aoa"], cfg["bump"], st)]
    cuda_sync()
    t0 = time.perf_counter()
    losses = learned.train(net, data, args.reps, batch=8)
    cuda_sync()
    ms = (time.perf_counter() - t0) / args.reps * 1e3
    net.close()
    g.close()
    return {"kernel": args.kernel, "config": cfg["workload"], "ms": ms, "pairs": int(x0.shape[0]),
            "loss_first": losses[0], "loss_last": losses[-1]}


def run_setup_probe(cfg, kf, path):
    """--kernel setup: the set-up of the workload's mesh, host wall time per
    stage: the .msh load (reference-order GEOMETRY), the device mirror (block
    pattern, incidence lists and edge storage built on the device), the
    spatial ILU(0) order's set (built by the first entry point that runs in
    it), and the same block pattern built on the host threads for comparison.
    CUDA's own start-up is paid before the timers start."""
    import torch
    if torch.cuda.is_available():
        torch.zeros(1, device="cuda")
    t0 = time.perf_counter()
    m = kf.Mesh(path)
    t1 = time.perf_counter()
    m.query("setup_us")                  # builds the device mirror
    t2 = time.perf_counter()
    m.flux(m.view.q.copy())              # the first entry point builds the workload's ILU(0) order
    t3 = time.perf_counter()
    us = lambda k: m.query(k) / 1e6      # noqa: E731
    out = {"kernel": "setup", "config": cfg["workload"], "load_s": t1 - t0, "mirror_s": t2 - t1,
           "first_flux_s": t3 - t2, "mirror_in_library_s": us("setup_us"), "pattern_on_device_s": us("pattern_us"),
           "spatial_order_s": us("spatial_setup_us") if cfg.get("ilu_order", 0) else 0.0}
    out["pattern_matches_host"] = m.query("pattern_matches_host") == 1
    out["pattern_on_host_threads_s"] = us("host_pattern_us")
    out["lists_match_host"] = m.query("lists_match_host") == 1
    m.close()
    return out


def run_kernel_probe(args, cfg):
    """--kernel NAME: time one kernel family `reps` times on the workload's mesh
    and print {"kernel", "ms", "gbs"} -- the command the profiles use to
    capture a single kernel under ncu."""
    import kfun3d_b200 as kf
    configure(kf, cfg)
    path = mesh_path(cfg)
    if args.kernel == "setup":
        print(json.dumps(run_setup_probe(cfg, kf, path)))
        return
    m = kf.Mesh(path)
    if args.kernel in ("mpnn_apply", "mpnn_train"):
        print(json.dumps(run_network_probe(args, cfg, kf, m)))
        m.close()
        return
    v = m.view
    B = alg_bytes(v.nnodes, v.nedges, v.nfaces, v.ns, v.nf, v.nnodes + 2 * v.nedges, cfg["precision"])
    ms = m.time_kernel(args.kernel, args.reps)
    print(json.dumps({"kernel": args.kernel, "config": cfg["workload"], "ms": ms,
                      "gbs": B.get(args.kernel, 0) / (ms * 1e-3) / 1e9 if ms > 0 else None}))
    m.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=DEFAULT_CONFIG, choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-total-its", type=int, default=None,
                    help="GMRES iterations of the full solve used to extrapolate the reference sample "
                         "(default: the reference's own count from its full run, tests/golden/)")
    ap.add_argument("--kernel", default=None,
                    help="time one kernel family (flux, gradient, edge_flux, timestep, fill, ilu, sptrsv, mgs, "
                         "gmres_iter, mpnn_apply, mpnn_train) or the set-up (setup) instead of the solve")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--n", type=int, default=None,
                    help="with --kernel: mesh of n^3 nodes instead of the workload's (same seed and bump)")
    ap.add_argument("--precision", type=int, default=None, choices=[0, 1],
                    help="override the workload's preconditioner precision (with --kernel)")
    ap.add_argument("--ilu-order", type=int, default=None, choices=[0, 1],
                    help="override the workload's ILU(0) elimination order: 0 mesh numbering, 1 spatial (with --kernel)")
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.precision is not None:
        cfg["precision"] = args.precision
    if args.ilu_order is not None:
        cfg["ilu_order"] = args.ilu_order
    if args.n is not None and args.kernel:
        cfg["n"] = args.n
        cfg["workload"] += f" (kernel probe on the {args.n}^3 mesh)"
    if args.kernel:
        run_kernel_probe(args, cfg)
    elif args.impl == "reference":
        run_reference_arm(args, cfg)
    else:
        run_gpu_arm(args, cfg)


if __name__ == "__main__":
    main()
