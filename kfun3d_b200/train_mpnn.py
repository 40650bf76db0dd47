"""Train the learned right preconditioner on the GPU.

    python -m kfun3d_b200.train_mpnn --meshes 128 --n 40 --steps 3000 \
        --out kfun3d_b200/weights/mpnn_box40.npy

Training set: seeded Kuhn-box meshes of n^3 nodes, bump height U(0.05, 0.15)
and angle of attack U(0, 6) degrees, each solved from free stream by the
ILU(0)-FGMRES solve that writes (residual, correction) pairs on the device
(ILU(0) in the mesh's numbering, or with --ilu-order 1 in the spatial order).
Network and optimiser: the library's BF16 tensor-core forward/backward and
FP32 Adam (lr 1e-3, batch 8 pairs).  Afterwards the network is compared with
the same FGMRES without it on a held-out mesh (bump 0.12, 4.5 degrees) and a
JSON report is written beside the weights.
"""
import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import api as kf
from . import learned


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--meshes", type=int, default=128)
    ap.add_argument("--n", type=int, default=40, help="nodes per box edge of the training meshes")
    ap.add_argument("--stride", type=int, default=2,
                    help="pairs from every stride-th FGMRES iterate (negative: basis vectors)")
    ap.add_argument("--cap", type=int, default=200, help="at most this many pairs per mesh")
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--batch-by-mesh", action="store_true",
                    help="each batch is --batch different meshes, one pair from each")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--eval-n", type=int, default=40, help="held-out mesh size (0: no evaluation)")
    ap.add_argument("--precision", type=int, default=1, help="preconditioner precision of the evaluation")
    ap.add_argument("--ilu-order", type=int, default=0, choices=[0, 1],
                    help="ILU(0) elimination order of the pair solves and the evaluation: 0 the mesh's "
                         "numbering (the shipped network), 1 spatial")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "weights", "mpnn_box40.npy"))
    a = ap.parse_args(argv)

    kf.set_mode("fast")
    kf.set_precision(0)
    kf.set_ilu_order(a.ilu_order)
    log = lambda s: print(s, flush=True)   # noqa: E731
    args = dict(vars(a))
    # the weights' path as the package sees it (never a scratch folder of the run)
    args["out"] = os.path.join("kfun3d_b200", "weights", os.path.basename(a.out))
    rep = dict(args=args)
    with tempfile.TemporaryDirectory() as work:
        t0 = time.time()
        data = learned.training_set(work, n_meshes=a.meshes, n=a.n, seed=a.seed, stride=a.stride, cap=a.cap,
                                    log=log)
        rep["pairs"] = sum(len(s) for s in data)
        rep["pairs_seconds"] = time.time() - t0
        rep["zero_loss"] = learned.zero_loss(data)
        log(f"{rep['pairs']} pairs in {rep['pairs_seconds']:.1f} s; zero-correction loss {rep['zero_loss']:.4e}")
        net = learned.Network(seed=a.seed + 1)
        t0 = time.time()
        losses = learned.train(net, data, a.steps, batch=a.batch, lr=a.lr, seed=a.seed, log=log, log_every=250,
                               by_mesh=a.batch_by_mesh)
        rep["train_seconds"] = time.time() - t0
        rep["final_loss"] = float(np.mean(losses[-100:]))
        rep["loss_curve"] = [float(np.mean(losses[i:i + 100])) for i in range(0, len(losses), 100)]
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        net.save(a.out)
        del data
        if a.eval_n > 0:
            kf.set_precision(a.precision)
            kf.set_aoa(4.5)
            path = os.path.join(work, "heldout.msh")
            kf.generate_mesh(path, a.eval_n, bump_height=0.12, seed=12345)
            m = kf.Mesh(path)
            q0 = m.view.q.copy()
            ev = {}
            for name, nt in (("ilu_fgmres", None), ("learned_fgmres", net)):
                m.view.q[:] = q0
                t, h, st = m.time_solve_flexible(net=nt, ts_max=20, stop_ratio=1e8)
                ev[name] = dict(seconds=t, its=[s["gmres_its"] for s in h], stats=st,
                                forces=[h[-1]["lift"], h[-1]["drag"], h[-1]["momn"]])
                log(f"{name}: {t:.4f} s, {st['gmres_its']} its, {st}")
            rep["heldout"] = ev
    with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
        json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
