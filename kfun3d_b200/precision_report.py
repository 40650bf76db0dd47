"""Errors of the mixed-precision and learned forms against the FP64 form.

    python -m kfun3d_b200.precision_report --n 70 --seed 1 --bump 0.1 --aoa 3.06
    python -m kfun3d_b200.precision_report --n 120 --seed 4 --bump 0.12 --aoa 4.5 --learned

Solves the seeded Kuhn-box mesh to a 1e-8 residual drop (at most 20 Newton
steps, fast mode) with the plain FP64 solver -- the oracle of the other forms
-- and with the FP32 preconditioner (FP32 Jacobian blocks, ILU(0) factors and
triangular solves; FP64 residual, norms, CFL update, Gram-Schmidt and Givens),
plain GMRES and FGMRES, and with the learned FGMRES when --learned; then the
FP32 forms again with ILU(0) in the spatial elimination order.  Prints
one JSON object: per form the Newton steps, GMRES iterations, device seconds,
the max-norm relative error of the converged state and the relative error of
each wall-force component against FP64.
"""
import argparse
import json
import os
import tempfile

import numpy as np

from . import api as kf


def run(n, seed, bump, aoa, learned_weights=None, ts_max=20, stop_ratio=1e8):
    kf.set_mode("fast")
    kf.set_aoa(aoa)
    path = os.path.join(tempfile.gettempdir(), f"kfun3d_prec_{n}_{seed}_{bump}.msh")
    if not os.path.exists(path):
        kf.generate_mesh(path, n, bump_height=bump, seed=seed)
    m = kf.Mesh(path)
    q0 = m.view.q.copy()
    P = dict(ts_max=ts_max, stop_ratio=stop_ratio)
    out = {"mesh": dict(n=n, seed=seed, bump=bump, aoa=aoa, nodes=m.view.nnodes, edges=m.view.nedges)}

    def finish(name, t, h, st=None):
        q = m.view.q.copy()
        f = np.array([h[-1]["lift"], h[-1]["drag"], h[-1]["momn"]])
        out[name] = dict(seconds=t, newton_steps=len(h), gmres_its=sum(s["gmres_its"] for s in h),
                         drop=h[0]["fnorm"] / h[-1]["fnorm"], forces=f.tolist(), stats=st)
        m.view.q[:] = q0
        return q, f

    forms = []
    kf.set_precision(0)
    t, h = m.time_solve(**P)
    m.solve(**P)          # the converged state into q (time_solve leaves q untouched)
    q64, f64 = finish("fp64", t, h)
    kf.set_precision(1)
    t, h = m.time_solve(**P)
    m.solve(**P)
    forms.append(("mixed_gmres",) + finish("mixed_gmres", t, h))
    t, h, st = m.time_solve_flexible(**P)
    m.solve_flexible(**P)
    forms.append(("mixed_ilu_fgmres",) + finish("mixed_ilu_fgmres", t, h, st))
    net = None
    if learned_weights:
        from . import learned
        net = learned.Network.load(learned_weights)
        t, h, st = m.time_solve_flexible(net=net, **P)
        m.solve_flexible(net=net, **P)
        forms.append(("mixed_learned_fgmres",) + finish("mixed_learned_fgmres", t, h, st))
    # ILU(0) in the spatial elimination order
    kf.set_ilu_order(1)
    t, h = m.time_solve(**P)
    m.solve(**P)
    forms.append(("mixed_spatial_gmres",) + finish("mixed_spatial_gmres", t, h))
    if net is not None:
        t, h, st = m.time_solve_flexible(net=net, **P)
        m.solve_flexible(net=net, **P)
        forms.append(("mixed_spatial_learned_fgmres",) + finish("mixed_spatial_learned_fgmres", t, h, st))
    kf.set_ilu_order(0)
    for name, q, f in forms:
        out[name]["state_rel_err"] = float(np.max(np.abs(q - q64)) / np.max(np.abs(q64)))
        out[name]["forces_rel_err"] = (np.abs(f - f64) / np.abs(f64)).tolist()
    kf.set_precision(0)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n", type=int, default=70)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--bump", type=float, default=0.1)
    ap.add_argument("--aoa", type=float, default=3.06)
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(__file__), "weights", "mpnn_box40.npy"))
    a = ap.parse_args(argv)
    print(json.dumps(run(a.n, a.seed, a.bump, a.aoa, a.weights if a.learned else None)))


if __name__ == "__main__":
    main()
