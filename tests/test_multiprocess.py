"""The N > 1 path of bench.py on CPU: two gloo ranks, replicas of one mesh each.

bench.py runs one independent solve per rank (replicas: no collective on the
data path) and reduces the per-rank time with a max over ranks.  Here two gloo
processes run the host side of that path -- the native loader on the rank's
mesh and the oracle solve standing in for the device solve -- and check that
the max-over-ranks reduction and the barrier behave, and that the replicas
agree with each other.  A second pair of ranks takes one additive Schwarz
subdomain each, as a multi-GPU run would, and checks that the ranks compute
the same partition and together own every node exactly once.
"""
import os
import socket
import tempfile

import pytest


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def worker(rank, world, port, mesh, out):
    import numpy as np
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import kfun3d_b200 as kf
    from oracle import port as orc
    d = bench.Dist([0])
    assert d.world == world and d.rank == rank
    m = kf.Mesh(mesh)
    q = m.view.q.copy()
    hist = orc.solve(m.g, 3.0, q, ts_max=3)
    local = 1.0 + rank            # a per-rank "time"
    d.barrier()
    mx = d.max(local)
    np.save(os.path.join(out, f"r{rank}.npy"), np.array([mx, hist[-1]["fnorm"]] + list(q[:8])))
    d.close()


def test_two_rank_replicas(box_mesh):
    import torch.multiprocessing as mp
    mesh = box_mesh(6, seed=2)
    port = free_port()
    with tempfile.TemporaryDirectory() as out:
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=worker, args=(r, 2, port, mesh, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        import numpy as np
        a, b = np.load(os.path.join(out, "r0.npy")), np.load(os.path.join(out, "r1.npy"))
        assert a[0] == 2.0 and b[0] == 2.0          # max over ranks seen by both
        assert np.array_equal(a[1:], b[1:])          # identical replicas


def schwarz_worker(rank, world, port, mesh, out):
    """Rank `rank` takes subdomain `rank` of kfun3d_schwarz_partition(world):
    every rank computes the partition on its own, and a gloo all-gather
    checks that they computed the same one and that the owned nodes cover
    the mesh exactly once."""
    import numpy as np
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist
    import kfun3d_b200 as kf
    dist.init_process_group("gloo", rank=rank, world_size=world)
    m = kf.Mesh(mesh)
    part = m.schwarz_partition(world)
    owned = torch.from_numpy((part == rank).astype(np.int64))
    parts = [torch.zeros_like(owned) for _ in range(world)]
    dist.all_gather(parts, owned)
    full = torch.from_numpy(part)
    fulls = [torch.zeros_like(full) for _ in range(world)]
    dist.all_gather(fulls, full)
    cover = torch.stack(parts).sum(0)
    same = all(torch.equal(f, fulls[0]) for f in fulls)
    np.save(os.path.join(out, f"s{rank}.npy"),
            np.array([int(same), int(cover.min()), int(cover.max()), int(owned.sum())]))
    dist.destroy_process_group()


def test_two_rank_schwarz_subdomains(box_mesh):
    import torch.multiprocessing as mp
    mesh = box_mesh(7, seed=5)
    port = free_port()
    with tempfile.TemporaryDirectory() as out:
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=schwarz_worker, args=(r, 2, port, mesh, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        import numpy as np
        a, b = np.load(os.path.join(out, "s0.npy")), np.load(os.path.join(out, "s1.npy"))
        assert a[0] == 1 and b[0] == 1               # the same partition on both ranks
        assert a[1] == 1 and a[2] == 1               # every node owned by exactly one rank
        assert a[3] + b[3] == 7 ** 3 and abs(int(a[3]) - int(b[3])) <= 1
