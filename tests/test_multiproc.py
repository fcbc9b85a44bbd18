"""Multi-rank host logic on CPU (gloo, world size 2): the tile partition
covers every tile once with balanced work, and the one exchange of the LOO
search (an all-reduce of per-rank partial log likelihoods) reproduces the
single-process oracle sum and argmax."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mgpukde_tiled_b200 import shard


def test_tile_plan_and_assignment():
    tiles = shard.tile_plan(10_000, 10_000, 4096)
    assert len(tiles) == 9
    assert sum(nr * nc for (_, _, nr, nc) in tiles) == 10_000 * 10_000
    parts = shard.assign_tiles(tiles, 4)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(tiles)))
    assert shard.assign_tiles(tiles, 4) == parts  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import torch.distributed as dist

    import oracle_py as o
    from mgpukde_tiled_b200 import shard as sh
    from mgpukde_tiled_b200 import synth
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    x, y = synth.mixture_points(800, 3, 100.0, 4.0, 10.0, seed=5)
    hs = synth.log_h_grid(1.0, 10.0, 6)
    a, b = sh.query_range(len(x), rank, world)
    part = []
    for h in hs:
        _, loo, _ = o.loo_loglik(x, y, None, None, float(h))
        v = np.maximum(loo[a:b], float(np.float32(1e-14)))
        part.append(float(np.sum(np.log(v))))
    tot, am = sh.allreduce_loglik(part)
    # tile assignment is the same on every rank
    parts = sh.assign_tiles(sh.tile_plan(300, 500, 128), world)
    q.put((rank, tot.tolist(), am, parts))
    dist.destroy_process_group()


def test_two_rank_loo_allreduce():
    import oracle_py as o
    from mgpukde_tiled_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    x, y = synth.mixture_points(800, 3, 100.0, 4.0, 10.0, seed=5)
    hs = synth.log_h_grid(1.0, 10.0, 6)
    ref = np.array([o.loo_loglik(x, y, None, None, float(h))[0] for h in hs])
    (r0, t0, a0, p0), (r1, t1, a1, p1) = sorted(res)
    np.testing.assert_allclose(t0, ref, rtol=1e-12)
    assert t0 == t1 and a0 == a1 == int(np.argmax(ref))
    assert p0 == p1
