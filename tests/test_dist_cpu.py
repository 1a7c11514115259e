"""The replica path of bench.py on CPU: two gloo ranks (world size 2) join,
barrier, and agree on the max over ranks that every multi-GPU time uses; each
rank builds its own seeded problem (weak scaling, no collective on the path)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, l = bench.dist_setup(None)
    d = bench.Dist(w, r, l, use_gpu=False)
    d.barrier()
    m = d.max(1.5 + r)
    d.barrier()
    d.close()
    out.put((r, m))


def test_two_gloo_ranks_take_the_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 2.5, 1: 2.5}


def test_ranks_get_independent_problems():
    sys.path.insert(0, os.path.join(ROOT, "compressedsensingipm.jl_b200"))
    import csipm.problems as P
    a = P.make_spec("3d", dims=(16, 16, 16), seed=0)
    b = P.make_spec("3d", dims=(16, 16, 16), seed=1)
    assert not (a.beta_true == b.beta_true).all()
    sa, _ = P.serving_spec(1000)
    sb, _ = P.serving_spec(1000 + 100000)
    assert sa.seed != sb.seed
