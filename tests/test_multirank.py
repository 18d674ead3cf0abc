"""The multi-rank host logic of bench.py on CPU: two gloo ranks read their
rank from the environment, build disjoint seeded mesh sets (weak scaling: no
data-path collective), and agree on the job time as the maximum over ranks.
The same code runs under torchrun with NCCL on GPUs."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    from blitzremesher_b200 import synthetic as syn

    r, w, local = bench.dist_env()
    dist.init_process_group("gloo", rank=r, world_size=w, timeout=datetime.timedelta(seconds=60))
    meshes = syn.batched_set(3, seed=2 + 1000 * r, lo=2000, hi=4000)
    bench._barrier(w)
    t = bench._max_over_ranks(float(10 + r), w, torch.device("cpu"))
    out.put((r, w, local, t, [int(m.face_count) for m in meshes], float(meshes[0].positions[0, 0])))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_weak_scaling():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, t0, f0, x0), (r1, w1, l1, t1, f1, x1) = res
    assert (r0, r1) == (0, 1) and w0 == w1 == 2 and (l0, l1) == (0, 1)
    assert t0 == t1 == 11.0  # the max over ranks, the same on both
    assert x0 != x1  # each rank audits its own seeded set
