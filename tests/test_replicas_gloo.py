"""Replica plumbing of the N-GPU bench (q2d_b200/replicas.py) with 2 gloo ranks on CPU: each rank
builds its own batch from a rank seed (different cases per rank), the whole-job throughput uses
the sum of cells over ranks and the slowest rank's time, and no data crosses ranks otherwise."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from q2d_b200 import cases, replicas
    import torch.distributed as dist
    replicas.init("gloo", timeout_s=60)
    r, w, _ = replicas.dist_env()
    batch = cases.area_nozzle_batch(n=3, seed=replicas.rank_seed(cases.BASE_SEED + 3, r),
                                    nx_range=(16, 40), ny_range=(4, 8))
    cells = sum(c.cells for c in batch)
    replicas.barrier()
    seconds = 0.5 + r                       # stand-in for a device time
    smax = replicas.max_over_ranks(seconds)
    call = replicas.sum_over_ranks(cells)
    out[r] = (cells, smax, call, replicas.throughput(call, 10, smax), float(batch[0].blocks[0].prim[0, 0, 3]))
    dist.destroy_process_group()


def test_two_rank_replicas():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    c0, s0, a0, v0, p0 = out[0]
    c1, s1, a1, v1, p1 = out[1]
    assert s0 == s1 == 1.5                       # slowest rank
    assert a0 == a1 == c0 + c1                   # whole-job cells
    assert np.isclose(v0, (c0 + c1) * 10 / 1.5) and v0 == v1
    assert p0 != p1                              # independent batches per rank
