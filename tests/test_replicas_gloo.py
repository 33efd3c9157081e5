"""The N-GPU path of bench.py: independent replicas, max-over-ranks timing.

Runs 2 gloo ranks on the CPU; each rank advances its own oracle replica
(the CUDA step cannot run here) and the max-over-ranks reduction and the
aggregate rate are checked.
"""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import time
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from lag2d_b200 import workload
    from lag2d_b200.replicas import aggregate_rate, barrier, max_over_ranks
    from oracle.oracle import Oracle
    m, c = workload("tgv16")
    o = Oracle(m, c)
    g, a, u = o.init()
    x = m.coord.copy()
    us = np.zeros_like(x)
    barrier()
    t0 = time.perf_counter()
    o.run(u, x, m.coord, g, a, us, 1, 1 + rank, c.dtfix, 0.0)
    t = time.perf_counter() - t0
    tmax = max_over_ranks(t)
    rate = aggregate_rate(m.ncell * 24 * c.nstag, tmax, world)
    out[rank] = (t, tmax, rate, float(np.abs(u[:m.ncell, 1:3, :]).sum()))
    barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    world = 2
    port = _free_port()
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    t0, tmax0, rate0, s0 = out[0]
    t1, tmax1, rate1, s1 = out[1]
    assert tmax0 == tmax1 == max(t0, t1)
    assert rate0 == rate1
    assert s0 != s1  # the replicas are independent (rank 1 ran one more step)
