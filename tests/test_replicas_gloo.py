"""Multi-rank plumbing of the replica runs (bench.py under torchrun), on CPU
with the gloo backend and two ranks: the timed region's barrier, the maximum
over ranks and the weak-scaling aggregate."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from lbfast_b200 import replicas
    r, local, w = replicas.init_from_env(backend="gloo", timeout_s=60)
    replicas.barrier(w)
    ms = 10.0 + 5.0 * r  # rank 1 is the slowest
    mx = replicas.allmax(ms, w)
    out[r] = (mx, replicas.weak_scaling_value(1000, 20, mx, w))
    replicas.shutdown(w)


@pytest.mark.timeout(120)
def test_two_rank_max_and_weak_scaling():
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    assert out[0] == out[1]
    mx, val = out[0]
    assert mx == 15.0
    assert abs(val - 2 * 1000 * 20 / 15e-3 / 1e6) < 1e-12


