"""Rank plumbing of the z-slab decomposition (lbfast_b200/slabs.py) on CPU:
the partition of the box, the message schedule of one halo exchange, and the
exchange itself run by two gloo ranks on CPU tensors standing in
for each slab's fields -- after it every rank's halo planes hold its
neighbours' planes of the global box (periodic in z)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lbfast_b200 import slabs

NF, NZ, NY, NX = 4, 13, 5, 6  # fields, planes, rows, columns of the test box


def test_partition_and_schedule():
    assert slabs.partition(13, 2) == [(0, 7), (7, 13)]
    assert slabs.partition(9, 3) == [(0, 3), (3, 6), (6, 9)]
    with pytest.raises(ValueError):
        slabs.partition(8, 3)  # a slab needs HALO planes
    for n in (1, 2, 3, 5):
        sent = {}
        recv = {}
        for r in range(n):
            for kind, side, f, peer, tag in slabs.halo_schedule(r, n, NF):
                (sent if kind == "send" else recv).setdefault((r, peer, tag), []).append((side, f))
        # every message is received by its peer with the opposite side
        assert sum(map(len, sent.values())) == sum(map(len, recv.values())) == n * 2 * NF
        for (r, peer, tag), items in sent.items():
            assert recv[(peer, r, tag)] == [(1 - s, f) for s, f in items]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _global():
    return np.arange(NF * NZ * NY * NX, dtype=np.float32).reshape(NF, NZ, NY, NX)


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    z0, z1 = slabs.partition(NZ, world)[rank]
    g = _global()
    local = slabs.slab_of(g, z0, z1, axis=1).copy()
    H = slabs.HALO
    local[:, :H] = -1.0   # halos start empty
    local[:, -H:] = -1.0
    t = torch.from_numpy(local)
    n = z1 - z0
    regions = {}
    for kind, side, f, _, _ in slabs.halo_schedule(rank, world, NF):
        if kind == "send":
            first = H if side == 0 else n
        else:
            first = 0 if side == 0 else H + n
        regions[(kind, side, f)] = t[f, first:first + H]
    slabs.exchange_ranks(regions, slabs.halo_schedule(rank, world, NF))
    out[rank] = bool(np.array_equal(t.numpy(), slabs.slab_of(g, z0, z1, axis=1)))
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_halo_exchange_over_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
        assert p.exitcode == 0
    assert all(out[r] for r in range(world)), dict(out)


def test_single_rank_exchange_is_a_periodic_copy():
    """One slab is its own neighbour: the exchange copies its own top planes
    into its low halo and its bottom planes into its high halo."""
    import torch
    g = _global()
    local = slabs.slab_of(g, 0, NZ, axis=1).copy()
    H = slabs.HALO
    local[:, :H] = -1.0
    local[:, -H:] = -1.0
    t = torch.from_numpy(local)
    regions = {}
    for kind, side, f, _, _ in slabs.halo_schedule(0, 1, NF):
        first = (H if side == 0 else NZ) if kind == "send" else (0 if side == 0 else H + NZ)
        regions[(kind, side, f)] = t[f, first:first + H]
    slabs.exchange_ranks(regions, slabs.halo_schedule(0, 1, NF))
    assert np.array_equal(t.numpy(), slabs.slab_of(g, 0, NZ, axis=1))
