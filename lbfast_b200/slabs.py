"""One box split into z slabs: the halo exchange of the reference's MPI layer
(mpi_module.f90:2203-3650, the 26-direction exchanges of hfields, phi, aux
fields and forces between the ranks of a Cartesian decomposition) for a split
along z of a box periodic in z.

Each slab is a handle (lbf_create_slab) on planes [z0, z1) of the box plus
HALO planes on each side.  Its step advances its own planes; between steps
the halo planes of the current time level are refilled from the
neighbouring slabs:

* ``SlabSet``: several slabs in one process (one GPU or several), exchanged
  by ``lbf_slabs_exchange`` (device-to-device and peer copies);
* ``RankSlab``: one slab per process, exchanged with ``torch.distributed``
  send/receive of the slab's halo regions (NCCL on GPUs) following
  ``halo_schedule``.

The reference exchanges four groups of fields in separate calls, some of
them overlapped with interior work (ASYNCMPI, integrator_module.f90:278-368);
here one exchange per step moves every field a step reads across a slab
face: the moments, u_old (one plane would do) and phi (three planes).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .capi import Params, Solver, check, load

HALO = 3  # halo planes on each side of a slab (lbf_create_slab)


def partition(nz: int, nslabs: int) -> list[tuple[int, int]]:
    """Contiguous z ranges of nearly equal length (the first nz % nslabs one
    plane longer), each at least HALO planes."""
    if nslabs < 1 or nz < nslabs * HALO:
        raise ValueError(f"{nz} planes cannot make {nslabs} slabs of at least {HALO} planes")
    base, extra = divmod(nz, nslabs)
    out, z = [], 0
    for i in range(nslabs):
        n = base + (1 if i < extra else 0)
        out.append((z, z + n))
        z += n
    return out


def neighbours(i: int, n: int) -> tuple[int, int]:
    """(slab below, slab above) of slab i in the periodic ring of n slabs."""
    return (i - 1) % n, (i + 1) % n


def halo_schedule(rank: int, nranks: int, nfields: int):
    """The messages of one exchange for `rank`: (kind, side, field, peer, tag)
    with kind "send" / "recv" and side 0 (low z) / 1 (high z).  Field f going
    up carries tag 2 f, going down 2 f + 1, so every send has exactly one
    matching receive; with one rank the slab is its own neighbour."""
    lo, hi = neighbours(rank, nranks)
    ops = []
    for f in range(nfields):
        ops.append(("send", 1, f, hi, 2 * f))      # my top planes -> the low halo of the slab above
        ops.append(("recv", 0, f, lo, 2 * f))      # my low halo <- the top planes of the slab below
        ops.append(("send", 0, f, lo, 2 * f + 1))  # my bottom planes -> the high halo of the slab below
        ops.append(("recv", 1, f, hi, 2 * f + 1))  # my high halo <- the bottom planes of the slab above
    return ops


def exchange_ranks(regions, schedule, group=None) -> None:
    """Run one exchange: regions[(kind, side, field)] is the tensor (CUDA for
    NCCL, CPU for gloo) a message is sent from or received into.  Messages
    to oneself (one rank) are plain copies."""
    import torch.distributed as dist
    me = dist.get_rank(group) if dist.is_initialized() else 0
    reqs = []
    local = {}
    for kind, side, f, peer, tag in schedule:
        t = regions[(kind, side, f)]
        if peer == me:
            local.setdefault(tag, {})[kind] = t
        elif kind == "send":
            reqs.append(dist.isend(t, peer, group=group, tag=tag))
        else:
            reqs.append(dist.irecv(t, peer, group=group, tag=tag))
    for pair in local.values():
        pair["recv"].copy_(pair["send"])
    for r in reqs:
        r.wait()


class SlabSolver(Solver):
    """A handle on planes [z0, z1) of the box `params` (periodic in z) with
    HALO halo planes on each side; arrays are those of the slab's box
    (z1 - z0 + 2 HALO planes)."""

    def __init__(self, params: Params, z0: int, z1: int):
        self.lib = load()
        self.global_params = params
        self.params = Params(**{**params.__dict__, "lz": z1 - z0 + 2 * HALO, "pbc_z": 0})
        self.z0, self.z1 = z0, z1
        self.h = C.c_void_p()
        check(self.lib.lbf_create_slab(C.byref(params.to_c()), int(z0), int(z1), C.byref(self.h)))
        self.shape = self.params.shape
        n = C.c_int()
        check(self.lib.lbf_slab_nregions(self.h, C.byref(n)))
        self.nregions = n.value

    def region(self, side: int, recv: int, field: int) -> tuple[int, int]:
        """(device address, bytes) of a halo region of the current time level."""
        p, b = C.c_void_p(), C.c_size_t()
        check(self.lib.lbf_slab_region(self.h, int(side), int(recv), int(field), C.byref(p), C.byref(b)))
        return p.value, b.value


def slab_of(a: np.ndarray, z0: int, z1: int, axis: int = -3) -> np.ndarray:
    """Planes z0 - HALO .. z1 + HALO - 1 of a box field periodic in z."""
    nz = a.shape[axis]
    idx = np.arange(z0 - HALO, z1 + HALO) % nz
    return np.take(a, idx, axis=axis)


class SlabSet:
    """The box `params` as len(bounds) z slabs in this process, each on the
    device current when it is created (or devices[i])."""

    def __init__(self, params: Params, nslabs: int, devices=None):
        self.params = params
        self.bounds = partition(params.lz, nslabs)
        self.slabs = []
        for i, (z0, z1) in enumerate(self.bounds):
            if devices is not None:
                import torch
                torch.cuda.set_device(devices[i])
            self.slabs.append(SlabSolver(params, z0, z1))
        self._arr = (C.c_void_p * nslabs)(*[s.h.value for s in self.slabs])
        self.primed = False

    def close(self) -> None:
        for s in self.slabs:
            s.close()

    def set_isfluid(self, isf: np.ndarray) -> None:
        for s, (z0, z1) in zip(self.slabs, self.bounds):
            s.set_isfluid(slab_of(isf, z0, z1))

    def set_fields(self, mom10: np.ndarray, phi: np.ndarray | None = None) -> None:
        for s, (z0, z1) in zip(self.slabs, self.bounds):
            s.set_fields(slab_of(mom10, z0, z1), None if phi is None else slab_of(phi, z0, z1))
        self.primed = False

    def exchange(self) -> None:
        check(load().lbf_slabs_exchange(self._arr, len(self.slabs)))

    def step(self, n: int = 1, overlap: bool = True) -> None:
        """n steps.  overlap: lbf_slabs_step, each step's halo copies running
        beside the planes that do not read them; else one lbf_step per slab
        and a full exchange after it."""
        if overlap:
            check(load().lbf_slabs_step(self._arr, len(self.slabs), int(n)))
            self.primed = True
            return
        if not self.primed:
            # the pre-loop wetting runs in each slab's own planes; the halos
            # then take the neighbours' wetted planes
            for s in self.slabs:
                s.step(0)
            self.exchange()
            self.primed = True
        for _ in range(n):
            for s in self.slabs:
                s.step(1)
            self.exchange()

    def get_fields(self, dtype=np.float64):
        """The box's moments, phi and u_old assembled from the slabs' own planes."""
        parts = [s.get_fields(dtype) for s in self.slabs]
        cut = slice(HALO, -HALO)
        m = np.concatenate([p[0][:, cut] for p in parts], axis=1)
        ph = None if parts[0][1] is None else np.concatenate([p[1][cut] for p in parts], axis=0)
        u = np.concatenate([p[2][:, cut] for p in parts], axis=1)
        return m, ph, u


class _DeviceBytes:
    """A zero-copy view of device memory for torch.as_tensor."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


class RankSlab:
    """This process's slab of the box `params` over the ranks of the default
    process group (one slab per rank, rank r on planes partition(lz,
    world)[r]), exchanged with torch.distributed (NCCL on GPUs)."""

    def __init__(self, params: Params, rank: int, world: int):
        self.rank, self.world = rank, world
        self.z0, self.z1 = partition(params.lz, world)[rank]
        self.solver = SlabSolver(params, self.z0, self.z1)
        self.schedule = halo_schedule(rank, world, self.solver.nregions)
        self.primed = False

    def _regions(self):
        import torch
        regions = {}
        for kind, side, f, _, _ in self.schedule:
            ptr, nb = self.solver.region(side, 1 if kind == "recv" else 0, f)
            regions[(kind, side, f)] = torch.as_tensor(_DeviceBytes(ptr, nb), device="cuda")
        return regions

    def exchange(self) -> None:
        self.solver.sync()
        exchange_ranks(self._regions(), self.schedule)

    def step(self, n: int = 1) -> None:
        if not self.primed:
            self.solver.step(0)
            self.exchange()
            self.primed = True
        for _ in range(n):
            self.solver.step(1)
            self.exchange()


__all__ = ["HALO", "partition", "neighbours", "halo_schedule", "exchange_ranks", "SlabSolver", "SlabSet",
           "RankSlab", "slab_of"]
