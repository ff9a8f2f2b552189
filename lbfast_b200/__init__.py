"""lbfast_b200 -- B200-native (sm_100a) implementation of the LBFAST time step.

The numerics run in the CUDA library built in-tree (lbfast_b200/_lib); this
package binds its C ABI (include/lbfast_gpu.h) and adds the host-side pieces
of the LBFAST driver (namelist reader, set-up, output).
"""
from .capi import (LbfError, Params, Server, Solver, ic_droplet, ic_lamb, ic_taylor_green, load, mark_isfluid,  # noqa: F401
                   read_restart_raw, seed_solid_phi, write_raw_xdmf, write_restart_raw, write_vtk)

__all__ = ["LbfError", "Params", "Server", "Solver", "ic_droplet", "ic_lamb", "ic_taylor_green", "load", "mark_isfluid",
           "read_restart_raw", "seed_solid_phi", "write_raw_xdmf", "write_restart_raw", "write_vtk"]
