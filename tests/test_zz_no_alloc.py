"""lbf_reduce_noalloc: the reduction for callers that cannot let the library
allocate device memory (a Fortran integrator whose device arrays belong to
OpenACC data regions, an application that hands out all device memory from
its own pool, a solver held to a fixed device-memory budget).  Its fields are caller-owned device arrays
and its scratch is a static device array, so this test hands it device
tensors holding the state of a solver and checks the sums against the
library's allocating entry point, lbf_reduce, on the same state -- twice in a
row, with the state advanced in between, so that the second call cannot pass
on what the first call left in the shared scratch.

Kept in a file that pytest collects last: a failure here leaves every other
test already run.
"""
import ctypes as C

import numpy as np
import pytest

from cases import make_case
from lbfast_b200 import capi
from lbfast_b200.capi import Solver

pytestmark = pytest.mark.gpu


def _noalloc(lib, m_dev, phi_dev, isf_dev, shape):
    lz, ly, lx = shape
    out = np.zeros(5, dtype=np.float64)
    rc = lib.lbf_reduce_noalloc(C.c_void_p(m_dev.data_ptr()),
                                C.c_void_p(phi_dev.data_ptr()) if phi_dev is not None else None,
                                C.c_void_p(isf_dev.data_ptr()) if isf_dev is not None else None,
                                lx, ly, lz, out.ctypes.data_as(C.POINTER(C.c_double)))
    return rc, out


def _bind(lib):
    lib.lbf_reduce_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(C.c_double)]
    lib.lbf_reduce_noalloc.restype = C.c_int


def test_noalloc_reduce_matches_allocating_reduce_twice():
    import torch
    lib = capi.load()
    _bind(lib)
    p, isf, m, phi = make_case("obs_q27ho_2c_dr", "f32")
    s = Solver(p)
    s.set_isfluid(isf)
    s.set_fields(m, phi)
    isf_dev = torch.from_numpy(np.ascontiguousarray(isf, dtype=np.int8)).cuda()
    for call in range(2):
        s.step(5 + 3 * call)
        s.sync()
        ref = s.reduce()
        mg, pg, _ = s.get_fields(dtype=np.float32)
        m_dev = torch.from_numpy(np.ascontiguousarray(mg)).cuda()
        phi_dev = torch.from_numpy(np.ascontiguousarray(pg)).cuda()
        torch.cuda.synchronize()
        rc, out = _noalloc(lib, m_dev, phi_dev, isf_dev, p.shape)
        assert rc == capi.LBF_OK, capi.last_error()
        # same float32 values summed in FP64 in a different order
        scale = np.array([np.abs(pg[np.abs(isf) == 1]).sum()] +
                         [np.abs(mg[f][np.abs(isf) == 1]).sum() for f in range(4)])
        assert np.all(np.abs(out - ref) <= 1e-12 * scale + 1e-300), (call, out, ref)
    s.close()


def test_noalloc_reduce_rejects_boxes_beyond_its_scratch():
    import torch
    lib = capi.load()
    _bind(lib)
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = np.zeros(5, dtype=np.float64)
    rc = lib.lbf_reduce_noalloc(C.c_void_p(dummy.data_ptr()), None, None, 1, 1, 8193,
                                out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == -1
    assert "8192" in capi.last_error()
