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


def test_noalloc_reduce_null_phi_null_isfluid_and_many_planes():
    """phi = NULL and isfluid = NULL (every node fluid) on 4 x 4 x 300 random
    fields -- more z planes than the total kernel's 256 threads, so its
    strided loop runs -- against numpy FP64 sums, twice in a row."""
    import torch
    lib = capi.load()
    _bind(lib)
    rng = np.random.default_rng(11)
    shape = (300, 4, 4)
    for call in range(2):
        m = rng.standard_normal((10,) + shape).astype(np.float32)
        m_dev = torch.from_numpy(m).cuda()
        torch.cuda.synchronize()
        rc, out = _noalloc(lib, m_dev, None, None, shape)
        assert rc == capi.LBF_OK, capi.last_error()
        ref = np.array([0.0] + [m[f].astype(np.float64).sum() for f in range(4)])
        scale = np.array([1.0] + [np.abs(m[f]).astype(np.float64).sum() for f in range(4)])
        assert out[0] == 0.0
        assert np.all(np.abs(out - ref) <= 1e-12 * scale), (call, out, ref)
    # phi given, isfluid NULL
    phi = rng.random(shape, dtype=np.float32)
    rc, out = _noalloc(lib, m_dev, torch.from_numpy(phi).cuda(), None, shape)
    assert rc == capi.LBF_OK, capi.last_error()
    assert abs(out[0] - phi.astype(np.float64).sum()) <= 1e-12 * phi.sum()


def test_noalloc_reduce_rejects_host_pointers_before_launch():
    """A host address (a Fortran call made outside host_data use_device) is
    refused with LBF_E_ARG by the pointer check; nothing is launched."""
    import torch
    lib = capi.load()
    _bind(lib)
    host = np.zeros((10, 2, 2, 2), dtype=np.float32)
    out = np.zeros(5, dtype=np.float64)
    rc = lib.lbf_reduce_noalloc(C.c_void_p(host.ctypes.data), None, None, 2, 2, 2,
                                out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == capi.LBF_E_ARG
    assert "mom10" in capi.last_error()
    dev = torch.zeros((10, 2, 2, 2), dtype=torch.float32, device="cuda")
    rc = lib.lbf_reduce_noalloc(C.c_void_p(dev.data_ptr()), C.c_void_p(host.ctypes.data), None, 2, 2, 2,
                                out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == capi.LBF_E_ARG
    assert "phi" in capi.last_error()
    # the context is intact: a valid call still works
    rc = lib.lbf_reduce_noalloc(C.c_void_p(dev.data_ptr()), None, None, 2, 2, 2,
                                out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == capi.LBF_OK, capi.last_error()


def test_noalloc_reduce_reports_non_finite_sums():
    """A NaN in the fields returns LBF_E_NUMERIC (sums still written), as lbf_reduce does."""
    import torch
    lib = capi.load()
    _bind(lib)
    m = np.zeros((10, 3, 3, 3), dtype=np.float32)
    m[2, 1, 1, 1] = np.nan
    rc, out = _noalloc(lib, torch.from_numpy(m).cuda(), None, None, (3, 3, 3))
    assert rc == capi.LBF_E_NUMERIC
    assert np.isnan(out[3]) and "u" in capi.last_error()


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
