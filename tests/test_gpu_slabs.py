"""The z-slab decomposition (lbf_create_slab, lbfast_b200/slabs.py) on one
GPU: a box split into 2 or 3 slabs, each a handle of its own with 3 halo
planes on each side refilled between steps by lbf_slabs_exchange, gives the
single box's results bit for bit -- periodic droplets, obstacles with walls,
wetting and bounce-back, one component; FP32 and FP64 storage."""
import numpy as np
import pytest

import lbfast_b200 as L
from cases import make_case
from lbfast_b200.slabs import SlabSet

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,storage", [("q27ho_2c_dr", "f32"), ("q27ho_2c_dr", "f64"), ("obs_q27ho_2c_dr", "f32"),
                                          ("obs_q27ho_2c_dr_bb", "f32"), ("tg_q19", "f32"), ("q27_1c", "f32")])
@pytest.mark.parametrize("nslabs,overlap", [(1, True), (2, True), (3, True), (2, False)])
def test_slabs_equal_the_single_box(name, storage, nslabs, overlap):
    """overlap: lbf_slabs_step (the halo copies beside the inner planes);
    else lbf_step per slab and a full exchange after each step."""
    p, isf, m, phi = make_case(name, storage)
    p.tile_y = 8 if storage == "f64" else 16
    a = L.Solver(p)
    if p.obstacles:
        a.set_isfluid(isf)
    a.set_fields(m, phi)
    a.step(12)
    ref = a.get_fields()
    a.close()
    s = SlabSet(p, nslabs)
    if p.obstacles:
        s.set_isfluid(isf)
    s.set_fields(m, phi)
    s.step(5, overlap=overlap)
    s.step(7, overlap=overlap)
    got = s.get_fields()
    s.close()
    for x, y, what in zip(got, ref, ("moments", "phi", "u_old")):
        if y is not None:
            assert np.array_equal(x, y, equal_nan=True), (name, storage, nslabs, overlap, what,
                                                          float(np.nanmax(np.abs(x - y))))


def test_slab_rejects_what_needs_the_whole_box():
    p, isf, m, phi = make_case("q27ho_2c_dr_corr", "f32")
    with pytest.raises(L.LbfError):
        SlabSet(p, 2)
    p, isf, m, phi = make_case("obs_q27ho_2c_dr", "f32")  # walls in y, periodic in z: fine
    SlabSet(p, 2).close()
    p.pbc_z = 0
    with pytest.raises(L.LbfError):
        SlabSet(p, 2)
