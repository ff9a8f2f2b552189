"""The two-component channel with obstacles at its full size, 512 x 256 x 256.

The CPU oracle cannot step 33.5 M nodes in test time, so at this size the
FP64 path of the library -- equal to the FP64 oracle to 1e-14 on the small
cases -- is the reference, and FP32 / FP16 / BF16 storage are compared with
it on the same inputs: walls at y = 1 and y = ly (pbc = 1, 0, 1), 64 seeded
solid spheres of radius U[6, 14] (seed 12345), phi from 32 seeded blobs of
radius U[8, 24] with a width-4 tanh profile (seed 67890), fx = 1e-6,
nu1 = 0.05, nu2 = 0.4, rho_r = 0.5, rho_b = 1.5, sigma = 0, wetting at 90
degrees (the twopoiseuille.inp parameters).  Spheres are kept clear of the
periodic faces: a sphere cut by one leaves solid nodes whose in-box seed is
0/0 next to fluid (init_conditions_module.f90:492-541), in the reference too.
"""
import numpy as np
import pytest

import lbfast_b200 as L
from bench import channel_geometry
from cases import rel_l2

pytestmark = pytest.mark.gpu

LX, LY, LZ = 512, 256, 256
NSTEPS = 200


def _geometry():
    return channel_geometry(LX, LY, LZ)


@pytest.fixture(scope="module")
def runs():
    isf, phi = _geometry()
    m = np.zeros((10, LZ, LY, LX))
    out = {}
    for storage in ("f64", "f32", "f16", "bf16"):
        p = L.Params(lx=LX, ly=LY, lz=LZ, pbc_y=0, lattice=27, highorder=1, twocomponent=1, densratio=1,
                     obstacles=1, visc1=0.05, visc2=0.4, rho_r=0.5, rho_b=1.5, sigma=0.0, width=4.0,
                     tau_diff=0.1, fx=1e-6, wettab_r=90.0, storage=storage)
        s = L.Solver(p)
        s.set_isfluid(isf)
        s.set_fields(m, phi)
        s.step(NSTEPS)
        mg, pg, _ = s.get_fields(np.float32)
        s.close()
        out[storage] = (mg, pg)
    return isf, out


def test_fullsize_fp32_against_fp64(runs):
    """FP32 storage and arithmetic: within 1e-5 rel-L2 of FP64 on the fluid."""
    isf, out = runs
    fl = np.abs(isf) == 1
    assert np.all(np.isfinite(out["f64"][0][:, fl])) and np.all(np.isfinite(out["f64"][1][fl]))
    eu, ep = rel_l2(out["f32"][0][1:4], out["f64"][0][1:4], fl), rel_l2(out["f32"][1], out["f64"][1], fl)
    assert eu < 1e-5 and ep < 1e-5, (eu, ep)


@pytest.mark.parametrize("storage,mant", [("f16", 11), ("bf16", 8)])
def test_fullsize_16bit_against_fp64(runs, storage, mant):
    """16-bit storage: velocity and phi within the storage format's bar of FP64.

    The body force adds ~1e-6 per step to a velocity of ~2e-4, so every step
    re-rounds u to the format's mantissa (half an ulp, 2^-mant relative); the
    roundings add as a random walk, sqrt(steps) * 2^-mant: 3.5e-3 for FP16,
    2.8e-2 for BF16 after 200 steps."""
    bar = np.sqrt(NSTEPS) * 2.0 ** -mant
    isf, out = runs
    fl = np.abs(isf) == 1
    eu, ep = rel_l2(out[storage][0][1:4], out["f64"][0][1:4], fl), rel_l2(out[storage][1], out["f64"][1], fl)
    assert eu < bar and ep < bar, (eu, ep)
