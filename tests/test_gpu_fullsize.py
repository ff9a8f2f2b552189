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
NSTEPS = 2000


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
    """FP32 storage and arithmetic against FP64 on the fluid after 2000 steps:
    phi within 1e-5 rel-L2 (measured 4.0e-6); the velocity, driven from rest
    by the body force, collects FP32 roundings as it grows and differs by
    6.2e-5 (1e-5 holds over the first 200 steps), bounded here by 1e-4."""
    isf, out = runs
    fl = np.abs(isf) == 1
    assert np.all(np.isfinite(out["f64"][0][:, fl])) and np.all(np.isfinite(out["f64"][1][fl]))
    eu, ep = rel_l2(out["f32"][0][1:4], out["f64"][0][1:4], fl), rel_l2(out["f32"][1], out["f64"][1], fl)
    print(f"channel 512x256x256 FP32 vs FP64 after {NSTEPS} steps: u {eu:.2e} phi {ep:.2e}")
    assert eu < 1e-4 and ep < 1e-5, (eu, ep)


def test_fullsize_fp16_against_fp64(runs):
    """FP16 storage: velocity, P and phi within 1e-3 rel-L2 of FP64 after 2000
    steps.  The body force adds ~1e-6 per step to a velocity of ~2e-4, which a
    16-bit u would re-round every step (a random walk of half-ulp errors that
    passes 1e-3 within a few hundred steps); P, u, v, w and phi are stored in
    FP32, and only Pi - u u and u_old -- rewritten from the FP32 state every
    step, so their roundings do not accumulate -- in 16 bits."""
    isf, out = runs
    fl = np.abs(isf) == 1
    eu = rel_l2(out["f16"][0][1:4], out["f64"][0][1:4], fl)
    eP = rel_l2(out["f16"][0][0:1], out["f64"][0][0:1], fl)
    ep = rel_l2(out["f16"][1], out["f64"][1], fl)
    print(f"channel FP16 storage vs FP64 after {NSTEPS} steps: u {eu:.2e} P {eP:.2e} phi {ep:.2e}")
    assert eu < 1e-3 and eP < 1e-3 and ep < 1e-3, (eu, eP, ep)


def test_fullsize_bf16_against_fp64(runs):
    """BF16 storage keeps 8 mantissa bits for Pi - u u and u_old (a relative
    rounding of 2^-9 = 2e-3 per store, against 2^-12 for FP16): velocity, P
    and phi within 1e-2 rel-L2 of FP64 after 2000 steps."""
    isf, out = runs
    fl = np.abs(isf) == 1
    eu = rel_l2(out["bf16"][0][1:4], out["f64"][0][1:4], fl)
    eP = rel_l2(out["bf16"][0][0:1], out["f64"][0][0:1], fl)
    ep = rel_l2(out["bf16"][1], out["f64"][1], fl)
    print(f"channel BF16 storage vs FP64 after {NSTEPS} steps: u {eu:.2e} P {eP:.2e} phi {ep:.2e}")
    assert eu < 1e-2 and eP < 1e-2 and ep < 1e-2, (eu, eP, ep)
