"""The CPU oracle against what pins it: the reference's Minv_mrt table, the
reference's analytic Taylor-Green check (statistics.f90:918-956), and the
invariants of the scheme.  No GPU."""
import json
import os

import numpy as np
import pytest

from cases import make_case, rel_l2, run_oracle
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_minv_table_matches_reference_table():
    ref = np.load(os.path.join(GOLDEN, "minv_mrt.npy"))  # parsed from vars_module.f90:360-521
    assert np.abs(O.minv_table() - ref).max() < 1e-15


def _tg(L, u0, nu, steps, chunk, prec="f64"):
    p = dict(lx=L, ly=L, lz=L, pbc_x=1, pbc_y=1, pbc_z=1, lattice=19, highorder=0, twocomp=0, densratio=0,
             obstacles=0, visc1=nu)
    o = O.Oracle(p, prec)
    o.set_isfluid(np.ones((L, L, L), np.int8))
    o.set_fields(O.ic_taylor_green(L, L, L, u0))
    t, e = [], []
    for _ in range(steps // chunk + 1):
        _, vel, _ = o.get_print()
        t.append(o.nstep)
        e.append(0.5 * np.mean((vel ** 2).sum(0)))
        o.step(chunk)
    return np.array(t), np.array(e), o


def test_taylor_green_viscous_decay():
    """statistics.f90:918-956: E/E0 ~ exp(-6 nu k^2 t); fit nu in the linear regime."""
    L, nu = 24, 0.01
    t, e, _ = _tg(L, 5e-4, nu, 300, 50)
    k = 2 * np.pi / L
    sel = t >= 50  # after the initial non-equilibrium transient of the regularised start
    slope = np.polyfit(t[sel], np.log(e[sel] / e[0]), 1)[0]
    nu_fit = -slope / (6 * k * k)
    assert abs(nu_fit / nu - 1) < 0.03, nu_fit


def test_one_component_conserves_mass_and_momentum():
    _, _, o = _tg(16, 0.05, 0.02, 60, 60)
    h0 = O.ic_taylor_green(16, 16, 16, 0.05)
    h, _, _ = o.get_fields()
    assert abs(h[0].sum() - h0[0].sum()) < 1e-12
    for f in (1, 2, 3):
        assert abs(h[f].sum() - h0[f].sum()) < 1e-12


def test_rest_state_is_stationary():
    for name in ("q27ho_2c_dr", "q19_2c", "tg_q19"):
        p, isf, m, phi = make_case(name)
        d = p.oracle_dict()
        d.update(fx=0.0, fy=0.0, fz=0.0)  # no body force: the rest state must stay at rest
        o = O.Oracle(d, "f64")
        o.set_isfluid(isf)
        z = np.zeros_like(m)
        ph = None if phi is None else np.full(phi.shape, 0.3)
        o.set_fields(z, ph)
        o.step(5)
        h, phi2, _ = o.get_fields()
        assert np.abs(h).max() < 1e-14
        if ph is not None:
            assert np.abs(phi2 - 0.3).max() < 1e-14


@pytest.mark.parametrize("name", ["q27ho_2c_dr", "obs_q19_1c"])
def test_single_precision_build_tracks_double(name):
    a = run_oracle(name, 10, "f64")
    b = run_oracle(name, 10, "f32")
    p, isf, _, _ = make_case(name)
    fl = np.abs(isf) == 1
    ha, pa, _ = a.get_fields()
    hb, pb, _ = b.get_fields()
    assert rel_l2(hb, ha, fl) < 1e-5
    if p.twocomponent:
        assert rel_l2(pb, pa, fl) < 1e-6


def test_prime_wetting_copies_donor_phi():
    """integrator_module.f90:186-190 runs the wetting before the loop with aux = 0:
    every updated ghost equals its donor's phi (gradient terms vanish)."""
    p, isf, m, phi = make_case("obs_q27ho_2c_dr")
    o = O.Oracle(p.oracle_dict(), "f64")
    o.set_isfluid(isf)
    o.set_fields(m, phi)
    o.step(0)
    a, _ = o.get_phi_buffers()
    solid = (isf == 0) & np.isfinite(phi)
    changed = solid & (np.abs(a - phi) > 0)
    assert changed.sum() > 0
    vals = a[changed]
    assert np.all((vals >= 0) & (vals <= 1))


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_phi_mass_correction_restores_the_initial_sum(prec):
    """boundary_cds_module.f90:1864-1885: the correction restores the FP64 sum
    of the input phi of every step to its initial value (inside
    bcs_mesoscopic_phifields, integrator_module.f90:297), so the sum of a
    step's output differs from the initial one by that step's own change only
    and the drift does not accumulate; without it this droplet loses about
    0.13 % in 200 steps."""
    dev = {}
    for corr in (0, 1):
        p, isf, m, phi = make_case("q27ho_2c_dr")
        p.phi_correction = corr
        o = O.Oracle(p.oracle_dict(), prec)
        o.set_isfluid(isf)
        o.set_fields(m, phi)
        o.step(199)
        s199 = np.sum(o.get_fields()[1].astype(np.float64))
        o.step(1)
        s200 = np.sum(o.get_fields()[1].astype(np.float64))
        dev[corr] = (s200, s199)
    s0 = np.sum(phi)
    # uncorrected: the accumulated drift
    assert abs(dev[0][0] - s0) / s0 > 1e-3
    # corrected: the output of step 200 is the corrected input (sum s0) plus
    # the change of step 200 itself -- of the size of one step's change of
    # the uncorrected run (about 1e-5 of the sum here), not of the drift
    step_change = abs(dev[0][0] - dev[0][1])
    assert abs(dev[1][0] - s0) < 2 * step_change, (dev, step_change)
    assert abs(dev[1][0] - s0) / s0 < 2e-5


@pytest.mark.parametrize("name", ["q27ho_1c_force", "obs_q27ho_2c_dr"])
def test_smagorinsky_changes_the_relaxation(name):
    """SMAGORINSKI raises tau where the non-equilibrium stress is large
    (lb_cuda_fused_module.f90:609-616): the run departs from the molecular one
    by more than the FP64 noise and stays finite."""
    out = {}
    for smag in (0, 1):
        p, isf, m, phi = make_case(name)
        p.smagorinsky = smag
        o = O.Oracle(p.oracle_dict(), "f64")
        o.set_isfluid(isf)
        o.set_fields(m, phi)
        o.step(10)
        out[smag] = o.get_fields()[0]
    fl = np.abs(isf) == 1
    assert np.all(np.isfinite(out[1][:, fl]))
    assert rel_l2(out[1], out[0], fl) > 1e-6


@pytest.mark.parametrize("lattice", [27, 19, 15])
def test_lattice_tables_match_the_reference(lattice):
    """Link vectors, opposites and weights of D3Q27 / D3Q19 / D3Q15 as the
    reference defines them (vars_module.f90:319-338, 666-684, 685-703; parsed
    into tests/golden/lattice_tables.json by make_lattice_golden.py), and
    D3Q19 / D3Q15 as subsets of the D3Q27 order (links 0-18; 0-6 and 19-26),
    which the kernels and the host code rely on."""
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "lattice_tables.json")))[str(lattice)]
    t = O.lattice_table(lattice)
    assert t["ex"] == g["ex"] and t["ey"] == g["ey"] and t["ez"] == g["ez"] and t["opp"] == g["opp"]
    assert np.allclose(t["w"], g["w"], rtol=1e-15, atol=0)
    g27 = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "lattice_tables.json")))["27"]
    sub = list(range(27)) if lattice == 27 else list(range(19)) if lattice == 19 else list(range(7)) + list(range(19, 27))
    assert [g27["ex"][l] for l in sub] == g["ex"]
    assert [g27["ey"][l] for l in sub] == g["ey"]
    assert [g27["ez"][l] for l in sub] == g["ez"]


def _open_channel(types, press, vel, lx=40, ly=14, lz=4, steps=2000):
    """Channel along x between resting velocity faces at y (walls at y = 0 and
    ly-1), periodic in z, open x faces; one component, D3Q19."""
    isf = O.mark_isfluid(np.zeros((lz, ly, lx), bool), (0, 0, 1), 19, True)
    p = dict(lx=lx, ly=ly, lz=lz, pbc_x=0, pbc_y=0, pbc_z=1, lattice=19, obstacles=1, visc1=0.1, openbc=1,
             openbc_type=(types, (0, 0), (0, 0)), openbc_press=(press, (0.0, 0.0), (0.0, 0.0)),
             openbc_vel=(vel, ((0.0,) * 3,) * 2, ((0.0,) * 3,) * 2))
    o = O.Oracle(p)
    o.set_isfluid(isf)
    o.set_fields(np.zeros((10, lz, ly, lx)))
    o.step(steps)
    h, _, _ = o.get_fields()
    return h


def test_open_pressure_faces_drive_poiseuille_flow():
    """Pressure faces at x (boundary_cds_module.f90:57-470, openbc_type 1):
    the steady flow is a Poiseuille profile for the interior pressure
    gradient, u(y) = G / (2 nu) (H^2 - (y - yc)^2) with p = P / 3 and the
    bounce-back walls on the solid rows (H = (ly - 1) / 2)."""
    lx, ly = 40, 14
    h = _open_channel((1, 1), (0.01, -0.01), ((0.0,) * 3,) * 2, lx=lx, ly=ly)
    # -dp/dx from a linear fit of P along the middle of the channel (the
    # faces distort the few planes next to them)
    xs = np.arange(10, lx - 10)
    G = -np.polyfit(xs, h[0, 2, ly // 2, xs], 1)[0] / 3.0
    assert G > 0
    y = np.arange(ly)
    Hh, yc = (ly - 1) / 2, (ly - 1) / 2
    theory = G / (2 * 0.1) * (Hh * Hh - (y - yc) ** 2)
    u = h[1, 2, :, lx // 2]
    inner = slice(1, ly - 1)
    assert np.abs(u[inner] - theory[inner]).max() < 0.02 * theory.max()
    assert np.abs(h[2:4, 2, inner, lx // 2]).max() < 1e-4 * theory.max()  # no cross flow


def test_open_velocity_inlet_conserves_the_flow_rate():
    """Velocity face at x low (openbc_type 0) and pressure face at x high: the
    steady flow rate through every interior plane is the same and positive."""
    lx, ly = 48, 14
    h = _open_channel((0, 1), (0.0, 0.0), ((0.01, 0.0, 0.0), (0.0,) * 3), lx=lx, ly=ly, steps=3000)
    q = h[1, 1, 1:ly - 1, :].sum(0)
    inner = q[10:lx - 10]  # planes away from the faces' distortion
    assert inner.min() > 0
    assert (inner.max() - inner.min()) < 1e-3 * inner.mean()


@pytest.mark.parametrize("bb,H_off", [(0, 1), (1, 2)])
def test_poiseuille_wall_position(bb, H_off):
    """Body-force Poiseuille between walls at y = 0 and ly-1: the moment-space
    bounce-back (LB_int_boundary) puts the no-slip plane on the solid rows,
    H = (ly-1)/2; BOUNCE_BACK half way between solid and fluid, H = (ly-2)/2
    (init_conditions_module.f90:248-252)."""
    lx, ly, lz, nu, fx = 4, 18, 4, 0.1, 1e-6
    isf = O.mark_isfluid(np.zeros((lz, ly, lx), bool), (1, 0, 1), 19, True)
    o = O.Oracle(dict(lx=lx, ly=ly, lz=lz, pbc_x=1, pbc_y=0, pbc_z=1, lattice=19, obstacles=1, visc1=nu, fx=fx,
                      bounce_back=bb))
    o.set_isfluid(isf)
    o.set_fields(np.zeros((10, lz, ly, lx)))
    o.step(6000)
    h, _, _ = o.get_fields()
    y = np.arange(ly)
    H, yc = (ly - H_off) / 2, (ly - 1) / 2
    theory = fx / (2 * nu) * (H * H - (y - yc) ** 2)
    u = h[1, 1, :, 1]
    assert np.abs(u[1:-1] - theory[1:-1]).max() < 0.01 * theory.max()


def _rep_run(name, far, on, steps=12):
    p, isf, m, phi = make_case(name)
    d = p.oracle_dict()
    d["repulsive_flux"] = on
    if far:
        # droplets of R = 7 (interfacial band q >= q_th from r = 4.8 to 9.2:
        # no two band nodes of one droplet with normals 120 degrees apart fit
        # the +-3 node window) 24 nodes apart both ways in a 48 x 24 x 24 box:
        # no facing pair exists
        L = (48, 24, 24)
        d.update(lx=L[0], ly=L[1], lz=L[2])
        m1, p1 = O.ic_droplet(*L, (12.0, 12.0, 12.0), 7.0, 3.0, 0.02, p.rho_r, p.rho_b, bool(p.densratio))
        m2, p2 = O.ic_droplet(*L, (36.0, 12.5, 12.0), 7.0, 3.0, 0.02, p.rho_r, p.rho_b, bool(p.densratio))
        phi, m = np.maximum(p1, p2), m1 + m2
        isf = np.ones(L[::-1], np.int8)
    o = O.Oracle(d)
    o.set_isfluid(isf)
    o.set_fields(m, phi)
    o.step(steps)
    return o.get_fields()


def test_repulsive_flux_acts_only_across_thin_films():
    """REPULSIVE_FLUX (lb_cuda_repulsive_module.f90:19-292): two droplets whose
    interfaces face each other across a film of about three nodes feel the
    film force, first in the film; droplets whose interfaces are further
    apart than the +-3 node window feel none, and the run equals the one
    without the switch bit for bit."""
    a_on, a_off = _rep_run("rep_q27ho_2c_dr", False, 1), _rep_run("rep_q27ho_2c_dr", False, 0)
    assert np.abs(a_on[0] - a_off[0]).max() > 1e-6
    # the difference of phi is largest in the film between the droplets (x = 15 .. 19)
    d = np.abs(a_on[1] - a_off[1]).max(axis=(0, 1))
    assert d[14:21].max() > 10 * max(d[:5].max(), d[-5:].max())
    b_on, b_off = _rep_run("rep_q27ho_2c_dr", True, 1), _rep_run("rep_q27ho_2c_dr", True, 0)
    assert all(np.array_equal(x, y) for x, y in zip(b_on, b_off))
