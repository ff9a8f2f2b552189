"""Physics-level checks on the GPU: 16-bit storage against the FP64 oracle,
the reference's analytic benchmarks (statistics.f90: Taylor-Green viscous
decay, Laplace law), the Taylor-Green configuration of the reference's CPU
case against the oracle, and the C++ driver end to end."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from cases import make_case, rel_l2, run_oracle
import lbfast_b200 as L
from lbfast_b200 import statistics as ST

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(name, storage, n):
    p, isf, m, phi = make_case(name, storage)
    s = L.Solver(p)
    if p.obstacles:
        s.set_isfluid(isf)
    s.set_fields(m, phi)
    s.step(n)
    out = s.get_fields()
    s.close()
    return p, isf, out


def _fp16_errors(name, n=100):
    o = run_oracle(name, n, "f64")
    mo, po, _ = o.get_fields()
    p, isf, (mg, pg, _) = _run(name, "f16", n)
    fl = np.abs(isf) == 1
    err = {"P": rel_l2(mg[0:1], mo[0:1], fl), "u": rel_l2(mg[1:4], mo[1:4], fl),
           "Pi": rel_l2(mg[4:10], mo[4:10], fl)}
    if p.twocomponent:
        err["phi"] = rel_l2(pg, po, fl)
    return err


@pytest.mark.parametrize("name,p_bar", [("q27ho_2c_dr", 1e-3), ("obs_q27ho_2c_dr", 1e-3), ("open_q27ho_2c_dr", 1.5e-3),
                                        ("obs_q27ho_2c_dr_bb", 1e-3)])
def test_fp16_storage_two_component_within_1e3(name, p_bar):
    """16-bit storage (u_old and Pi - u u in FP16, one power-of-two scale per
    field group; P, u and phi in FP32; FP32 arithmetic) after 100 steps against the
    FP64 oracle: the observables P, u and phi within 1e-3 rel-L2, Pi within 3e-3.

    Open faces: there P is the small perturbation that the pressure face (0.001)
    drives through a closed box, and its FP16-storage error, 25-50x that of the
    periodic and obstacle cases, moves between 0.94e-3 and 1.25e-3 when the
    step kernel is compiled in ways that change only the last bit of FP32
    results (summation order, loop unrolling): the rounding of the 16-bit
    fields decides it, not the arithmetic.  Its bar is 1.5e-3, above that
    measured spread."""
    err = _fp16_errors(name)
    assert err["P"] <= p_bar and err["u"] <= 1e-3 and err["phi"] <= 1e-3 and err["Pi"] <= 3e-3, err


@pytest.mark.parametrize("name", ["q27ho_1c_force", "tg_q19"])
def test_fp16_storage_one_component(name):
    """One component: u within 1e-3, P within 3e-3, Pi (its non-equilibrium
    part stored in FP16) within 5e-3."""
    err = _fp16_errors(name)
    assert err["u"] <= 1e-3 and err["P"] <= 3e-3 and err["Pi"] <= 5e-3, err


@pytest.mark.parametrize("name", ["q27ho_2c_dr", "tg_q19"])
def test_bf16_storage_is_finite_and_close(name):
    """BF16 keeps 8 mantissa bits: finite and within 5e-2 of the FP64 oracle."""
    n = 100
    o = run_oracle(name, n, "f64")
    mo, po, _ = o.get_fields()
    p, isf, (mg, pg, _) = _run(name, "bf16", n)
    assert np.all(np.isfinite(mg))
    assert rel_l2(mg, mo) < 5e-2


def test_taylor_green_viscous_decay_linear_regime():
    """statistics.f90:918-956 on the GPU: 64^3 D3Q19, nu = 0.01, u0 = 5e-4
    (Re << 1, where E/E0 = exp(-6 nu k^2 t) holds): fitted nu within 1%."""
    n, nu = 64, 0.01
    s = L.Solver(L.Params(lx=n, ly=n, lz=n, lattice=19, visc1=nu))
    s.set_fields(L.ic_taylor_green(n, n, n, 5e-4))
    t, e = [], []
    for _ in range(11):
        _, vel, _ = s.get_print()
        t.append(s.nstep)
        e.append(ST.kinetic_energy(vel))
        s.step(100)
    s.close()
    t, e = np.array(t[1:]), np.array(e[1:])  # after the start-up transient of the regularised IC
    assert abs(ST.fit_viscosity(t, e, n) / nu - 1) < 0.01


def test_taylor_green_config_matches_oracle():
    """The reference's CPU case at its full length (64^3 D3Q19, nu = 0.01,
    u0 = 0.05, 1000 steps): the FP32 GPU run within 1e-5 rel-L2 of the FP64
    oracle after 200 and after 1000 steps, the FP64 GPU run within 1e-10."""
    n = 64
    from oracle import oracle as O
    m = L.ic_taylor_green(n, n, n, 0.05)
    o = O.Oracle(L.Params(lx=n, ly=n, lz=n, lattice=19, visc1=0.01).oracle_dict(), "f64")
    o.set_isfluid(np.ones((n, n, n), np.int8))
    o.set_fields(m)
    o.step(200)
    ref = {200: o.get_fields()[0]}
    o.step(800)
    ref[1000] = o.get_fields()[0]
    for storage, bar in (("f32", 1e-5), ("f64", 1e-10)):
        s = L.Solver(L.Params(lx=n, ly=n, lz=n, lattice=19, visc1=0.01, storage=storage))
        s.set_fields(m)
        done = 0
        for k in (200, 1000):
            s.step(k - done)
            done = k
            err = rel_l2(s.get_fields()[0], ref[k])
            assert err < bar, (storage, k, err)
        s.close()


def test_laplace_law():
    """statistics.f90:88-275 on a 128^3 droplet, R = 20, density ratio 100:
    the pressure jump settles (sigma_eff steady to 1% over the last 1000
    steps) and sigma_eff = dp R / 2 is within 30% of sigma (measured +21 %
    with this width-3 interface on R = 20, the same in the FP64 oracle: the
    scheme's, not the implementation's)."""
    n, R, sig = 128, 20.0, 0.03
    p = L.Params(lx=n, ly=n, lz=n, lattice=27, highorder=1, twocomponent=1, densratio=1, visc1=0.1, visc2=0.1,
                 rho_r=100.0, rho_b=1.0, sigma=sig, width=3.0, tau_diff=0.1, printphi=1)
    c = (n / 2, n / 2, n / 2)
    m, phi = L.ic_droplet(n, n, n, c, R, 3.0, sig, 100.0, 1.0, True)
    s = L.Solver(p)
    s.set_fields(m, phi)
    vals = []
    for _ in range(4):
        s.step(1000)
        rho, vel, press = s.get_print()
        vals.append(ST.laplace_observables(rho, press, c, (1, n // 2, n // 2), 100.0, 1.0))
        assert np.all(np.isfinite(vel))
    s.close()
    se = [v[0] for v in vals]
    assert abs(se[-1] / se[-2] - 1) < 0.01, se
    assert abs(se[-1] / sig - 1) < 0.3, se
    assert abs(vals[-1][2] - R) < 1.0


def test_driver_matches_library(tmp_path):
    """lbfast_b200/_lib/lbfast on a channel with walls, a droplet and
    obstacles-enabled wetting: runs, writes the reference's output files, and
    its last frame equals the same run driven through the Python binding."""
    exe = os.path.join(ROOT, "lbfast_b200", "_lib", "lbfast")
    shutil.copy(os.path.join(ROOT, "tests", "golden", "channel.inp"), tmp_path / "channel.inp")
    flags = ["-DLATTICE=27", "-DHIGHORDER", "-DTWOCOMPONENT", "-DDENSRATIO", "-DINTERNAL_OBSTACLES", "-DPRINTPHI"]
    r = subprocess.run([exe, *flags, "channel.inp"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "glups:" in r.stdout and "program correctly closed" in r.stdout
    out = tmp_path / "output"
    for f in ("out_rho_000000.raw", "out_vel_000002.raw", "out_rho_000002.xdmf"):
        assert (out / f).exists(), f
    lx, ly, lz = 36, 20, 24
    rho_drv = np.fromfile(out / "out_rho_000002.raw", dtype=np.float32).reshape(lz, ly, lx)
    vel_drv = np.fromfile(out / "out_vel_000002.raw", dtype=np.float32).reshape(lz, ly, lx, 3)
    # the same run through the binding
    isf = L.mark_isfluid(np.ones((lz, ly, lx), np.int8), (1, 0, 1), 27, True)
    m, phi = L.ic_droplet(lx, ly, lz, (18.0, 10.0, 12.0), 6.0, 4.0, 0.01, 0.5, 1.5, True, isf)
    phi = L.seed_solid_phi(phi, isf, 27)
    p = L.Params(lx=lx, ly=ly, lz=lz, pbc_y=0, lattice=27, highorder=1, twocomponent=1, densratio=1, obstacles=1,
                 visc1=0.05, visc2=0.2, rho_r=0.5, rho_b=1.5, sigma=0.01, width=4.0, tau_diff=0.1, fx=1e-5,
                 wettab_r=90.0, printphi=1)
    s = L.Solver(p)
    s.set_isfluid(isf)
    s.set_fields(m, phi)
    s.step(40)
    rho, vel, _ = s.get_print()
    s.close()
    assert np.array_equal(rho_drv, rho, equal_nan=True)
    assert np.array_equal(vel_drv, np.moveaxis(vel, 0, -1))


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_phi_mass_correction_holds_the_sum(storage):
    """The phi mass correction restores the FP64 sum of every step's input phi
    to its initial value (the reference corrects the input phi,
    integrator_module.f90:297), so after 1000 steps the output's sum is off
    by one step's change only -- the same size as the change of the last
    step of the uncorrected run -- while without it the droplet case drifts
    by more than 1e-4 (phi is stored in FP32 in both modes)."""
    sums = {}
    for corr in (0, 1):
        p, isf, m, phi = make_case("q27ho_2c_dr", storage)
        p.phi_correction = corr
        s = L.Solver(p)
        s.set_fields(m, phi)
        s.step(999)
        prev = float(np.sum(s.get_fields()[1].astype(np.float64)))
        s.step(1)
        sums[corr] = (float(np.sum(s.get_fields()[1].astype(np.float64))), prev)
        s.close()
    s0 = float(np.sum(phi.astype(np.float64)))
    step_change = abs(sums[0][0] - sums[0][1])
    assert abs(sums[0][0] - s0) / s0 > 1e-4, sums
    assert abs(sums[1][0] - s0) < 2 * step_change + 1e-7 * s0, (sums, step_change)


def test_restart_resumes_the_run(tmp_path):
    """A run stopped after 20 steps, written to restart.raw and resumed stays
    within 1e-3 rel-L2 of the uninterrupted 40-step run.  The restart is the
    reference's (print_module.f90:1474-1677): one time level in float32, so the
    resumed run starts from rounded fields and from u_old = u."""
    p, isf, m, phi = make_case("q27ho_2c_dr", "f32")
    a = L.Solver(p)
    a.set_fields(m, phi)
    a.step(40)
    ma, pa, _ = a.get_fields()
    a.close()
    b = L.Solver(p)
    b.set_fields(m, phi)
    b.step(20)
    mb, pb, _ = b.get_fields(np.float32)
    b.close()
    L.write_restart_raw(str(tmp_path), mb, pb, 1, 0)
    m2, p2, fr, _ = L.read_restart_raw(str(tmp_path), p.lx, p.ly, p.lz, True)
    assert fr == 1
    c = L.Solver(p)
    c.set_fields(m2, p2)
    c.step(20)
    mc, pc, _ = c.get_fields()
    c.close()
    assert rel_l2(mc, ma) < 1e-3 and rel_l2(pc, pa) < 1e-4, (rel_l2(mc, ma), rel_l2(pc, pa))


@pytest.mark.parametrize("name,storage", [("obs_q27ho_2c_dr_corr", "f32"), ("obs_q27ho_2c_dr_corr", "f16"),
                                          ("open_q27ho_2c_dr_corr", "f32"), ("q27ho_2c_dr", "f64"),
                                          ("rep_q27ho_2c_dr", "f32"), ("tg_q19", "bf16")])
def test_checkpoint_resumes_bit_for_bit(tmp_path, name, storage):
    """The full-state checkpoint (lbf_write_checkpoint): a run stopped after
    17 steps, checkpointed, and resumed in a new handle from the file for 23
    steps equals the uninterrupted 40-step run bit for bit -- moments, phi
    and u_old -- with obstacles and wetting (whose ghost values are written
    one step late), the phi mass correction, open faces, REPULSIVE_FLUX and
    every storage format; also when the checkpoint is taken at step 0."""
    p, isf, m, phi = make_case(name, storage)

    def fresh():
        s = L.Solver(p)
        if p.obstacles:
            s.set_isfluid(isf)
        return s

    a = fresh()
    a.set_fields(m, phi)
    a.step(40)
    ref = a.get_fields()
    a.close()
    for k in (0, 17):
        b = fresh()
        b.set_fields(m, phi)
        b.step(k)
        path = tmp_path / f"ckpt_{k}.bin"
        b.write_checkpoint(path)
        b.close()
        c = fresh()
        c.read_checkpoint(path)
        assert c.nstep == k
        c.step(40 - k)
        got = c.get_fields()
        c.close()
        for x, y in zip(got, ref):
            if y is not None:
                assert np.array_equal(x, y, equal_nan=True), (k, name, storage)


def test_checkpoint_rejects_another_configuration(tmp_path):
    """A checkpoint read into a handle of another storage or box is refused
    with LBF_E_ARG and leaves that handle unchanged."""
    p, isf, m, phi = make_case("q27ho_2c_dr", "f32")
    s = L.Solver(p)
    s.set_fields(m, phi)
    s.step(3)
    s.write_checkpoint(tmp_path / "c.bin")
    s.close()
    for change in ({"storage": "f16"}, {"lx": p.lx + 2}):
        q = L.Params(**{**p.__dict__, **change})
        t = L.Solver(q)
        with pytest.raises(L.LbfError):
            t.read_checkpoint(tmp_path / "c.bin")
        t.close()


def test_driver_writes_and_reads_restart(tmp_path):
    """lwriterestart writes output/restart.raw at the end of the run
    (integrator_module.f90:834-840); lrestart resumes from it with the frame
    counter restored (integrator_module.f90:167-176)."""
    exe = os.path.join(ROOT, "lbfast_b200", "_lib", "lbfast")
    text = open(os.path.join(ROOT, "tests", "golden", "channel.inp")).read()
    flags = ["-DLATTICE=27", "-DHIGHORDER", "-DTWOCOMPONENT", "-DDENSRATIO", "-DINTERNAL_OBSTACLES", "-DPRINTPHI"]
    (tmp_path / "a.inp").write_text(text.replace("   nsteps=40", "   nsteps=40\n   lwriterestart=.true."))
    r = subprocess.run([exe, *flags, "a.inp"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    n = 36 * 20 * 24
    assert (tmp_path / "output" / "restart.raw").stat().st_size == 4 * n * 11 + 8
    (tmp_path / "b.inp").write_text(text.replace("   nsteps=40", "   nsteps=20\n   lrestart=.true."))
    r = subprocess.run([exe, *flags, "b.inp"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "restart read: iframe 2" in r.stdout
    assert (tmp_path / "output" / "out_rho_000003.raw").exists()


@pytest.mark.parametrize("lattice", [19, 27])
def test_poiseuille_profile(lattice):
    """The reference's POISEUILLE case (poiseuille.inp: lx = 64 with walls at
    gi = 1 and lx, fz = 0.5e-5, nu = 0.1; statistics.f90:825-880) run to the
    steady state: the plane-averaged velocity matches the reference's
    parabola, H = (lx - 1)/2 about xc = (lx + 1)/2 -- the moment-space
    bounce-back of lb_cuda_boundary_module.f90:162-199 puts the no-slip plane
    on the solid nodes -- within 0.5 % of its peak (the half-way parabola is
    3 % off)."""
    lx, ly, lz, fz, nu = 64, 8, 32, 0.5e-5, 0.1
    isf = L.mark_isfluid(np.ones((lz, ly, lx), np.int8), (0, 1, 1), lattice, True)
    p = L.Params(lx=lx, ly=ly, lz=lz, pbc_x=0, lattice=lattice, obstacles=1, visc1=nu, fz=fz)
    s = L.Solver(p)
    s.set_isfluid(isf)
    s.set_fields(np.zeros((10, lz, ly, lx)))
    s.step(40000)
    _, vel, _ = s.get_print()
    s.close()
    num = ST.poiseuille_profile(vel[2], isf)
    th = ST.poiseuille_theory(lx, fz, nu, H=(lx - 1) / 2, xc=(lx + 1) / 2)
    err = np.abs(num[1:-1] - th[1:-1]).max() / th.max()
    assert err < 0.005, err


@pytest.mark.parametrize("lattice", [19, 27])
def test_poiseuille_profile_bounce_back(lattice):
    """The POISEUILLE case with BOUNCE_BACK: the half-way bounce-back puts the
    no-slip plane between the solid and the first fluid node, and the profile
    matches the reference's parabola for it, H = (lx - 2)/2
    (init_conditions_module.f90:248-252), within 0.5 % of its peak."""
    lx, ly, lz, fz, nu = 64, 8, 32, 0.5e-5, 0.1
    isf = L.mark_isfluid(np.ones((lz, ly, lx), np.int8), (0, 1, 1), lattice, True)
    p = L.Params(lx=lx, ly=ly, lz=lz, pbc_x=0, lattice=lattice, obstacles=1, visc1=nu, fz=fz, bounce_back=1)
    s = L.Solver(p)
    s.set_isfluid(isf)
    s.set_fields(np.zeros((10, lz, ly, lx)))
    s.step(40000)
    _, vel, _ = s.get_print()
    s.close()
    num = ST.poiseuille_profile(vel[2], isf)
    th = ST.poiseuille_theory(lx, fz, nu, H=(lx - 2) / 2, xc=(lx + 1) / 2)
    err = np.abs(num[1:-1] - th[1:-1]).max() / th.max()
    assert err < 0.005, err


def test_lamb_oscillation_frequency():
    """Lamb's n = 2 oscillation (the observable and theory of statistics.f90:
    377-471, 959-1050; sigma 0.03, nu 0.001, equal densities of lamb.inp) of
    a droplet R = 20 in 128^3 with a small P2 surface perturbation
    (r = R (1 + 0.05 P2(cos theta)), where linear theory holds; the reference's
    own LAMBTEST starts from a 2:1 ellipsoid, far outside it).  The z
    half-axis swings through one clean cycle (trough near step 1200, peak near
    2450, trough near 3400); after it the damped mode gives way to wiggles of
    about 0.1 node, where counting every local maximum above the mean (the
    reference's mean_period) picks up noise and moves with the last bits of
    the arithmetic.  So the period is the first cycle's, trough to trough,
    in FP32 and FP64 storage: the two agree to 0.5 % and along the series to
    1e-3 nodes, and the period is 1.3-1.6 times Lamb's with the reference's
    viscous correction -- measured 1.45, the scheme's, with a width-4
    interface on R = 20 and the phase-field relaxation (the FP64 step equals
    the oracle's to 1e-14)."""
    n, R, sig, nu, W, eps = 128, 20.0, 0.03, 0.001, 4.0, 0.05
    c = n / 2
    x = np.arange(1, n + 1) - c
    z, y, xx = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(xx * xx + y * y + z * z)
    ct = np.divide(z, r, out=np.zeros_like(r), where=r > 0)
    phi = 0.5 * (1 - np.tanh((r - R * (1 + eps * 0.5 * (3 * ct * ct - 1))) / (0.5 * W)))
    m = np.zeros((10, n, n, n))
    m[0] = phi * (2 * sig) / R / (1.0 / 3.0)  # the reference's Laplace pressure, rho_phi = 1
    runs = {}
    for storage in ("f32", "f64"):
        p = L.Params(lx=n, ly=n, lz=n, lattice=27, highorder=1, twocomponent=1, visc1=nu, visc2=nu, sigma=sig,
                     width=W, tau_diff=0.1, printphi=1, storage=storage)
        s = L.Solver(p)
        s.set_fields(m, phi)
        steps, dosc = [], []
        for k in range(181):
            rho, _, _ = s.get_print()
            steps.append(k * 20)
            dosc.append(ST.lamb_observables(rho)[2])
            s.step(20)
        s.close()
        runs[storage] = (np.array(steps, dtype=np.float64), np.array(dosc))
    T_th = 2 * np.pi / ST.lamb_theory_omega(sig, R, 1.0, 1.0, nu, nu)
    ex = {k: ST.first_extrema(*v, 3) for k, v in runs.items()}
    for k, e in ex.items():
        assert [kind for _, _, kind in e] == ["min", "max", "min"], (k, e)
    T = {k: e[2][0] - e[0][0] for k, e in ex.items()}
    dev = float(np.max(np.abs(runs["f32"][1] - runs["f64"][1])))
    print(f"lamb first cycle: period FP32 {T['f32']:.1f} FP64 {T['f64']:.1f} steps, "
          f"{T['f64'] / T_th:.3f} x Lamb's {T_th:.1f}; max |FP32 - FP64| of the z half-axis {dev:.2e}")
    assert abs(T["f32"] / T["f64"] - 1) < 0.005, T
    assert dev < 1e-3, dev
    assert 1.3 <= T["f64"] / T_th <= 1.6, (T, T_th)
    # damped: the second trough is shallower than the first
    e = ex["f64"]
    assert e[2][1] > e[0][1], e
