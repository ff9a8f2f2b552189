"""Host side of the library (no GPU): the C ABI loads and exports every
declared symbol, the set-up helpers agree with the oracle's restatements of
the reference, the namelist reader accepts the reference's input format, the
raw/XDMF writer produces the reference's files, and invalid parameters are
rejected before any device work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from cases import _spheres_solid
import lbfast_b200 as L
from lbfast_b200 import capi
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbfast_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


class Run(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nsteps stamp stamp2D stamp_term stepskip lreadisfluid lreadinit lprint "
                                       "lvtk lraw lrestart lwriterestart openbc nplanes every_time_check iprobe "
                                       "jprobe kprobe").split()] + \
               [("time_limit", C.c_double), ("uwall", C.c_double), ("radius", C.c_double), ("width", C.c_double),
                ("center", C.c_double * 3)]


def read_nml(path):
    lib = capi.load()
    lib.lbf_read_namelists.argtypes = [C.c_char_p, C.POINTER(capi.LbfParams), C.POINTER(Run)]
    p = capi.LbfParams()
    r = Run()
    rc = lib.lbf_read_namelists(str(path).encode(), C.byref(p), C.byref(r))
    return rc, p, r


@pytest.mark.parametrize("pbc", [(1, 1, 1), (1, 0, 1), (0, 1, 0)])
@pytest.mark.parametrize("lattice", [19, 27])
def test_mark_isfluid_matches_restatement(pbc, lattice):
    rng = np.random.default_rng(11 + lattice)
    solid = _spheres_solid(rng, (14, 18, 22), 3, 2.0, 3.5)
    a = capi.mark_isfluid((~solid).astype(np.int8), pbc, lattice, True)
    b = O.mark_isfluid(solid, pbc, lattice, True)
    assert np.array_equal(a, b)
    assert (a == -1).sum() > 0


def test_initial_conditions_match_restatement():
    m = capi.ic_taylor_green(32, 24, 16, 0.05)
    assert np.allclose(m, O.ic_taylor_green(32, 24, 16, 0.05), rtol=0, atol=1e-15)
    m, phi = capi.ic_droplet(40, 24, 28, (20.5, 12, 14.5), 7, 3, 0.03, 1.0, 0.1, True)
    m2, phi2 = O.ic_droplet(40, 24, 28, (20.5, 12, 14.5), 7, 3, 0.03, 1.0, 0.1, True)
    assert np.allclose(m, m2, rtol=1e-14, atol=1e-16) and np.allclose(phi, phi2, rtol=1e-14, atol=1e-16)
    # the droplet straddles the periodic faces: nearest-image distance
    m, phi = capi.ic_droplet(24, 24, 24, (1.0, 23.0, 12.0), 5, 3, 0.03, 1.0, 0.1, True)
    assert phi[11, 22, 0] > 0.99 and phi[11, 0, 1] > 0.5


def test_seed_solid_phi_matches_restatement_including_nan():
    rng = np.random.default_rng(5)
    isf = O.mark_isfluid(_spheres_solid(rng, (12, 16, 20), 3, 2.0, 3.5), (1, 1, 1), 27, True)
    phi = rng.random(isf.shape)
    a = capi.seed_solid_phi(phi, isf, 27)
    b = O.seed_solid_phi(phi, isf, 27)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    assert np.nanmax(np.abs(a - b)) < 1e-15


def test_namelist_reader_defaults_and_values():
    rc, p, r = read_nml(os.path.join(ROOT, "tests", "golden", "channel.inp"))
    assert rc == 0
    assert (p.lx, p.ly, p.lz, p.pbc_x, p.pbc_y, p.pbc_z) == (36, 20, 24, 1, 0, 1)
    assert p.fx == 1e-5 and p.visc1 == 0.05 and p.visc2 == 0.2 and p.rho_r == 0.5 and p.rho_b == 1.5
    assert p.sigma == 0.01 and p.width == 4.0 and p.tau_diff == 0.1 and p.wettab_r == 60.0
    assert (r.nsteps, r.stamp, r.stamp_term, r.iprobe, r.jprobe, r.kprobe) == (40, 20, 10, 5, 10, 12)
    assert list(r.center) == [18.0, 10.0, 12.0] and r.radius == 6.0
    assert r.time_limit == -1.0 and r.every_time_check == 1000  # vars_module.f90:777-779


def test_namelist_reader_rejects_bad_input(tmp_path):
    base = open(os.path.join(ROOT, "tests", "golden", "channel.inp")).read()
    cases = {"unknown": base.replace("lx=36", "lx=36\n   bogus_key=3"),
             "badreal": base.replace("fx=1.0d-5", "fx=1.0x-5"),
             "badelement": base.replace("openbc=0", "openbc=1\n   openbc_type_x(3)=1"),
             "badopenkey": base.replace("openbc=0", "openbc=1\n   openbc_q_x=1"),
             "nofluid": base.split("&fluid")[0]}
    for name, text in cases.items():
        f = tmp_path / f"{name}.inp"
        f.write_text(text)
        rc, _, _ = read_nml(f)
        assert rc != 0, name


def test_namelist_reader_reads_open_faces(tmp_path):
    """openbc and the openbc_* arrays of vars_module.f90:238-255, whole-array
    and element assignments, go to the parameters."""
    base = open(os.path.join(ROOT, "tests", "golden", "channel.inp")).read()
    text = base.replace("openbc=0", "openbc=1\n   openbc_type_x=1,2\n   openbc_press_x(1)=0.01d0\n"
                                    "   openbc_type_y(2)=0\n   openbc_u_y(2)=0.05\n   openbc_w_z=0.5,-0.25")
    f = tmp_path / "open.inp"
    f.write_text(text)
    rc, p, r = read_nml(f)
    assert rc == 0 and p.openbc == 1 and r.openbc == 1
    assert [list(t) for t in p.openbc_type] == [[1, 2], [0, 0], [0, 0]]
    assert p.openbc_press[0][0] == 0.01 and p.openbc_press[0][1] == 0.0
    assert p.openbc_vel[1][1][0] == 0.05 and list(p.openbc_vel[2][0]) == [0.0, 0.0, 0.5]
    assert p.openbc_vel[2][1][2] == -0.25


def test_namelist_reader_reads_repulsive_parameters(tmp_path):
    """A_rep, cosOppT and q_th of the &fluid namelist (LBFAST.f90:57-58)."""
    base = open(os.path.join(ROOT, "tests", "golden", "channel.inp")).read()
    text = base.replace("&fluid", "&fluid\n   A_rep=0.05d0\n   cosOppT=-0.8\n   q_th=0.125", 1)
    f = tmp_path / "rep.inp"
    f.write_text(text)
    rc, p, _ = read_nml(f)
    assert rc == 0 and (p.a_rep, p.cos_opp_t, p.q_th) == (0.05, -0.8, 0.125)


def test_namelist_reader_reads_reference_inputs():
    """Every *.inp file of the LBFAST sources, when their directory is given
    in LBFAST_REFERENCE_DIR."""
    ref = os.environ.get("LBFAST_REFERENCE_DIR", "")
    files = sorted(f for f in os.listdir(ref) if f.endswith(".inp")) if ref and os.path.isdir(ref) else []
    if not files:
        pytest.skip("LBFAST_REFERENCE_DIR does not name a directory of LBFAST .inp files")
    for f in files:
        rc, p, r = read_nml(os.path.join(ref, f))
        assert rc == 0, f
        assert p.lx > 0 and r.nsteps > 0


def test_raw_xdmf_writer(tmp_path):
    lz, ly, lx = 3, 4, 5
    rho = np.arange(lx * ly * lz, dtype=np.float32).reshape(lz, ly, lx)
    vel = np.stack([rho, -rho, 2 * rho])
    capi.write_raw_xdmf(str(tmp_path), 7, rho, vel, rho + 1)
    names = sorted(os.listdir(tmp_path))
    assert names == ["out_press_000007.raw", "out_press_000007.xdmf", "out_rho_000007.raw", "out_rho_000007.xdmf",
                     "out_vel_000007.raw", "out_vel_000007.xdmf"]
    r = np.fromfile(tmp_path / "out_rho_000007.raw", dtype=np.float32)
    assert np.array_equal(r, rho.ravel())
    v = np.fromfile(tmp_path / "out_vel_000007.raw", dtype=np.float32).reshape(lz, ly, lx, 3)
    assert np.array_equal(v[..., 1], -rho)  # velprint(1:3,i,j,k): components innermost
    x = (tmp_path / "out_vel_000007.xdmf").read_text()
    assert 'Dimensions="3 4 5"' in x and 'Dimensions="3 4 5 3"' in x and "out_vel_000007.raw" in x


@pytest.mark.parametrize("bad", [dict(lattice=13), dict(highorder=1, lattice=19), dict(densratio=1),
                                 dict(lx=0), dict(storage="f8"), dict(visc1=-1.0), dict(openbc=1, pbc_x=0),
                                 dict(openbc=1, obstacles=1, pbc_y=0, ly=2), dict(bounce_back=1),
                                 dict(repulsive_flux=1)])
def test_create_rejects_invalid_parameters_before_device_work(bad):
    kw = dict(lx=8, ly=8, lz=8, lattice=27)
    kw.update(bad)
    if kw.get("storage") == "f8":
        p = capi.Params(**{k: v for k, v in kw.items() if k != "storage"}).to_c()
        p.storage = 9
    else:
        p = capi.Params(**kw).to_c()
    h = C.c_void_p()
    rc = capi.load().lbf_create(C.byref(p), C.byref(h))
    assert rc in (-1, -5) and not h
    assert capi.last_error()


@pytest.mark.parametrize("two", [True, False])
def test_restart_file_layout_and_round_trip(tmp_path, two):
    """restart.raw as print_module.f90:1474-1677 writes it: float32 moments in
    the reference's hfields order 1,2,3,4,5,8,9,6,10,7, phi (two components),
    then iframe and iframe2D; the reader restores the header's order."""
    lx, ly, lz = 6, 5, 4
    rng = np.random.default_rng(3)
    m = rng.standard_normal((10, lz, ly, lx)).astype(np.float32)
    phi = rng.random((lz, ly, lx)).astype(np.float32) if two else None
    L.write_restart_raw(str(tmp_path), m, phi, 17, 3)
    raw = np.fromfile(tmp_path / "restart.raw", dtype=np.uint8)
    n = lx * ly * lz
    assert raw.size == 4 * n * (11 if two else 10) + 8
    f = raw[: 4 * n * (11 if two else 10)].view(np.float32).reshape(-1, lz, ly, lx)
    assert np.array_equal(f[:10], m[[0, 1, 2, 3, 4, 7, 8, 5, 9, 6]])
    if two:
        assert np.array_equal(f[10], phi)
    assert list(raw[-8:].view(np.int32)) == [17, 3]
    m2, p2, fr, fr2 = L.read_restart_raw(str(tmp_path), lx, ly, lz, two)
    assert np.array_equal(m2, m) and (fr, fr2) == (17, 3)
    if two:
        assert np.array_equal(p2, phi)
    with pytest.raises(L.LbfError):  # size check: a one-component file is not a two-component restart
        L.read_restart_raw(str(tmp_path), lx, ly, lz, not two)


def test_vtk_files_in_the_reference_layout(tmp_path):
    """print_vtk_sync (print_module.f90:22-244, 2789-2814): fixed-width XML
    header of 435 bytes ending in '_', int32 byte count, float32 data (vectors
    interleaved per node), 30-byte footer; names out_<var>_NNNNNN.vti."""
    lx, ly, lz = 36, 20, 7
    rng = np.random.default_rng(5)
    rho = rng.random((lz, ly, lx)).astype(np.float32)
    vel = rng.standard_normal((3, lz, ly, lx)).astype(np.float32)
    L.write_vtk(str(tmp_path), 12, rho, vel)
    ext = "     1     36      1     20      1      7"
    for var, data, nc in (("rho", rho, 1), ("vel", np.moveaxis(vel, 0, -1), 3)):
        b = (tmp_path / f"out_{var}_000012.vti").read_bytes()
        lines = ['<?xml version="1.0"?>',
                 '<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian">',
                 f'  <ImageData WholeExtent="{ext}">', f'    <Piece Extent="{ext}">', "      <PointData>",
                 f'        <DataArray type="Float32" Name="{var:<8s}" NumberOfComponents="{nc}" '
                 f'format="appended" offset="{0:>12d}"/>',
                 "      </PointData>", "    </Piece>", "  </ImageData>", '  <AppendedData encoding="raw">']
        widths = [22, 67, 70, 63, 18, 115, 19, 13, 15, 32]
        head = "".join(s.ljust(w - 1) + "\n" for s, w in zip(lines, widths)) + "_"
        assert len(head) == 435
        assert b[:435] == head.encode()
        n = lx * ly * lz * nc * 4
        assert np.frombuffer(b[435:439], np.int32)[0] == n
        assert np.array_equal(np.frombuffer(b[439:439 + n], np.float32), data.reshape(-1))
        assert b[439 + n:] == b"\n  </AppendedData>\n</VTKFile>\n"
    assert not (tmp_path / "out_press_000012.vti").exists()


def test_printhalf_files_in_the_reference_layout(tmp_path):
    """PRINTHALF (vars_module.f90:184-188, print_module.f90:110-121 and
    2053-2164): the print values rounded to IEEE binary16, written as their
    bit patterns; the VTK DataArray says UnsignedShort (a 121-byte header
    line, so a 441-byte header), the XDMF NumberType="UInt" Precision="2".
    Values include subnormals, overflow and exact halfway cases, which must
    round to nearest even as numpy's float16 does."""
    lx, ly, lz = 12, 5, 3
    rng = np.random.default_rng(9)
    rho = rng.standard_normal((lz, ly, lx)).astype(np.float32)
    special = np.array([0.0, -0.0, 1e-8, 3e-5, 6.1e-5, 65504.0, 65520.0, 1e6, -1e6, 1.0 + 2.0 ** -11,
                        1.0 + 3 * 2.0 ** -11, 2.0 ** -24, 2.0 ** -25, 1.5 * 2.0 ** -25, np.inf, -np.inf],
                       dtype=np.float32)
    rho.reshape(-1)[:special.size] = special
    vel = rng.standard_normal((3, lz, ly, lx)).astype(np.float32) * 1e-3
    L.write_vtk(str(tmp_path), 3, rho, vel, half=True)
    b = (tmp_path / "out_rho_000003.vti").read_bytes()
    line = (f'        <DataArray type="UnsignedShort" Name="{"rho":<8s}" NumberOfComponents="1" '
            f'format="appended" offset="{0:>12d}"/>')
    assert len(line) == 120
    assert b[:441].decode().endswith('  <AppendedData encoding="raw">\n_')
    assert line.encode() in b[:441]
    n = lx * ly * lz * 2
    assert np.frombuffer(b[441:445], np.int32)[0] == n
    with np.errstate(over="ignore"):  # 1e6 overflows to infinity, as intended
        want = rho.reshape(-1).astype(np.float16).view(np.uint16)
    assert np.array_equal(np.frombuffer(b[445:445 + n], np.uint16), want)
    assert len(b) == 445 + n + 30
    L.write_raw_xdmf(str(tmp_path), 4, rho, vel, half=True)
    r = np.fromfile(tmp_path / "out_rho_000004.raw", dtype=np.uint16)
    assert np.array_equal(r, want)
    v = np.fromfile(tmp_path / "out_vel_000004.raw", dtype=np.uint16).reshape(lz, ly, lx, 3)
    assert np.array_equal(v, np.moveaxis(vel, 0, -1).astype(np.float16).view(np.uint16))
    x = (tmp_path / "out_vel_000004.xdmf").read_text()
    assert 'NumberType="UInt" Precision="2" Dimensions="3 5 12 3"' in x


def test_first_extrema_of_a_damped_oscillation():
    """statistics.first_extrema: the first cycle of a damped cosine sampled
    every 20 steps, followed by small wiggles that would add local maxima."""
    from lbfast_b200 import statistics as ST
    T, tau = 2200.0, 6000.0
    t = np.arange(0, 8000, 20, dtype=np.float64)
    d = 20.3 + 0.9 * np.exp(-t / tau) * np.cos(2 * np.pi * t / T) + 0.05 * np.sin(2 * np.pi * t / 230.0) * (t > 4000)
    ex = ST.first_extrema(t, d, 3)
    assert [k for _, _, k in ex] == ["min", "max", "min"]
    # a damped cosine's extrema sit slightly before the undamped ones
    assert abs(ex[0][0] - T / 2) < 40 and abs(ex[1][0] - T) < 40 and abs(ex[2][0] - 1.5 * T) < 40, ex
    assert abs((ex[2][0] - ex[0][0]) - T) < 10, ex
    assert ex[2][1] > ex[0][1]
