"""ctypes front end of the CPU oracle (test infrastructure only).

Loaded by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` -- never by the product.  The numerics live in lbf_oracle.c,
whose header states what of the reference it restates and its parity status
(unpinned against a reference binary; pinned against the reference's
analytic checks and its Minv_mrt table).

Also holds numpy restatements of the reference's isfluid marking
(LBFAST.f90:258-325) and initial conditions (init_conditions_module.f90),
so that the host-side implementations in the product can be checked.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")


class OrcParams(C.Structure):
    _fields_ = [
        ("lx", C.c_int), ("ly", C.c_int), ("lz", C.c_int),
        ("pbc_x", C.c_int), ("pbc_y", C.c_int), ("pbc_z", C.c_int),
        ("lattice", C.c_int), ("highorder", C.c_int), ("twocomp", C.c_int),
        ("densratio", C.c_int), ("obstacles", C.c_int),
        ("visc1", C.c_double), ("visc2", C.c_double), ("rho_r", C.c_double),
        ("rho_b", C.c_double), ("sigma", C.c_double), ("width", C.c_double),
        ("tau_diff", C.c_double), ("fx", C.c_double), ("fy", C.c_double),
        ("fz", C.c_double), ("wettab_r", C.c_double), ("phi_correction", C.c_int), ("smagorinsky", C.c_int),
        ("openbc", C.c_int), ("obc_type", (C.c_int * 2) * 3), ("obc_press", (C.c_double * 2) * 3),
        ("obc_vel", ((C.c_double * 3) * 2) * 3), ("bounce_back", C.c_int),
        ("repulsive", C.c_int), ("a_rep", C.c_double), ("cos_opp_t", C.c_double), ("q_th", C.c_double),
    ]


_libs: dict[str, C.CDLL] = {}


def build() -> None:
    """Compile the oracle shared libraries (oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(prec: str) -> C.CDLL:
    if prec not in ("f64", "f32"):
        raise ValueError(prec)
    if prec not in _libs:
        path = os.path.join(_BUILD, f"liblbf_oracle_{prec}.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        P = C.POINTER
        dp = P(C.c_double)
        lib.orc_create.argtypes = [P(OrcParams)]
        lib.orc_create.restype = C.c_void_p
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_set_isfluid.argtypes = [C.c_void_p, P(C.c_int8)]
        lib.orc_set_fields.argtypes = [C.c_void_p, dp, dp]
        lib.orc_step.argtypes = [C.c_void_p, C.c_int]
        lib.orc_get_fields.argtypes = [C.c_void_p, dp, dp, dp]
        lib.orc_get_phi_buffers.argtypes = [C.c_void_p, dp, dp]
        lib.orc_get_print.argtypes = [C.c_void_p, dp, dp, dp]
        lib.orc_get_step.argtypes = [C.c_void_p]
        lib.orc_get_step.restype = C.c_long
        lib.orc_set_threads.argtypes = [C.c_int]
        lib.orc_minv_table.argtypes = [dp]
        ip = C.POINTER(C.c_int)
        lib.orc_lattice_table.argtypes = [C.c_int, ip, ip, ip, ip, dp]
        lib.orc_lattice_table.restype = C.c_int
        _libs[prec] = lib
    return _libs[prec]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def minv_table() -> np.ndarray:
    out = np.zeros((27, 27), dtype=np.float64)
    _lib("f64").orc_minv_table(_dp(out))
    return out


def lattice_table(lattice: int) -> dict:
    """ex, ey, ez, opp, w of a lattice as the oracle builds them."""
    a = {k: np.zeros(27, dtype=np.int32) for k in ("ex", "ey", "ez", "opp")}
    w = np.zeros(27, dtype=np.float64)
    ip = lambda v: v.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
    n = _lib("f64").orc_lattice_table(int(lattice), ip(a["ex"]), ip(a["ey"]), ip(a["ez"]), ip(a["opp"]), _dp(w))
    out = {k: v[:n].tolist() for k, v in a.items()}
    out["w"] = w[:n].tolist()
    return out


def set_threads(n: int) -> None:
    for p in ("f64", "f32"):
        _lib(p).orc_set_threads(int(n))


PARAM_KEYS = ("lx", "ly", "lz", "pbc_x", "pbc_y", "pbc_z", "lattice", "highorder",
              "twocomp", "densratio", "obstacles", "visc1", "visc2", "rho_r", "rho_b",
              "sigma", "width", "tau_diff", "fx", "fy", "fz", "wettab_r", "phi_correction", "smagorinsky",
              "openbc")


class Oracle:
    """One simulation box on the CPU.  Arrays are (lz, ly, lx) numpy views of
    Fortran-order (i fastest) fields; moments are stacked as (10, lz, ly, lx)
    in the order P, u, v, w, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz."""

    def __init__(self, params: dict, prec: str = "f64"):
        self.lib = _lib(prec)
        p = OrcParams()
        for k in PARAM_KEYS:
            setattr(p, k, params.get(k, 0) if k not in ("rho_r", "rho_b") else params.get(k, 1.0))
        # open faces: openbc_type / openbc_press [axis][side], openbc_vel [axis][side][u, v, w]
        ty = params.get("openbc_type") or ((0, 0),) * 3
        pr = params.get("openbc_press") or ((0.0, 0.0),) * 3
        ve = params.get("openbc_vel") or (((0.0,) * 3,) * 2,) * 3
        p.bounce_back = int(params.get("bounce_back", 0))
        p.repulsive = int(params.get("repulsive_flux", 0))
        p.a_rep = float(params.get("a_rep", 0.0))
        p.cos_opp_t = float(params.get("cos_opp_t", 0.0))
        p.q_th = float(params.get("q_th", 0.0))
        for a in range(3):
            for sd in range(2):
                p.obc_type[a][sd] = int(ty[a][sd])
                p.obc_press[a][sd] = float(pr[a][sd])
                for d in range(3):
                    p.obc_vel[a][sd][d] = float(ve[a][sd][d])
        self.p = dict(params)
        self.shape = (int(params["lz"]), int(params["ly"]), int(params["lx"]))
        self.n = int(np.prod(self.shape))
        self.h = self.lib.orc_create(C.byref(p))
        if not self.h:
            raise MemoryError("orc_create failed")

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.orc_destroy(h)
            self.h = None

    def set_isfluid(self, isf: np.ndarray) -> None:
        a = np.ascontiguousarray(isf, dtype=np.int8).reshape(self.shape)
        self.lib.orc_set_isfluid(self.h, a.ctypes.data_as(C.POINTER(C.c_int8)))

    def set_fields(self, h10: np.ndarray, phi: np.ndarray | None = None) -> None:
        a = np.ascontiguousarray(h10, dtype=np.float64).reshape((10,) + self.shape)
        if phi is None:
            self.lib.orc_set_fields(self.h, _dp(a), None)
        else:
            b = np.ascontiguousarray(phi, dtype=np.float64).reshape(self.shape)
            self.lib.orc_set_fields(self.h, _dp(a), _dp(b))

    def step(self, n: int = 1) -> None:
        self.lib.orc_step(self.h, int(n))

    @property
    def nstep(self) -> int:
        return int(self.lib.orc_get_step(self.h))

    def get_fields(self):
        h10 = np.zeros((10,) + self.shape)
        phi = np.zeros(self.shape)
        uold = np.zeros((3,) + self.shape)
        self.lib.orc_get_fields(self.h, _dp(h10), _dp(phi), _dp(uold))
        return h10, phi, uold

    def get_phi_buffers(self):
        a = np.zeros(self.shape)
        b = np.zeros(self.shape)
        self.lib.orc_get_phi_buffers(self.h, _dp(a), _dp(b))
        return a, b

    def get_print(self):
        rho = np.zeros(self.shape)
        vel = np.zeros((3,) + self.shape)
        press = np.zeros(self.shape)
        self.lib.orc_get_print(self.h, _dp(rho), _dp(vel), _dp(press))
        return rho, vel, press


# ---------------------------------------------------------------------------
# Restatements of the reference's host-side set-up (checked against the
# product's C++ host code in tests/).
# ---------------------------------------------------------------------------

EX27 = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, 1, -1])
EY27 = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, -1, 1])
EZ27 = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1])


def lattice_links(lattice: int):
    """D3Q27 indices of the links of a lattice, in the reference's order:
    D3Q19 = 0-18 (vars_module.f90:666-684), D3Q15 = 0-6 and 19-26 (:685-703)."""
    if lattice == 27:
        return list(range(27))
    if lattice == 19:
        return list(range(19))
    return list(range(7)) + list(range(19, 27))


def mark_isfluid(solid: np.ndarray, pbc, lattice: int, obstacles: bool) -> np.ndarray:
    """LBFAST.f90:258-325.  ``solid`` (lz, ly, lx) bool marks nodes read from
    isfluid.raw as 0; returns int8 isfluid in {1, -1, 0}.  The halo is 1 in
    non-periodic directions and wrapped in periodic ones."""
    lz, ly, lx = solid.shape
    isf = np.where(solid, 0, 1).astype(np.int8)
    if obstacles:
        if not pbc[0]:
            isf[:, :, 0] = 0
            isf[:, :, lx - 1] = 0
        if not pbc[1]:
            isf[:, 0, :] = 0
            isf[:, ly - 1, :] = 0
        if not pbc[2]:
            isf[0, :, :] = 0
            isf[lz - 1, :, :] = 0
    pad = np.ones((lz + 2, ly + 2, lx + 2), dtype=np.int8)
    pad[1:-1, 1:-1, 1:-1] = isf
    # periodic halo: x, then y, then z (mpi_module.f90:646-710)
    if pbc[0]:
        pad[1:-1, 1:-1, 0] = pad[1:-1, 1:-1, lx]
        pad[1:-1, 1:-1, lx + 1] = pad[1:-1, 1:-1, 1]
    if pbc[1]:
        pad[1:-1, 0, :] = pad[1:-1, ly, :]
        pad[1:-1, ly + 1, :] = pad[1:-1, 1, :]
    if pbc[2]:
        pad[0, :, :] = pad[lz, :, :]
        pad[lz + 1, :, :] = pad[1, :, :]
    out = isf.copy()
    core = pad[1:-1, 1:-1, 1:-1]
    for l in lattice_links(lattice)[1:]:
        nb = pad[1 + EZ27[l]:1 + EZ27[l] + lz, 1 + EY27[l]:1 + EY27[l] + ly, 1 + EX27[l]:1 + EX27[l] + lx]
        out[(core == 1) & (np.abs(nb) != 1)] = -1
    return out


def fcut_tanh(r, rc, w):
    """vars_module.f90:1306-1329"""
    return 0.5 * (1.0 - np.tanh((r - rc) / (0.5 * w)))


def ic_taylor_green(lx, ly, lz, u0):
    """init_conditions_module.f90:298-314 (TAYLORGREEN, one component)."""
    gi = np.arange(1, lx + 1)[None, None, :]
    gj = np.arange(1, ly + 1)[None, :, None]
    gk = np.arange(1, lz + 1)[:, None, None]
    x = 2 * np.pi * (gi - 1) / lx
    y = 2 * np.pi * (gj - 1) / ly
    z = 2 * np.pi * (gk - 1) / lz
    u = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    v = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(u + v)
    press = ((u0 * u0 / 16.0) * (np.cos(2 * x) + np.cos(2 * y)) * (2 + np.cos(2 * z))) / (1.0 / 3.0)
    u, v, w, press = np.broadcast_arrays(u, v, w, press)
    h = np.stack([press, u, v, w, u * u, v * v, w * w, u * v, u * w, v * w]).astype(np.float64)
    return h


def ic_droplet(lx, ly, lz, center, radius, width, sigma, rho_r, rho_b, densratio=True):
    """init_conditions_module.f90:394-426 (default DOBENCHMARK branch: a
    droplet at rest with the Laplace pressure inside; nearest periodic image
    as pbc_images, :591-600)."""
    gi = np.arange(1, lx + 1, dtype=np.float64)[None, None, :]
    gj = np.arange(1, ly + 1, dtype=np.float64)[None, :, None]
    gk = np.arange(1, lz + 1, dtype=np.float64)[:, None, None]
    dx = gi - center[0]
    dy = gj - center[1]
    dz = gk - center[2]

    def nint(a):
        return np.where(a >= 0, np.floor(a + 0.5), -np.floor(-a + 0.5))

    dx = dx - lx * nint(dx / lx)
    dy = dy - ly * nint(dy / ly)
    dz = dz - lz * nint(dz / lz)
    r = np.sqrt(dx ** 2 + dy ** 2 + dz ** 2)
    phi = fcut_tanh(r, radius, width)
    rhophi = rho_r * phi + (1 - phi) * rho_b if densratio else np.ones_like(phi)
    press = phi * (sigma * 2.0) / radius / (rhophi * (1.0 / 3.0))
    z = np.zeros_like(phi)
    h = np.stack([press, z, z, z, z, z, z, z, z, z])
    return h, phi


def seed_solid_phi(phi: np.ndarray, isf: np.ndarray, lattice: int = 27) -> np.ndarray:
    """init_conditions_module.f90:492-541: phi at solid nodes = link-weighted
    mean of fluid neighbours inside the local box (no wrap).  A solid node with
    no fluid neighbour gets 0/0, i.e. NaN, exactly as the reference."""
    lz, ly, lx = phi.shape
    out = phi.copy()
    num = np.zeros_like(phi)
    den = np.zeros_like(phi)
    pad_phi = np.zeros((lz + 2, ly + 2, lx + 2))
    pad_phi[1:-1, 1:-1, 1:-1] = phi
    pad_isf = np.zeros((lz + 2, ly + 2, lx + 2), dtype=np.int8)  # outside the box: skipped
    pad_isf[1:-1, 1:-1, 1:-1] = isf
    inside = np.zeros((lz + 2, ly + 2, lx + 2), dtype=bool)
    inside[1:-1, 1:-1, 1:-1] = True
    for l in lattice_links(lattice)[1:]:
        d2 = EX27[l] ** 2 + EY27[l] ** 2 + EZ27[l] ** 2
        sc = 1.0 if d2 == 1 else (0.70710678118654752440 if d2 == 2 else 0.57735026918962576450)
        sl = (slice(1 + EZ27[l], 1 + EZ27[l] + lz), slice(1 + EY27[l], 1 + EY27[l] + ly),
              slice(1 + EX27[l], 1 + EX27[l] + lx))
        ok = inside[sl] & (pad_isf[sl] != 0)
        num += np.where(ok, sc * pad_phi[sl], 0.0)
        den += np.where(ok, sc, 0.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        out[isf == 0] = (num / den)[isf == 0]
    return out
