"""ctypes binding of the C ABI in include/lbfast_gpu.h.

This is the Python-side stand-in for the Fortran ``bind(C)`` interface a
reference driver would use: every call goes through the
same exported C symbols.  The shared library is the in-tree build
``lbfast_b200/_lib/liblbfast_b200.so``; there is no fallback -- if it is
missing or fails to load, importing the solver raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field, fields

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "liblbfast_b200.so")

LBF_OK = 0
LBF_E_ARG, LBF_E_CUDA, LBF_E_NOMEM, LBF_E_STATE, LBF_E_UNSUPPORTED, LBF_E_IO, LBF_E_NUMERIC = -1, -2, -3, -4, -5, -6, -7
STORE = {"f32": 0, "f16": 1, "bf16": 2, "f64": 3}
LBF_F32, LBF_F64 = 0, 1

EXPORTED = (
    "lbf_version", "lbf_last_error", "lbf_create", "lbf_destroy", "lbf_set_stream", "lbf_set_isfluid",
    "lbf_set_fields", "lbf_step", "lbf_sync", "lbf_get_step", "lbf_get_fields", "lbf_get_print_fields",
    "lbf_reduce", "lbf_mark_isfluid", "lbf_seed_solid_phi", "lbf_ic_taylor_green", "lbf_ic_droplet", "lbf_ic_lamb",
    "lbf_write_raw_xdmf", "lbf_server_create", "lbf_server_destroy", "lbf_server_submit", "lbf_server_run",
    "lbf_server_poll", "lbf_server_fetch", "lbf_server_cancel", "lbf_get_tuning", "lbf_write_restart_raw",
    "lbf_read_restart_raw", "lbf_write_vtk", "lbf_write_vtk_half", "lbf_write_raw_xdmf_half",
    "lbf_write_checkpoint", "lbf_read_checkpoint", "lbf_create_slab", "lbf_slab_nregions", "lbf_slab_region",
    "lbf_slabs_exchange", "lbf_slabs_step",
)
SOLVE_STATE = {0: "queued", 1: "active", 2: "done", 3: "failed", 4: "cancelled"}


class LbfParams(C.Structure):
    _fields_ = [
        ("lx", C.c_int), ("ly", C.c_int), ("lz", C.c_int),
        ("pbc_x", C.c_int), ("pbc_y", C.c_int), ("pbc_z", C.c_int),
        ("lattice", C.c_int), ("highorder", C.c_int), ("twocomponent", C.c_int),
        ("densratio", C.c_int), ("obstacles", C.c_int), ("storage", C.c_int),
        ("visc1", C.c_double), ("visc2", C.c_double), ("rho_r", C.c_double), ("rho_b", C.c_double),
        ("sigma", C.c_double), ("width", C.c_double), ("tau_diff", C.c_double),
        ("fx", C.c_double), ("fy", C.c_double), ("fz", C.c_double), ("wettab_r", C.c_double),
        ("printphi", C.c_int), ("zseg", C.c_int), ("tile_y", C.c_int), ("phi_correction", C.c_int),
        ("smagorinsky", C.c_int), ("openbc", C.c_int), ("openbc_type", (C.c_int * 2) * 3),
        ("openbc_press", (C.c_double * 2) * 3), ("openbc_vel", ((C.c_double * 3) * 2) * 3),
        ("bounce_back", C.c_int), ("repulsive_flux", C.c_int), ("a_rep", C.c_double), ("cos_opp_t", C.c_double),
        ("q_th", C.c_double),
    ]


class LbfServerConfig(C.Structure):
    _fields_ = [("mem_budget", C.c_longlong), ("max_active", C.c_int), ("chunk", C.c_int), ("use_graph", C.c_int)]


class LbfSolveInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("steps_done", C.c_longlong), ("nsteps", C.c_longlong),
                ("device_bytes", C.c_longlong), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double)]


class LbfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m lbfast_b200.build` (or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp, dp, fp, i8p = C.c_void_p, P(C.c_double), P(C.c_float), P(C.c_int8)
    lib.lbf_version.restype = C.c_char_p
    lib.lbf_last_error.argtypes = [C.c_char_p, C.c_size_t]
    lib.lbf_create.argtypes = [P(LbfParams), P(vp)]
    lib.lbf_destroy.argtypes = [vp]
    lib.lbf_set_stream.argtypes = [vp, vp]
    lib.lbf_set_isfluid.argtypes = [vp, i8p]
    lib.lbf_set_fields.argtypes = [vp, vp, vp, C.c_int]
    lib.lbf_step.argtypes = [vp, C.c_int]
    lib.lbf_sync.argtypes = [vp]
    lib.lbf_get_step.argtypes = [vp, P(C.c_longlong)]
    lib.lbf_get_fields.argtypes = [vp, vp, vp, vp, C.c_int]
    lib.lbf_get_tuning.argtypes = [vp, P(C.c_int), P(C.c_int)]
    lib.lbf_get_print_fields.argtypes = [vp, fp, fp, fp]
    lib.lbf_reduce.argtypes = [vp, dp]
    lib.lbf_create_slab.argtypes = [P(LbfParams), C.c_int, C.c_int, P(vp)]
    lib.lbf_slab_nregions.argtypes = [vp, P(C.c_int)]
    lib.lbf_slab_region.argtypes = [vp, C.c_int, C.c_int, C.c_int, P(vp), P(C.c_size_t)]
    lib.lbf_slabs_exchange.argtypes = [P(vp), C.c_int]
    lib.lbf_slabs_step.argtypes = [P(vp), C.c_int, C.c_int]
    lib.lbf_write_checkpoint.argtypes = [vp, C.c_char_p]
    lib.lbf_read_checkpoint.argtypes = [vp, C.c_char_p]
    lib.lbf_mark_isfluid.argtypes = [C.c_int] * 8 + [i8p, i8p]
    lib.lbf_seed_solid_phi.argtypes = [C.c_int] * 4 + [i8p, dp]
    lib.lbf_ic_taylor_green.argtypes = [C.c_int] * 3 + [C.c_double, dp]
    lib.lbf_ic_droplet.argtypes = [C.c_int] * 3 + [dp] + [C.c_double] * 5 + [C.c_int, i8p, dp, dp]
    lib.lbf_ic_lamb.argtypes = [C.c_int] * 3 + [dp] + [C.c_double] * 5 + [C.c_int, i8p, dp, dp]
    lib.lbf_write_raw_xdmf.argtypes = [C.c_char_p] + [C.c_int] * 4 + [fp, fp, fp]
    lib.lbf_write_vtk.argtypes = [C.c_char_p] + [C.c_int] * 4 + [fp, fp, fp]
    lib.lbf_write_raw_xdmf_half.argtypes = [C.c_char_p] + [C.c_int] * 4 + [fp, fp, fp]
    lib.lbf_write_vtk_half.argtypes = [C.c_char_p] + [C.c_int] * 4 + [fp, fp, fp]
    lib.lbf_write_restart_raw.argtypes = [C.c_char_p] + [C.c_int] * 3 + [fp, fp, C.c_int, C.c_int]
    lib.lbf_read_restart_raw.argtypes = [C.c_char_p] + [C.c_int] * 3 + [fp, fp, P(C.c_int), P(C.c_int)]
    lib.lbf_server_create.argtypes = [P(LbfServerConfig), P(vp)]
    lib.lbf_server_destroy.argtypes = [vp]
    lib.lbf_server_submit.argtypes = [vp, P(LbfParams), i8p, vp, vp, C.c_int, C.c_longlong, P(C.c_longlong)]
    lib.lbf_server_run.argtypes = [vp, C.c_int, P(C.c_int), P(C.c_int)]
    lib.lbf_server_poll.argtypes = [vp, C.c_longlong, P(LbfSolveInfo)]
    lib.lbf_server_fetch.argtypes = [vp, C.c_longlong, vp, vp]
    lib.lbf_server_cancel.argtypes = [vp, C.c_longlong]
    lib.lbf_server_solve_bytes.argtypes = [P(LbfParams)]
    lib.lbf_server_solve_bytes.restype = C.c_longlong
    for name in EXPORTED:
        getattr(lib, name).restype = C.c_int if name != "lbf_version" else C.c_char_p
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().lbf_last_error(buf, 1024)
    return buf.value.decode()


def check(rc: int) -> None:
    if rc != LBF_OK:
        raise LbfError(rc, last_error())


def _ptr(a: np.ndarray | None, ctype=C.c_void_p):
    if a is None:
        return None
    if ctype is C.c_void_p:
        return C.c_void_p(a.ctypes.data)
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class Params:
    """Run parameters (the reference's macros + `simulation`/`fluid` namelists)."""
    lx: int
    ly: int
    lz: int
    pbc_x: int = 1
    pbc_y: int = 1
    pbc_z: int = 1
    lattice: int = 27
    highorder: int = 0
    twocomponent: int = 0
    densratio: int = 0
    obstacles: int = 0
    storage: str = "f32"
    visc1: float = 0.1
    visc2: float = 0.1
    rho_r: float = 1.0
    rho_b: float = 1.0
    sigma: float = 0.0
    width: float = 4.0
    tau_diff: float = 0.1
    fx: float = 0.0
    fy: float = 0.0
    fz: float = 0.0
    wettab_r: float = 90.0
    printphi: int = 0
    zseg: int = 0
    tile_y: int = 0
    phi_correction: int = 0
    smagorinsky: int = 0
    # open faces on the non-periodic axes (requires obstacles); per axis
    # (x, y, z) and side (low, high): type 2 zero gradient, 1 pressure, other
    # velocity; pressure moment P; velocity (u, v, w)
    openbc: int = 0
    openbc_type: tuple = ((0, 0), (0, 0), (0, 0))
    openbc_press: tuple = ((0.0, 0.0), (0.0, 0.0), (0.0, 0.0))
    openbc_vel: tuple = (((0.0,) * 3,) * 2,) * 3
    bounce_back: int = 0  # half-way bounce-back at obstacles (BOUNCE_BACK)
    repulsive_flux: int = 0  # film repulsion between facing interfaces (REPULSIVE_FLUX)
    a_rep: float = 0.0
    cos_opp_t: float = 0.0
    q_th: float = 0.0

    def to_c(self) -> LbfParams:
        p = LbfParams()
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "storage":
                v = STORE[v]
            if f.name.startswith("openbc_"):
                arr = getattr(p, f.name)
                for a in range(3):
                    for sd in range(2):
                        if f.name == "openbc_vel":
                            for d in range(3):
                                arr[a][sd][d] = float(v[a][sd][d])
                        else:
                            arr[a][sd] = v[a][sd]
                continue
            setattr(p, f.name, v)
        return p

    def oracle_dict(self) -> dict:
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        d["twocomp"] = d.pop("twocomponent")
        return d

    @property
    def shape(self):
        return (self.lz, self.ly, self.lx)


class Solver:
    """One box on the current CUDA device, driven through the C ABI.

    Arrays are numpy (lz, ly, lx) views of Fortran-order fields; moments are
    (10, lz, ly, lx) in the order P, u, v, w, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz.
    """

    def __init__(self, params: Params):
        self.lib = load()
        self.params = params
        self.h = C.c_void_p()
        check(self.lib.lbf_create(C.byref(params.to_c()), C.byref(self.h)))
        self.shape = params.shape

    def close(self) -> None:
        if self.h:
            check(self.lib.lbf_destroy(self.h))
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_ptr: int) -> None:
        check(self.lib.lbf_set_stream(self.h, C.c_void_p(stream_ptr)))

    def set_isfluid(self, isf: np.ndarray) -> None:
        a = np.ascontiguousarray(isf, dtype=np.int8).reshape(self.shape)
        check(self.lib.lbf_set_isfluid(self.h, _ptr(a, C.c_int8)))

    def set_fields(self, mom10: np.ndarray, phi: np.ndarray | None = None) -> None:
        dt = LBF_F64 if mom10.dtype == np.float64 else LBF_F32
        npdt = np.float64 if dt == LBF_F64 else np.float32
        m = np.ascontiguousarray(mom10, dtype=npdt).reshape((10,) + self.shape)
        p = None if phi is None else np.ascontiguousarray(phi, dtype=npdt).reshape(self.shape)
        check(self.lib.lbf_set_fields(self.h, _ptr(m), _ptr(p), dt))

    def step(self, n: int = 1) -> None:
        check(self.lib.lbf_step(self.h, int(n)))

    def sync(self) -> None:
        check(self.lib.lbf_sync(self.h))

    @property
    def nstep(self) -> int:
        s = C.c_longlong()
        check(self.lib.lbf_get_step(self.h, C.byref(s)))
        return s.value

    @property
    def tuning(self) -> tuple[int, int]:
        """(tile rows, z segment) of the step kernel in use."""
        ty, zs = C.c_int(), C.c_int()
        check(self.lib.lbf_get_tuning(self.h, C.byref(ty), C.byref(zs)))
        return ty.value, zs.value

    def get_fields(self, dtype=np.float64):
        dt = LBF_F64 if dtype == np.float64 else LBF_F32
        m = np.empty((10,) + self.shape, dtype=dtype)
        p = np.empty(self.shape, dtype=dtype) if self.params.twocomponent else None
        u = np.empty((3,) + self.shape, dtype=dtype)
        check(self.lib.lbf_get_fields(self.h, _ptr(m), _ptr(p), _ptr(u), dt))
        return m, p, u

    def get_print(self):
        """copy_print fields: rho (lz,ly,lx), vel (3,lz,ly,lx), press (lz,ly,lx), float32."""
        rho = np.empty(self.shape, dtype=np.float32)
        vel = np.empty(self.shape + (3,), dtype=np.float32)
        press = np.empty(self.shape, dtype=np.float32)
        check(self.lib.lbf_get_print_fields(self.h, _ptr(rho, C.c_float), _ptr(vel, C.c_float),
                                            _ptr(press, C.c_float)))
        return rho, np.moveaxis(vel, -1, 0), press

    def write_checkpoint(self, path: str) -> None:
        """Full state of the run (both time levels in the storage precision),
        from which read_checkpoint resumes it bit for bit."""
        check(self.lib.lbf_write_checkpoint(self.h, str(path).encode()))

    def read_checkpoint(self, path: str) -> None:
        """Resume from write_checkpoint's file (same parameters; with obstacles
        call set_isfluid first)."""
        check(self.lib.lbf_read_checkpoint(self.h, str(path).encode()))

    def reduce(self) -> np.ndarray:
        out = np.zeros(5, dtype=np.float64)
        check(self.lib.lbf_reduce(self.h, _ptr(out, C.c_double)))
        return out


class Server:
    """Batched solve server (lbf_server_* of the C ABI): solves of uneven box
    sizes are submitted as they arrive, admitted first in, first out against a
    device-memory budget, and advanced together, one kernel launch per time
    step for all resident solves of a kernel class, in CUDA-graph chunks."""

    def __init__(self, mem_budget: int = 0, max_active: int = 0, chunk: int = 32, use_graph: bool = True):
        self.lib = load()
        cfg = LbfServerConfig(int(mem_budget), int(max_active), int(chunk), int(bool(use_graph)))
        self.s = C.c_void_p()
        check(self.lib.lbf_server_create(C.byref(cfg), C.byref(self.s)))
        self._meta: dict[int, tuple] = {}

    def close(self) -> None:
        if self.s:
            check(self.lib.lbf_server_destroy(self.s))
            self.s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def solve_bytes(params: Params) -> int:
        return int(load().lbf_server_solve_bytes(C.byref(params.to_c())))

    def submit(self, params: Params, mom10: np.ndarray, phi: np.ndarray | None = None, nsteps: int = 1,
               isf: np.ndarray | None = None) -> int:
        dt = LBF_F64 if mom10.dtype == np.float64 else LBF_F32
        npdt = np.float64 if dt == LBF_F64 else np.float32
        shape = params.shape
        m = np.ascontiguousarray(mom10, dtype=npdt).reshape((10,) + shape)
        p = None if phi is None else np.ascontiguousarray(phi, dtype=npdt).reshape(shape)
        i = None if isf is None else np.ascontiguousarray(isf, dtype=np.int8).reshape(shape)
        sid = C.c_longlong()
        check(self.lib.lbf_server_submit(self.s, C.byref(params.to_c()), _ptr(i, C.c_int8), _ptr(m), _ptr(p), dt,
                                         int(nsteps), C.byref(sid)))
        self._meta[sid.value] = (shape, npdt, bool(params.twocomponent))
        return sid.value

    def run(self, max_chunks: int = 1) -> tuple[int, int]:
        """Advance up to max_chunks chunks; returns (resident, queued) solves."""
        a, q = C.c_int(), C.c_int()
        check(self.lib.lbf_server_run(self.s, int(max_chunks), C.byref(a), C.byref(q)))
        return a.value, q.value

    def drain(self) -> None:
        while self.run(1 << 20) != (0, 0):
            pass

    def poll(self, sid: int) -> dict:
        info = LbfSolveInfo()
        check(self.lib.lbf_server_poll(self.s, int(sid), C.byref(info)))
        return {"state": SOLVE_STATE[info.state], "steps_done": info.steps_done, "nsteps": info.nsteps,
                "device_bytes": info.device_bytes, "t_submit": info.t_submit, "t_admit": info.t_admit,
                "t_done": info.t_done}

    def fetch(self, sid: int):
        """(mom10, phi) of a finished solve in the dtype it was submitted with."""
        shape, npdt, tc = self._meta[sid]
        m = np.empty((10,) + shape, dtype=npdt)
        p = np.empty(shape, dtype=npdt) if tc else None
        check(self.lib.lbf_server_fetch(self.s, int(sid), _ptr(m), _ptr(p)))
        del self._meta[sid]
        return m, p

    def cancel(self, sid: int) -> None:
        check(self.lib.lbf_server_cancel(self.s, int(sid)))
        self._meta.pop(sid, None)


# ---- host-side set-up helpers (C++ behind the C ABI) ----

def mark_isfluid(raw: np.ndarray, pbc=(1, 1, 1), lattice: int = 27, obstacles: bool = True) -> np.ndarray:
    lib = load()
    lz, ly, lx = raw.shape
    r = np.ascontiguousarray(raw, dtype=np.int8)
    out = np.empty_like(r)
    check(lib.lbf_mark_isfluid(lx, ly, lz, int(pbc[0]), int(pbc[1]), int(pbc[2]), int(lattice), int(obstacles),
                               _ptr(r, C.c_int8), _ptr(out, C.c_int8)))
    return out


def seed_solid_phi(phi: np.ndarray, isf: np.ndarray, lattice: int = 27) -> np.ndarray:
    lib = load()
    lz, ly, lx = phi.shape
    p = np.ascontiguousarray(phi, dtype=np.float64).copy()
    i = np.ascontiguousarray(isf, dtype=np.int8)
    check(lib.lbf_seed_solid_phi(lx, ly, lz, int(lattice), _ptr(i, C.c_int8), _ptr(p, C.c_double)))
    return p


def ic_taylor_green(lx: int, ly: int, lz: int, u0: float) -> np.ndarray:
    m = np.empty((10, lz, ly, lx), dtype=np.float64)
    check(load().lbf_ic_taylor_green(lx, ly, lz, float(u0), _ptr(m, C.c_double)))
    return m


def ic_droplet(lx, ly, lz, center, radius, width, sigma, rho_r, rho_b, densratio=True, isf=None):
    m = np.empty((10, lz, ly, lx), dtype=np.float64)
    phi = np.empty((lz, ly, lx), dtype=np.float64)
    c = np.ascontiguousarray(center, dtype=np.float64)
    i = None if isf is None else np.ascontiguousarray(isf, dtype=np.int8)
    check(load().lbf_ic_droplet(lx, ly, lz, _ptr(c, C.c_double), float(radius), float(width), float(sigma),
                                float(rho_r), float(rho_b), int(densratio), _ptr(i, C.c_int8),
                                _ptr(m, C.c_double), _ptr(phi, C.c_double)))
    return m, phi


def ic_lamb(lx, ly, lz, center, radius, width, sigma, rho_r, rho_b, densratio=True, isf=None):
    """LAMBTEST initial droplet: as ic_droplet with the x distance halved."""
    m = np.empty((10, lz, ly, lx), dtype=np.float64)
    phi = np.empty((lz, ly, lx), dtype=np.float64)
    c = np.ascontiguousarray(center, dtype=np.float64)
    i = None if isf is None else np.ascontiguousarray(isf, dtype=np.int8)
    check(load().lbf_ic_lamb(lx, ly, lz, _ptr(c, C.c_double), float(radius), float(width), float(sigma),
                             float(rho_r), float(rho_b), int(densratio), _ptr(i, C.c_int8), _ptr(m, C.c_double),
                             _ptr(phi, C.c_double)))
    return m, phi


def write_restart_raw(directory: str, mom10: np.ndarray, phi: np.ndarray | None = None, iframe: int = 0,
                      iframe2D: int = 0) -> None:
    """The reference's restart.raw (float32, one time level) in `directory`."""
    _, lz, ly, lx = mom10.shape
    m = np.ascontiguousarray(mom10, dtype=np.float32)
    p = None if phi is None else np.ascontiguousarray(phi, dtype=np.float32)
    check(load().lbf_write_restart_raw(directory.encode(), lx, ly, lz, _ptr(m, C.c_float), _ptr(p, C.c_float),
                                       int(iframe), int(iframe2D)))


def read_restart_raw(directory: str, lx: int, ly: int, lz: int, twocomponent: bool):
    """(mom10, phi or None, iframe, iframe2D) from `directory`/restart.raw."""
    m = np.empty((10, lz, ly, lx), dtype=np.float32)
    p = np.empty((lz, ly, lx), dtype=np.float32) if twocomponent else None
    fr, fr2 = C.c_int(), C.c_int()
    check(load().lbf_read_restart_raw(directory.encode(), lx, ly, lz, _ptr(m, C.c_float), _ptr(p, C.c_float),
                                      C.byref(fr), C.byref(fr2)))
    return m, p, fr.value, fr2.value


def write_vtk(directory: str, iframe: int, rho, vel, press=None, half: bool = False) -> None:
    """VTK ImageData files of the reference's print_vtk_sync (half: its
    PRINTHALF layout, binary16 values)."""
    lz, ly, lx = rho.shape
    r = np.ascontiguousarray(rho, dtype=np.float32)
    v = np.ascontiguousarray(np.moveaxis(vel, 0, -1), dtype=np.float32)
    p = None if press is None else np.ascontiguousarray(press, dtype=np.float32)
    f = load().lbf_write_vtk_half if half else load().lbf_write_vtk
    check(f(directory.encode(), int(iframe), lx, ly, lz, _ptr(r, C.c_float), _ptr(v, C.c_float), _ptr(p, C.c_float)))


def write_raw_xdmf(directory: str, iframe: int, rho, vel, press=None, half: bool = False) -> None:
    """raw + XDMF files of the reference's print_raw_sync (half: PRINTHALF)."""
    lz, ly, lx = rho.shape
    r = np.ascontiguousarray(rho, dtype=np.float32)
    v = np.ascontiguousarray(np.moveaxis(vel, 0, -1), dtype=np.float32)
    p = None if press is None else np.ascontiguousarray(press, dtype=np.float32)
    f = load().lbf_write_raw_xdmf_half if half else load().lbf_write_raw_xdmf
    check(f(directory.encode(), int(iframe), lx, ly, lz, _ptr(r, C.c_float), _ptr(v, C.c_float), _ptr(p, C.c_float)))
