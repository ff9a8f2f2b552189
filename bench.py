"""Benchmark of the LBFAST time step on B200.

Workload (the reference's Laplace check, the configuration its headline
metric is quoted on that fits one GPU): two-component DENSRATIO D3Q27
HIGHORDER, 256^3 periodic, FP32, a centred droplet R=40 with the
fcut_tanh profile of width 3, density ratio 100 (rho_r = 100 in the droplet,
rho_b = 1 around it), sigma = 0.03, nu1 = nu2 = 0.1, tau_diff = 0.1, fluids at
rest.  Synthetic input generated in-process (no dataset exists for this
path).  The same ratio written as rho_r = 1, rho_b = 0.01 makes the scheme
unstable after ~3000 steps at this size, in FP64 as in FP32.

One "step" is one LB time step of the whole box.  The timed region covers
exactly --steps steps between barriers and device synchronisations, timed with
CUDA events on the launching stream (max over ranks).  The state (1.9 GB)
exceeds the 126 MB L2, so no flush is needed between steps.

Arms:
  default          this library, device-resident state ("value"), plus an
                   end-to-end run through the C ABI from pinned host buffers
                   ("e2e": initial state uploaded, steps, copy_print read back)
  --impl reference the reference's algorithm on the host cores: the C
                   restatement in oracle/ (the reference itself is CUDA
                   Fortran/OpenACC and cannot be built here), FP32, all host
                   threads, on a bounded number of steps of the same box.

Beside the headline the line carries "extra": device-resident MLUPS and
roofline of the other configurations the metric names -- FP16 storage on the
same box, the 512 x 256 x 256 channel with obstacles (FP32) and the 768^3
box of 200 seeded droplets (FP32 and FP16 storage) -- each timed the same
way on fewer steps.  "cpu_baseline" holds the oracle on the headline box
and, as "taylor_green", the 64^3 D3Q19 Taylor-Green case at its full 1000
steps.  Clocks are sampled by nvidia-smi over a window of steady stepping
that contains the timed steps (a second of steps before them, a fraction
after).

Multi-GPU (torchrun): every rank advances its own replica of the box (the
single-GPU path has no exchange step); "value" sums the ranks' lattice
updates over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS (D3Q27 high-order two-component lattice updates per second)"
UNIT = "MLUPS"
LBOX = 256
RHO_R, RHO_B = 100.0, 1.0
# algorithmic bytes per lattice update, two components with density ratio:
# 2 x (10 moments + 3 u_old + phi); 16-bit storage keeps P, u, v, w and phi in
# FP32 and Pi - u u and u_old in 16 bits: 2 x (4 x 4 + 6 x 2 + 3 x 2 + 4)
B_LUP = {"f32": 112, "f16": 76, "bf16": 76, "f64": 224}
# DRAM bytes (read + write) of one step launch of the tuned kernel, measured
# by ncu (dram__bytes_read.sum + dram__bytes_write.sum) at this workload
NCU_TRAFFIC = {("f32", 256): 1883155456}
# warp instructions of one step launch (ncu smsp__inst_executed.sum) at this
# workload: the issue ceiling is 4 warp instructions per SM cycle
NCU_WARP_INST = {("f32", 256): 705.10e6}


CHANNEL = (512, 256, 256)  # the two-component channel with obstacles (lx, ly, lz)


def _helpers(oracle_helpers: bool):
    """Set-up helpers (isfluid marking, solid phi seeding, the droplet initial
    condition): the library's, or the oracle's numpy restatements of the same
    reference routines -- the reference arm uses those, so it never loads the
    product library."""
    if oracle_helpers:
        from oracle import oracle as O
        return O.mark_isfluid, O.seed_solid_phi, O.ic_droplet
    import lbfast_b200 as lbf
    return lbf.mark_isfluid, lbf.seed_solid_phi, lbf.ic_droplet


def channel_geometry(lx=CHANNEL[0], ly=CHANNEL[1], lz=CHANNEL[2], oracle_helpers=False):
    """isfluid and phi of the channel: walls at y = 0 and ly-1 (pbc 1, 0, 1),
    64 seeded solid spheres of radius U[6, 14] kept clear of the periodic faces
    (seed 12345), phi from 32 seeded blobs of radius U[8, 24] with a width-4
    tanh profile (seed 67890), solid-node phi seeded from fluid neighbours."""
    import numpy as np

    mark_isfluid, seed_solid_phi, _ = _helpers(oracle_helpers)
    rng = np.random.default_rng(12345)
    solid = np.zeros((lz, ly, lx), dtype=bool)
    for _ in range(64):
        r = rng.uniform(6.0, 14.0)
        lo = r + 1.5
        c = [rng.uniform(lo, n - 1 - lo) for n in (lx, ly, lz)]
        z0, z1 = int(c[2] - r) - 1, int(c[2] + r) + 2
        y0, y1 = int(c[1] - r) - 1, int(c[1] + r) + 2
        x0, x1 = int(c[0] - r) - 1, int(c[0] + r) + 2
        z, y, x = np.ogrid[z0:z1, y0:y1, x0:x1]
        solid[z0:z1, y0:y1, x0:x1] |= (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r
    if oracle_helpers:
        isf = mark_isfluid(solid, (1, 0, 1), 27, True)
    else:
        isf = mark_isfluid(np.where(solid, 0, 1).astype(np.int8), (1, 0, 1), 27, True)
    rng = np.random.default_rng(67890)
    phi = np.zeros((lz, ly, lx))
    for _ in range(32):
        r = rng.uniform(8.0, 24.0)
        c = rng.uniform(0, 1, 3) * np.array([lx, ly, lz])
        h = int(r + 10)
        zi = (np.arange(int(c[2]) - h, int(c[2]) + h + 1)) % lz
        yi = np.clip(np.arange(int(c[1]) - h, int(c[1]) + h + 1), 0, ly - 1)
        xi = (np.arange(int(c[0]) - h, int(c[0]) + h + 1)) % lx
        dz = np.arange(int(c[2]) - h, int(c[2]) + h + 1)[:, None, None] - c[2]
        dy = np.arange(int(c[1]) - h, int(c[1]) + h + 1)[None, :, None] - c[1]
        dx = np.arange(int(c[0]) - h, int(c[0]) + h + 1)[None, None, :] - c[0]
        blob = 0.5 * (1.0 - np.tanh((np.sqrt(dx * dx + dy * dy + dz * dz) - r) / 2.0))
        sub = phi[np.ix_(zi, yi, xi)]
        phi[np.ix_(zi, yi, xi)] = np.maximum(sub, blob)
    phi = np.where(isf == 0, 0.0, phi)
    phi = seed_solid_phi(phi, isf, 27)
    return isf, phi


def droplets_field(L: int, n: int = 200, seed: int = 2024, rmin: float = 10.0, rmax: float = 30.0,
                   width: float = 4.0, sigma: float = 0.01, rho_r: float = 5.0, rho_b: float = 0.5):
    """Moments and phi (float32) of a periodic L^3 box holding n seeded
    droplets (centres U[0,L)^3, radii U[rmin, rmax], the fcut_tanh profile of
    width 4) at rest, each node's P the Laplace pressure of the droplet that
    dominates it (init_conditions_module.f90:413-414)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    phi = np.zeros((L, L, L), np.float32)
    press = np.zeros((L, L, L), np.float32)
    for _ in range(n):
        c = rng.uniform(0.0, L, 3)
        r = rng.uniform(rmin, rmax)
        h = int(r + 2 * width) + 1
        idx = [np.arange(int(c[d]) - h, int(c[d]) + h + 1) for d in range(3)]
        d2 = ((idx[2][:, None, None] - c[2]) ** 2 + (idx[1][None, :, None] - c[1]) ** 2 +
              (idx[0][None, None, :] - c[0]) ** 2)
        f = (0.5 * (1.0 - np.tanh((np.sqrt(d2) - r) / (0.5 * width)))).astype(np.float32)
        ix = np.ix_(idx[2] % L, idx[1] % L, idx[0] % L)
        sub = phi[ix]
        take = f > sub
        rhophi = rho_r * f + (1.0 - f) * rho_b
        pr = (f * (2.0 * sigma) / r / (rhophi / 3.0)).astype(np.float32)
        phi[ix] = np.where(take, f, sub)
        press[ix] = np.where(take, pr, press[ix])
    m = np.zeros((10, L, L, L), np.float32)
    m[0] = press
    return m, phi


def workload(storage: str = "f32", L: int = LBOX, kind: str = "laplace", oracle_helpers: bool = False):
    """(Params, moments, phi, isfluid or None) of the Laplace droplet (L^3,
    the headline), of the channel with obstacles (512 x 256 x 256: walls,
    spheres and wetting at 90 degrees, body force 1e-6, the twopoiseuille.inp
    fluid parameters), of the box of 200 seeded droplets (L^3, the bench.inp
    fluid parameters) or of the Taylor-Green vortex (64^3 D3Q19, one
    component)."""
    import numpy as np

    from lbfast_b200.capi import Params
    _, _, ic_droplet = _helpers(oracle_helpers)
    if kind == "channel":
        lx, ly, lz = CHANNEL
        p = Params(lx=lx, ly=ly, lz=lz, pbc_y=0, lattice=27, highorder=1, twocomponent=1, densratio=1,
                   obstacles=1, visc1=0.05, visc2=0.4, rho_r=0.5, rho_b=1.5, sigma=0.0, width=4.0,
                   tau_diff=0.1, fx=1e-6, wettab_r=90.0, printphi=1, storage=storage)
        isf, phi = channel_geometry(lx, ly, lz, oracle_helpers)
        return p, np.zeros((10, lz, ly, lx)), phi, isf
    if kind == "droplets":
        p = Params(lx=L, ly=L, lz=L, lattice=27, highorder=1, twocomponent=1, densratio=1, visc1=0.2,
                   visc2=0.025, rho_r=5.0, rho_b=0.5, sigma=0.01, width=4.0, tau_diff=0.12, fx=1e-6,
                   printphi=1, storage=storage)
        m, phi = droplets_field(L)
        return p, m, phi, None
    if kind == "taylorgreen":
        from oracle import oracle as O
        p = Params(lx=64, ly=64, lz=64, lattice=19, visc1=0.01, storage=storage)
        return p, O.ic_taylor_green(64, 64, 64, 0.05), None, None
    p = Params(lx=L, ly=L, lz=L, lattice=27, highorder=1, twocomponent=1, densratio=1,
               visc1=0.1, visc2=0.1, rho_r=RHO_R, rho_b=RHO_B, sigma=0.03, width=3.0, tau_diff=0.1,
               printphi=1, storage=storage)
    R = 40.0 * L / 256
    m, phi = ic_droplet(L, L, L, (L / 2, L / 2, L / 2), R, 3.0, 0.03, RHO_R, RHO_B, True)
    return p, m, phi, None


def box_of(kind, L=LBOX):
    if kind == "taylorgreen":
        return [64, 64, 64]
    return list(CHANNEL) if kind == "channel" else [L, L, L]


def bytes_per_lup(storage, kind):
    if kind == "taylorgreen":
        return {"f32": 80, "f64": 160}.get(storage, 56)  # one component: 10 moments
    return B_LUP[storage] + (1 if kind == "channel" else 0)  # + the isfluid byte with obstacles


def config_dict(storage, L=LBOX, kind="laplace"):
    box = box_of(kind, L)
    n = box[0] * box[1] * box[2]
    b = bytes_per_lup(storage, kind)
    if kind == "channel":
        text = ("two-component channel with obstacles 512x256x256, D3Q27 HIGHORDER DENSRATIO (rho 0.5/1.5, "
                "nu 0.05/0.4), walls at y = 0 and 255, 64 seeded spheres R U[6,14], seeded phi blobs, "
                "wetting 90 degrees, fx 1e-6, fluids at rest")
    elif kind == "droplets":
        text = (f"{L}^3 periodic, 200 seeded droplets R U[10,30] (seed 2024, width 4), D3Q27 HIGHORDER "
                f"two-component DENSRATIO (rho 5/0.5, nu 0.2/0.025, sigma 0.01, tau_diff 0.12, fx 1e-6)")
    elif kind == "taylorgreen":
        text = "Taylor-Green vortex 64^3 periodic, one-component D3Q19, nu 0.01, u0 0.05, 1000 steps"
    else:
        text = (f"Laplace droplet {L}^3 periodic, D3Q27 HIGHORDER two-component DENSRATIO "
                f"(rho_r/rho_b = {RHO_R:g}/{RHO_B:g}), R={int(40 * L / 256)}, width 3, sigma 0.03")
    tg = kind == "taylorgreen"
    return {"workload": text, "box": box, "lattice": "D3Q19" if tg else "D3Q27", "highorder": not tg,
            "twocomponent": not tg, "densratio": not tg, "obstacles": kind == "channel", "storage": storage,
            "bytes_per_lup": b,
            "l2_policy": ("state (%.2f GB) larger than the 126 MB L2; no flush" % (n * b / 1e9)
                          if n * b / 2 > 126e6 else
                          "state (%.3f GB) fits in the 126 MB L2: not a valid headline size" % (n * b / 1e9))}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons of one GPU, sampled every 100 ms
    while the context is open.  The GPU is named by its UUID (torch's device
    index need not be nvidia-smi's index under CUDA_VISIBLE_DEVICES); entering
    waits until the first sample is written, because nvidia-smi takes about a
    second to start and a short timed region would otherwise see none."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = str(gpu_index)
        try:
            import torch
            self.gpu = "GPU-" + str(torch.cuda.get_device_properties(gpu_index).uuid)
        except Exception:  # noqa: BLE001 -- fall back to the index
            pass
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="lbf_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        t0 = time.monotonic()
        while self.proc is not None and time.monotonic() - t0 < 15.0:
            if self.proc.poll() is not None or os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[2:]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


from lbfast_b200.replicas import allmax, barrier, init_from_env, shutdown, weak_scaling_value  # noqa: E402


def run_ours(args, rank, local, world):
    import numpy as np
    import torch

    import lbfast_b200 as lbf
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    p, m, phi, isf = workload(args.storage, args.box, args.workload)
    p.tile_y, p.zseg = args.tile, args.zseg
    N = p.lx * p.ly * p.lz
    s = lbf.Solver(p)
    s.set_stream(stream.cuda_stream)
    if isf is not None:
        s.set_isfluid(isf)
    s.set_fields(m, phi)
    s.step(args.warmup)  # the first step runs the autotuner (schedule: z segments or persistent)
    s.sync()
    tuning = s.tuning
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # steps per second of steady stepping before and after the timed steps, so
    # that the clock samples describe the GPU under this load
    e0.record(stream)
    s.step(3)
    e1.record(stream)
    torch.cuda.synchronize()
    per_step = max(e0.elapsed_time(e1) / 3, 1e-3)
    soak_before = max(1, int(args.clock_window_ms / per_step))
    soak_after = max(1, int(0.3 * args.clock_window_ms / per_step))
    with ClockSampler(local) as clk:
        s.step(soak_before)
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        s.step(soak_after)
        torch.cuda.synchronize()
    ms = allmax(e0.elapsed_time(e1), world)
    clocks = clk.summary()
    clocks["window"] = (f"{soak_before} steps before the {args.steps} timed steps and {soak_after} after, "
                        "sampled every 100 ms")
    ms_step = ms / args.steps
    value = weak_scaling_value(N, args.steps, ms, world)
    # the step kernel is the only launch per step (with obstacles the small
    # wetting kernel precedes it): the step time bounds its average duration
    bytes_launch = bytes_per_lup(args.storage, args.workload) * N
    achieved = bytes_launch / (ms_step * 1e-3) / 1e9
    try:
        ok = bool(np.all(np.isfinite(s.reduce())))
    except lbf.LbfError:  # a non-finite sum
        ok = False
    s.close()

    # end to end through the C ABI with pinned host buffers
    pin_m = torch.empty((10, p.lz, p.ly, p.lx), dtype=torch.float32, pin_memory=True)
    pin_phi = torch.empty((p.lz, p.ly, p.lx), dtype=torch.float32, pin_memory=True)
    pin_m.numpy()[...] = m
    pin_phi.numpy()[...] = phi
    rho = torch.empty((p.lz, p.ly, p.lx), dtype=torch.float32, pin_memory=True).numpy()
    vel = torch.empty((p.lz, p.ly, p.lx, 3), dtype=torch.float32, pin_memory=True).numpy()
    press = torch.empty((p.lz, p.ly, p.lx), dtype=torch.float32, pin_memory=True).numpy()
    s = lbf.Solver(p)
    s.set_stream(stream.cuda_stream)
    if isf is not None:
        s.set_isfluid(isf)
    import ctypes as C
    lib = lbf.load()
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    # warm the path once (allocations of the staging buffer)
    lbf.capi.check(lib.lbf_set_fields(s.h, C.c_void_p(pin_m.data_ptr()), C.c_void_p(pin_phi.data_ptr()), 0))
    s.step(1)
    lbf.capi.check(lib.lbf_get_print_fields(s.h, fp(rho), fp(vel), fp(press)))
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    lbf.capi.check(lib.lbf_set_fields(s.h, C.c_void_p(pin_m.data_ptr()), C.c_void_p(pin_phi.data_ptr()), 0))
    s.step(args.steps)
    lbf.capi.check(lib.lbf_get_print_fields(s.h, fp(rho), fp(vel), fp(press)))
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    barrier(world)
    ms_e2e = allmax(max(e0.elapsed_time(e1), wall * 1e3), world)
    s.close()
    h2d = (10 + 1) * N * 4
    d2h = 5 * N * 4
    e2e = {"value": weak_scaling_value(N, args.steps, ms_e2e, world), "unit": UNIT,
           "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
           "path": "lbf_set_fields (pinned host, f32) + lbf_step + lbf_get_print_fields; the initial state is "
                   "uploaded once and copy_print read back once per run, the reference's stamp = nsteps cadence"}
    return {"value": value, "ms": ms, "ms_step": ms_step, "achieved": achieved, "clocks": clocks, "e2e": e2e,
            "finite": ok, "tuning": {"tile": [32, tuning[0]], "zseg": tuning[1]}}


def measure_extra(kind: str, storage: str, L: int, steps: int, warmup: int, peak: float):
    """Device-resident MLUPS and roofline of one more configuration on this
    GPU, timed like the headline (CUDA events on the launching stream,
    warm-up first; every state here is larger than the L2)."""
    import numpy as np
    import torch

    import lbfast_b200 as lbf
    stream = torch.cuda.current_stream()
    t_setup = time.monotonic()
    p, m, phi, isf = workload(storage, L, kind)
    N = p.lx * p.ly * p.lz
    s = lbf.Solver(p)
    s.set_stream(stream.cuda_stream)
    if isf is not None:
        s.set_isfluid(isf)
    s.set_fields(m, phi)
    del m, phi
    s.step(warmup)
    s.sync()
    t_setup = time.monotonic() - t_setup
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ms_step = ms / steps
    b = bytes_per_lup(storage, kind) * N
    try:
        ok = bool(np.all(np.isfinite(s.reduce())))
    except lbf.LbfError:
        ok = False
    tuning = s.tuning
    s.close()
    torch.cuda.empty_cache()
    achieved = b / (ms_step * 1e-3) / 1e9
    return {"config": config_dict(storage, L, kind), "value": N * steps / (ms * 1e-3) / 1e6, "unit": UNIT,
            "steps": steps, "warmup": warmup, "ms_per_step": ms_step,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "bytes_per_launch": b},
            "launch": {"tile": [32, tuning[0]], "zseg": tuning[1]}, "finite": ok, "setup_s": t_setup}


# ---- serving: an ensemble of droplet solves of uneven box sizes ----------

SERVE_EDGES = (32, 48, 64, 96, 128)


def p2_droplet(edge: int, eps: float, ratio: float, sigma: float = 0.03, width: float = 5.0, _cache={}):
    """Droplet of radius R = edge/4 at the box centre with the surface
    r_s(theta) = R (1 + eps P2(cos theta)), the fcut_tanh profile and the
    Laplace pressure of the reference's droplet set-up
    (init_conditions_module.f90:394-426); fluids at rest.  float32 fields."""
    import numpy as np
    if edge not in _cache:
        c = edge / 2
        x = np.arange(1, edge + 1) - c
        z, y, xx = np.meshgrid(x, x, x, indexing="ij")
        r = np.sqrt(xx * xx + y * y + z * z)
        ct = np.divide(z, r, out=np.zeros_like(r), where=r > 0)
        _cache[edge] = (r.astype(np.float32), (0.5 * (3 * ct * ct - 1)).astype(np.float32))
    r, p2 = _cache[edge]
    R = edge / 4
    rs = R * (1 + eps * p2)
    phi = 0.5 * (1 - np.tanh((r - rs) / (0.5 * width)))
    rhophi = ratio * phi + (1 - phi)
    m = np.zeros((10, edge, edge, edge), np.float32)
    m[0] = phi * (2 * sigma) / R / (rhophi / 3)
    return m, phi.astype(np.float32)


def serving_jobs(n: int, seed: int = 7):
    """n solves: edge uniform over SERVE_EDGES, eps ~ U[0.05, 0.15], density
    ratio log-uniform over [10, 1000] (rho_b = 1); D3Q27 two-component
    DENSRATIO, FP16 storage, sigma 0.03, nu 0.001, tau_diff 0.1, width 5."""
    import numpy as np
    import lbfast_b200 as lbf
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n):
        e = int(rng.choice(SERVE_EDGES))
        eps = float(rng.uniform(0.05, 0.15))
        ratio = float(np.exp(rng.uniform(np.log(10.0), np.log(1000.0))))
        p = lbf.Params(lx=e, ly=e, lz=e, lattice=27, highorder=0, twocomponent=1, densratio=1, visc1=0.001,
                       visc2=0.001, rho_r=ratio, rho_b=1.0, sigma=0.03, width=5.0, tau_diff=0.1, storage="f16")
        m, phi = p2_droplet(e, eps, ratio)
        jobs.append((p, m, phi))
    return jobs


def _drain(srv, jobs, nsteps):
    ids = [srv.submit(p, m, phi, nsteps) for p, m, phi in jobs]
    srv.drain()
    return ids


def run_serving(n: int, nsteps: int, seed: int = 7):
    """Solves/s of the batched server against the same solves run one at a
    time on the same engine (max_active = 1: same kernel, same graphs, no
    batching) and one at a time through lbf_step (each solve with its own
    autotuned kernel), the saturated throughput (all submitted at once), and
    per-solve latency under seeded Poisson arrivals at 1.5x the one-at-a-time
    rate."""
    import numpy as np
    import lbfast_b200 as lbf
    jobs = serving_jobs(n, seed)
    lups = sum(p.lx * p.ly * p.lz for p, _, _ in jobs) * nsteps
    # warm-up: kernel attributes, graph machinery, allocator
    with lbf.Server(chunk=32) as srv:
        _drain(srv, jobs[:2], 64)
    # one at a time
    with lbf.Server(max_active=1, chunk=32) as srv:
        t0 = time.monotonic()
        ids = _drain(srv, jobs, nsteps)
        t_seq = time.monotonic() - t0
        svc = {}
        for (p, _, _), i in zip(jobs, ids):
            info = srv.poll(i)
            svc.setdefault(p.lx, []).append(info["t_done"] - info["t_admit"])
        seq_out = [srv.fetch(i) for i in ids]
    # lattice updates per second of one solve running alone, by box edge
    alone_mlups = {e: e ** 3 * nsteps / float(np.mean(v)) / 1e6 for e, v in sorted(svc.items())}
    # one at a time through the single-box entry point (lbf_step, autotuned
    # 16-row kernel), fields uploaded and read back per solve like the server
    t0 = time.monotonic()
    for p, m, phi in jobs:
        s = lbf.Solver(p)
        s.set_fields(m, phi)
        s.step(nsteps)
        s.get_fields(np.float32)
        s.close()
    t_step = time.monotonic() - t0
    # batched, saturated
    with lbf.Server(chunk=32) as srv:
        t0 = time.monotonic()
        ids = _drain(srv, jobs, nsteps)
        t_bat = time.monotonic() - t0
        peak_bytes = sum(srv.poll(i)["device_bytes"] for i in ids)
        same = all(all(np.array_equal(a, b, equal_nan=True) for a, b in zip(srv.fetch(i), ref))
                   for i, ref in zip(ids, seq_out))
    del seq_out
    # batched, open loop: Poisson arrivals at 1.5x the one-at-a-time rate
    lam = 1.5 * n / t_seq
    rng = np.random.default_rng(seed)
    arrive = np.cumsum(rng.exponential(1.0 / lam, n))
    lat = []
    with lbf.Server(chunk=32) as srv:
        t0 = time.monotonic()
        nxt, pending = 0, {}
        while nxt < n or pending:
            now = time.monotonic() - t0
            while nxt < n and arrive[nxt] <= now:
                p, m, phi = jobs[nxt]
                pending[srv.submit(p, m, phi, nsteps)] = t0 + arrive[nxt]
                nxt += 1
            active, queued = srv.run(1)
            for sid in [i for i in pending if srv.poll(i)["state"] == "done"]:
                lat.append(srv.poll(sid)["t_done"] - pending.pop(sid))
                srv.fetch(sid)
            if active == 0 and queued == 0 and nxt < n:
                time.sleep(max(0.0, arrive[nxt] - (time.monotonic() - t0)))
        t_open = time.monotonic() - t0
    lat = np.sort(np.array(lat))
    edges = {e: sum(1 for p, _, _ in jobs if p.lx == e) for e in SERVE_EDGES}
    return {
        "workload": f"{n} droplet solves x {nsteps} steps, edges {list(SERVE_EDGES)} (counts {edges}), "
                    "R = edge/4 with a P2 shape perturbation eps ~ U[0.05,0.15], density ratio log-uniform "
                    "[10,1000], D3Q27 two-component DENSRATIO, FP16 storage, nu 0.001, sigma 0.03, width 5, seed 7",
        "solves_per_s": n / t_bat, "solves_per_s_one_at_a_time": n / t_seq, "speedup": t_seq / t_bat,
        "solves_per_s_lbf_step": n / t_step, "speedup_vs_lbf_step": t_step / t_bat,
        "mlups_batched": lups / t_bat / 1e6, "mlups_one_at_a_time": lups / t_seq / 1e6,
        "mlups_alone_by_edge": alone_mlups,
        "open_loop": {"arrival_rate_per_s": lam, "solves_per_s": n / t_open,
                      "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                      "latency_max_s": float(lat[-1])},
        "peak_resident_bytes": peak_bytes, "alone_equals_mix_bitwise": bool(same),
        "timing": "host monotonic clock from first submit to last result on the host (fields copied back)",
    }


def cpu_baseline(storage: str, L: int, nsteps: int, threads: int, kind: str = "laplace", warmup: int = 0):
    """The oracle (C restatement of the reference, FP32 build stand-in) on the
    host cores: `warmup` untimed steps, then `nsteps` timed steps of the same
    box, set up with the oracle's own helpers."""
    import numpy as np
    from oracle import oracle as O
    p, m, phi, isf = workload(storage, L, kind, oracle_helpers=True)
    O.set_threads(threads)
    o = O.Oracle(p.oracle_dict(), "f32")
    o.set_isfluid(isf if isf is not None else np.ones(p.shape, np.int8))
    o.set_fields(m, phi)
    o.step(0)
    if warmup > 0:
        o.step(warmup)
    t0 = time.perf_counter()
    o.step(nsteps)
    dt = time.perf_counter() - t0
    return p.lx * p.ly * p.lz * nsteps / dt / 1e6, dt


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16", "f64"])
    ap.add_argument("--box", type=int, default=LBOX, help="edge of the Laplace box")
    ap.add_argument("--workload", default="laplace", choices=["laplace", "channel"],
                    help="laplace: the droplet box (headline); channel: 512x256x256 with obstacles")
    ap.add_argument("--tile", type=int, default=0, help="kernel tile rows (8 or 16); 0: autotuned")
    ap.add_argument("--zseg", type=int, default=0,
                    help="planes per z segment; negative: columns split at plane -zseg; 0: autotuned / automatic")
    ap.add_argument("--cpu-steps", type=int, default=2, help="steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-solves", type=int, default=40, help="solves of the serving measurement (0: skip)")
    ap.add_argument("--serve-steps", type=int, default=3000)
    ap.add_argument("--extra", default="f16,channel,c4,c4f16",
                    help="comma list of extra device-resident lines: f16 (FP16 storage, headline box), channel "
                         "(512x256x256 FP32), c4 / c4f16 (768^3 seeded droplets, FP32 / FP16); '' for none")
    ap.add_argument("--extra-steps", type=int, default=20)
    ap.add_argument("--no-tg-baseline", action="store_true",
                    help="skip the CPU Taylor-Green baseline (64^3 D3Q19, 1000 steps)")
    ap.add_argument("--clock-window-ms", type=float, default=1000.0,
                    help="steady stepping before the timed steps while nvidia-smi samples clocks")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, local, world = init_from_env()
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            shutdown(world)
            return
        # each step of the reference arm is one full oracle step of the box
        # (about 1.3 s on 16 host cores at 256^3): all --warmup steps run
        # untimed, the timed steps are capped at 20 so the arm ends in a minute
        k = max(1, min(args.steps, 20))
        mlups, dt = cpu_baseline(args.storage, args.box, k, threads, args.workload, warmup=args.warmup)
        line = {"impl": "reference", "metric": METRIC, "value": mlups, "unit": UNIT, "n_gpus": args.gpus,
                "steps": k, "warmup": args.warmup, "ms_per_step": dt / k * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(config_dict(args.storage, args.box, args.workload),
                               parallelism=f"replicas x{args.gpus}"),
                "cpu_baseline": {"value": mlups, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": f"{k} steps of the {box_of(args.workload, args.box)} box, FP32 C restatement of the "
                                           f"reference kernels (oracle/lbf_oracle.c), OpenMP over z"},
                "e2e": {"value": mlups, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        shutdown(world)
        return

    import json as _json
    peaks = {}
    try:
        peaks = _json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    r = run_ours(args, rank, local, world)
    extra = []
    if rank == 0 and world == 1:
        table = {"f16": ("laplace", "f16", args.box), "channel": ("channel", "f32", args.box),
                 "c4": ("droplets", "f32", 768), "c4f16": ("droplets", "f16", 768)}
        for name in [x for x in args.extra.split(",") if x]:
            kind, storage, L = table[name]
            try:
                extra.append(dict(measure_extra(kind, storage, L, args.extra_steps, args.warmup, peak), name=name))
            except Exception as ex:  # noqa: BLE001 -- one failed extra line must not lose the headline
                extra.append({"name": name, "error": f"{type(ex).__name__}: {ex}"})
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        mlups, dt = cpu_baseline(args.storage, args.box, args.cpu_steps, threads, args.workload)
        cpu = {"value": mlups, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{args.cpu_steps} steps of the same {box_of(args.workload, args.box)} box ({dt:.1f} s), FP32 C restatement of "
                         f"the reference kernels (oracle/lbf_oracle.c), OpenMP"}
        if not args.no_tg_baseline:
            tg, dt = cpu_baseline("f32", 64, 1000, threads, "taylorgreen")
            cpu["taylor_green"] = {"value": tg, "unit": UNIT, "cores": threads, "kind": "port",
                                   "sample": f"Taylor-Green 64^3 D3Q19 one component, the full 1000 steps ({dt:.1f} s), "
                                             "FP32 oracle, OpenMP"}
    serving = None
    if rank == 0 and world == 1 and args.serve_solves > 0:
        serving = run_serving(args.serve_solves, args.serve_steps)
    if rank != 0:
        shutdown(world)
        return
    traffic = NCU_TRAFFIC.get((args.storage, args.box)) if args.workload == "laplace" else None
    winst = NCU_WARP_INST.get((args.storage, args.box)) if args.workload == "laplace" else None
    issue = None
    if winst:
        # the instruction-issue ceiling of the step: every SM issuing one warp
        # instruction per scheduler (4) per cycle at the sampled SM clock
        import torch
        nsm = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = r["clocks"].get("sm_mhz") or 1965.0
        n = args.box ** 3
        ceiling = nsm * 4 * mhz * 1e6 / (winst / n) / 1e6
        issue = {"warp_inst_per_launch": winst, "thread_inst_per_node": winst * 32 / n, "sms": nsm, "sm_mhz": mhz,
                 "ceiling_mlups": ceiling, "frac": r["value"] / world / ceiling,
                 "source": "ncu smsp__inst_executed.sum of one step launch (profiles/)"}
    nbox = box_of(args.workload, args.box)
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.storage != "f64" else "f64", "data": "synthetic",
        "config": dict(config_dict(args.storage, args.box, args.workload), parallelism=f"replicas x{world}"),
        "roofline": {"bound": "hbm", "achieved": r["achieved"], "peak": peak, "unit": "GB/s",
                     "frac": r["achieved"] / peak, "traffic": traffic, "peak_source": peak_src,
                     "kernel": "lbf::stream_kernel<27,HO,TC>", "launch": r["tuning"],
                     "bytes_per_launch": bytes_per_lup(args.storage, args.workload) * nbox[0] * nbox[1] * nbox[2],
                     "issue": issue},
        "e2e": r["e2e"], "gpu_launches": args.steps * (2 if args.workload == "channel" else 1), "clocks": r["clocks"],
        "cpu_baseline": cpu,
        "finite": r["finite"], "extra": extra, "serving": serving,
    }
    print(json.dumps(line))
    shutdown(world)


if __name__ == "__main__":
    main()
