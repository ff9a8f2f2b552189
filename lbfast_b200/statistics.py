"""Benchmark observables of the reference's statistics.f90, computed from the
copy_print fields (rho with PRINTPHI = phi, vel, press) a run returns.

* Laplace (statistics.f90:88-275): pressure inside at nint(center) and
  outside at the probe, p = rho_phi * cs^2 * P; radius from the
  phi(1-phi)-weighted interface positions along x through (ly/2, lz/2);
  sigma_eff = delta_p * radius / 2.
* Taylor-Green (statistics.f90:36-86, 918-956): mean kinetic energy and the
  viscosity fitted to E/E0 = exp(-6 nu k^2 t).
* Poiseuille (statistics.f90:825-880): the velocity along z averaged over each
  x plane, against fz / (2 nu) (H^2 - d^2).
* Lamb (statistics.f90:377-471, 959-1100): phi(1-phi)-weighted interface
  positions along the x and z lines through the box centre, the z half-axis
  (the reference's `dosc`), and Lamb's n = 2 frequency with the reference's
  viscous correction.
Indices follow the reference's 1-based global coordinates.
"""
from __future__ import annotations

import numpy as np

CSSQ = 1.0 / 3.0


def _nint(x: float) -> int:
    return int(np.floor(x + 0.5)) if x >= 0 else -int(np.floor(-x + 0.5))


def laplace_observables(phi, press, center, probe, rho_r, rho_b):
    """phi, press: (lz, ly, lx) print fields; center: namelist `center`
    (1-based); probe: (iprobe, jprobe, kprobe).  Returns
    (sigma_eff, delta_p, radius)."""
    lz, ly, lx = phi.shape
    phi = np.asarray(phi, dtype=np.float64)
    press = np.asarray(press, dtype=np.float64)

    def at(a, i, j, k):
        return a[k - 1, j - 1, i - 1]

    gj, gk = ly // 2, lz // 2
    line = phi[gk - 1, gj - 1, :]
    gi = np.arange(1, lx + 1, dtype=np.float64)
    w = line * (1.0 - line)
    h = lx // 2
    left = (gi[:h] * w[:h]).sum() / w[:h].sum()
    right = (gi[h:] * w[h:]).sum() / w[h:].sum()
    radius = right - 0.5 * (right + left)
    ci, cj, ck = (_nint(c) for c in center)
    ph_in = at(phi, ci, cj, ck)
    ph_out = at(phi, *probe)
    p_in = (rho_r * ph_in + (1 - ph_in) * rho_b) * CSSQ * at(press, ci, cj, ck)
    p_out = (rho_r * ph_out + (1 - ph_out) * rho_b) * CSSQ * at(press, *probe)
    dp = p_in - p_out
    return dp * radius * 0.5, dp, radius


def kinetic_energy(vel) -> float:
    """statistics.f90:36-86: 0.5 <|u|^2> over the box (vel: (3, lz, ly, lx))."""
    v = np.asarray(vel, dtype=np.float64)
    return 0.5 * float(np.mean((v * v).sum(0)))


def fit_viscosity(steps, energies, L: int) -> float:
    """nu from a least-squares fit of log(E/E0) = -6 nu k^2 t, k = 2 pi / L."""
    t = np.asarray(steps, dtype=np.float64)
    e = np.asarray(energies, dtype=np.float64)
    k = 2.0 * np.pi / L
    slope = np.polyfit(t, np.log(e / e[0]), 1)[0]
    return -slope / (6.0 * k * k)


def poiseuille_profile(w, isf):
    """statistics.f90:842-868: w (lz, ly, lx) velocity along z, 0 on solid
    nodes, averaged over each x plane (gi = 1..lx)."""
    w = np.where(np.asarray(isf) == 0, 0.0, np.asarray(w, dtype=np.float64))
    return w.mean(axis=(0, 1))


def poiseuille_theory(lx: int, fz: float, nu: float, H: float, xc: float):
    """fz / (2 nu) (H^2 - (gi - xc)^2) inside |gi - xc| <= H, 0 outside
    (statistics.f90:831-845: H = (lx-1)/2, xc = (lx+1)/2 puts the walls on the
    solid nodes; H = lx/2 - 1 the half-way walls of bounce-back)."""
    gi = np.arange(1, lx + 1, dtype=np.float64)
    d = np.abs(gi - xc)
    return np.where(d <= H, fz / (2.0 * nu) * (H * H - d * d), 0.0)


def _interface_pos(line, idx):
    w = line * (1.0 - line)
    return float((idx * w).sum() / w.sum())


def lamb_observables(phi):
    """print_lamb (statistics.f90:377-471): interface positions along the x
    line (gj = ly/2, gk = lz/2) and the z line (gi = lx/2, gj = ly/2), each
    half separately.  Returns (lamb_x, lamb_z, dosc) with lamb_* the extents
    and dosc = z half-axis (pos_z_right - centre), the series the reference's
    frequency analysis reads."""
    phi = np.asarray(phi, dtype=np.float64)
    lz, ly, lx = phi.shape
    gi, gj, gk = lx // 2, ly // 2, lz // 2
    zl = phi[:, gj - 1, gi - 1]
    xl = phi[gk - 1, gj - 1, :]
    kz = np.arange(1, lz + 1, dtype=np.float64)
    kx = np.arange(1, lx + 1, dtype=np.float64)
    zlo, zhi = _interface_pos(zl[: lz // 2], kz[: lz // 2]), _interface_pos(zl[lz // 2:], kz[lz // 2:])
    xlo, xhi = _interface_pos(xl[: lx // 2], kx[: lx // 2]), _interface_pos(xl[lx // 2:], kx[lx // 2:])
    lamb_z, lamb_x = zhi - zlo, xhi - xlo
    return lamb_x, lamb_z, zhi - 0.5 * (zhi + zlo)


def lamb_theory_omega(sigma, radius, rho_r, rho_b, visc1, visc2):
    """statistics.f90:973-981: Lamb's n = 2 angular frequency of a droplet
    (density rho_r) in a host fluid (rho_b), with the reference's viscous
    correction."""
    mu1, mu2 = rho_r * visc1, rho_b * visc2
    w0 = np.sqrt(24.0 * sigma / (radius ** 3 * (2.0 * rho_b + 3.0 * rho_r)))
    chi = ((2 * 2 + 1) ** 2 * np.sqrt(mu1 * mu2 * rho_r * rho_b)) / (
        np.sqrt(2.0) * radius * (2.0 * rho_b + 3.0 * rho_r) * (np.sqrt(mu1 * rho_r) + np.sqrt(mu2 * rho_b)))
    return w0 - 0.5 * chi * np.sqrt(w0) + 0.25 * chi ** 2


def mean_period(steps, series, min_dist: float):
    """Mean distance between the local maxima of `series` above its mean that
    are at least min_dist apart (statistics.f90:1020-1050)."""
    s = np.asarray(series, dtype=np.float64)
    t = np.asarray(steps, dtype=np.float64)
    ref = s.mean()
    peaks = []
    for i in range(1, len(s) - 1):
        if s[i] > s[i - 1] and s[i] >= s[i + 1] and s[i] > ref:
            if not peaks or t[i] - peaks[-1] >= min_dist:
                peaks.append(t[i])
    if len(peaks) < 2:
        return float("nan"), len(peaks)
    return float(np.mean(np.diff(peaks))), len(peaks)


def first_extrema(steps, series, count: int = 3):
    """The first `count` alternating extrema of `series` after its first
    maximum, beginning with a minimum: [(t, value, kind)], each refined by the
    parabola through the sampled extremum and its two neighbours.  A damped
    oscillation's first cycle is measured this way before later small
    wiggles, where counting every local maximum above the mean (mean_period,
    the reference's method) picks up noise."""
    s = np.asarray(series, dtype=np.float64)
    t = np.asarray(steps, dtype=np.float64)
    dt = t[1] - t[0]
    out = []
    # a series that falls from its first sample starts at its first maximum
    want = "min" if s[0] >= s[1] else None
    for i in range(1, len(s) - 1):
        is_max = s[i] > s[i - 1] and s[i] >= s[i + 1]
        is_min = s[i] < s[i - 1] and s[i] <= s[i + 1]
        if want is None:
            if is_max:
                want = "min"
            continue
        if (want == "min" and is_min) or (want == "max" and is_max):
            y0, y1, y2 = s[i - 1], s[i], s[i + 1]
            den = y0 - 2.0 * y1 + y2
            off = 0.5 * (y0 - y2) / den if den != 0 else 0.0
            out.append((t[i] + off * dt, y1 - 0.25 * (y0 - y2) * off, want))
            if len(out) == count:
                break
            want = "max" if want == "min" else "min"
    return out
