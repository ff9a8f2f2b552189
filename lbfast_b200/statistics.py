"""Benchmark observables of the reference's statistics.f90, computed from the
copy_print fields (rho with PRINTPHI = phi, vel, press) a run returns.

* Laplace (statistics.f90:88-275): pressure inside at nint(center) and
  outside at the probe, p = rho_phi * cs^2 * P; radius from the
  phi(1-phi)-weighted interface positions along x through (ly/2, lz/2);
  sigma_eff = delta_p * radius / 2.
* Taylor-Green (statistics.f90:36-86, 918-956): mean kinetic energy and the
  viscosity fitted to E/E0 = exp(-6 nu k^2 t).
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
