"""CPU restatement of molmot/mot/analysis.py for a trajectory ensemble stored
as arrays (test infrastructure: the checker of molmot_b200.analysis, never
called by it).

The reference takes a list of (t_arr, z_arr, v_arr) per molecule; every
trajectory of molmot/propagation/trajectories.py:19-75 has the same time
axis t_arr = arange(n_steps) * dt and keeps its last state after escaping, so
the ensemble is (t [S], Z [N, S], V [N, S]) here.

Pinned against the reference's own functions run on the seeded ensembles of
``synthetic_ensemble`` (tests/golden/analysis_golden.npz, written by
tests/golden/make_golden.py).
"""
from __future__ import annotations

import numpy as np

K_B = 1.380649e-23
R_ESCAPE = 0.015  # the trap radius analysis.py:166 and :230 hard-code


def synthetic_ensemble(seed: int = 7, n: int = 150, n_steps: int = 600, dt: float = 1e-5):
    """Seeded ensemble shaped like simulate_trajectory output: damped random
    walks in z with v = dz/dt, a fifth of them drifting out of the trap; a
    molecule that passes |z| > 0.015 m keeps its state from then on."""
    rng = np.random.default_rng(seed)
    t = np.arange(n_steps) * dt
    Z = np.zeros((n, n_steps))
    V = np.zeros((n, n_steps))
    z = rng.normal(0.0, 1.5e-3, n)
    v = rng.normal(0.0, 0.3, n)
    drift = np.where(rng.random(n) < 0.2, rng.normal(0.0, 3000.0, n), 0.0)
    Z[:, 0], V[:, 0] = z, v
    done = np.abs(z) > R_ESCAPE
    for j in range(1, n_steps):
        a = -4e3 * z - 50.0 * v + drift + rng.normal(0.0, 40.0, n)
        v_new = v + a * dt
        z_new = z + v_new * dt
        v = np.where(done, v, v_new)
        z = np.where(done, z, z_new)
        done = done | (np.abs(z) > R_ESCAPE)
        Z[:, j], V[:, j] = z, v
    return t, Z, V


def _bin_indices(t, time_bins):
    """Time-bin centres and the sample index of each (analysis.py:152-170)."""
    edges = np.linspace(0, t[-1], time_bins + 1)
    centres = 0.5 * (edges[:-1] + edges[1:])
    idx = np.minimum(np.searchsorted(t, centres), len(t) - 1)
    return centres, idx


def sigma_vs_time(t, Z, V, time_bins=50):
    """analysis.py:128-192: std of z and v over molecules with |z| < 0.015."""
    centres, idx = _bin_indices(t, time_bins)
    sz = np.full(time_bins, np.nan)
    sv = np.full(time_bins, np.nan)
    n_alive = np.zeros(time_bins)
    for b, j in enumerate(idx):
        alive = np.abs(Z[:, j]) < R_ESCAPE
        n_alive[b] = alive.sum()
        if n_alive[b] > 1:
            sz[b] = np.std(Z[alive, j])
            sv[b] = np.std(V[alive, j])
    return centres, sz, sv, n_alive


def temperature_vs_time(t, Z, V, mass, time_bins=50):
    """analysis.py:195-246: T = m <v^2> / k_B over molecules with |z| < 0.015."""
    centres, idx = _bin_indices(t, time_bins)
    T = np.full(time_bins, np.nan)
    for b, j in enumerate(idx):
        alive = np.abs(Z[:, j]) < R_ESCAPE
        if alive.sum() > 1:
            T[b] = mass * np.mean(V[alive, j] ** 2) / K_B
    return centres, T


def density_vs_time(t, Z, V, N_total=2000, time_bins=50):
    """analysis.py:249-287: n0 = N_eff / (sigma^3 (2 pi)^1.5), N_eff scaled by survival."""
    centres, sz, _, n_alive = sigma_vs_time(t, Z, V, time_bins)
    n0 = np.zeros(time_bins)
    ok = np.isfinite(sz) & (sz > 0)
    n_eff = N_total * (n_alive / Z.shape[0])
    n0[ok] = n_eff[ok] / (sz[ok] ** 3 * (2 * np.pi) ** 1.5)
    return centres, n0


def survived(z_traj, r_max=3e-3):
    """analysis.py:290-312: |z_final| < r_max (per molecule)."""
    return np.abs(np.asarray(z_traj)[..., -1]) < r_max


def capture_fraction(t, Z, r_max=3e-3, t_min=1e-3):
    """analysis.py:315-355: share of molecules with |z(t_min)| < r_max, among
    trajectories that reach t_min (all or none on a shared time axis)."""
    if Z.shape[0] == 0 or t[-1] < t_min:
        return 0.0
    j = min(int(np.searchsorted(t, t_min)), len(t) - 1)
    return float(np.mean(np.abs(Z[:, j]) < r_max))


def _gauss(x, A, mu, sigma):
    return A * np.exp(-0.5 * ((x - mu) / sigma) ** 2)


def _fit_sigma(x, bins, lo, hi, sigma_floor):
    from scipy.optimize import curve_fit
    counts, edges = np.histogram(x, bins=bins, range=(lo, hi))
    centres = 0.5 * (edges[:-1] + edges[1:])
    counts = counts.astype(float)
    if np.max(counts) < 1:
        return np.inf
    p0 = [np.max(counts), np.mean(x), np.std(x)]
    if p0[2] < 1e-10:
        p0[2] = sigma_floor
    try:
        popt, _ = curve_fit(_gauss, centres, counts, p0=p0, maxfev=5000)
        return abs(popt[2])
    except (RuntimeError, ValueError):
        return np.inf


def gaussian_fit(positions, bins=200, range_mm=(-2, 2)):
    """analysis.py:28-71: sigma (m) of a Gaussian fitted to the histogram."""
    return _fit_sigma(np.asarray(positions), bins, range_mm[0] * 1e-3, range_mm[1] * 1e-3, 1e-4)


def maxwell_boltzmann_fit_1d(velocities, mass, bins=100, range_ms=(-1, 1)):
    """analysis.py:74-125: T = m sigma_v^2 / k_B of a Gaussian fitted to the histogram."""
    s = _fit_sigma(np.asarray(velocities), bins, range_ms[0], range_ms[1], 0.01)
    return mass * s ** 2 / K_B if np.isfinite(s) else np.inf
