"""Ensemble post-processing of trajectories on the GPU; drop-in for
molmot.mot.analysis (molmot/mot/analysis.py:28-355).

Every function takes the ensemble in the reference's form (a list of
(t_arr, z_arr, v_arr) per molecule) or as arrays: a tuple (t, Z, V) with Z, V
of shape [N, n_steps] (numpy or CUDA tensors), or ``ensemble_from_traj`` of a
``molmot_b200.engine.traj(..., save_full=True)`` result.  The reductions over
molecules run as device kernels (mm_ensemble_stats: per-time-bin counts,
means and two-pass variances of the molecules inside the trap; mm_histogram:
numpy.histogram's binning); only the three-parameter Gaussian fits of
gaussian_fit / maxwell_boltzmann_fit_1d run on the host (scipy curve_fit on
the histogram, started from numpy's mean and std, as the reference).
"""
from __future__ import annotations

import ctypes
from typing import Tuple

import numpy as np
import torch

from . import _lib
from .constants import k_B
from .engine import _device, _dptr, _stream_handle

R_ESCAPE = 0.015  # trap radius that sigma_vs_time / temperature_vs_time use (analysis.py:166, :230)


def ensemble_from_traj(out: dict, dt: float, axis: int = 0):
    """(t, Z, V) of one axis from engine.traj(..., save_full=True)."""
    rt, vt = out["r_traj"], out["v_traj"]
    t = np.arange(rt.shape[1]) * dt
    return t, rt[:, :, axis], vt[:, :, axis]


def _as_ensemble(results):
    """(t host array, Z, V contiguous CUDA float64 [N, S])."""
    if isinstance(results, (list,)):
        if not results:
            raise ValueError("empty ensemble")
        t = np.asarray(results[0][0], dtype=np.float64)
        if any(len(r[0]) != len(t) for r in results):
            raise ValueError("trajectories of one ensemble share their time axis")
        Z = np.stack([np.asarray(r[1], dtype=np.float64) for r in results])
        V = np.stack([np.asarray(r[2], dtype=np.float64) for r in results])
    else:
        t, Z, V = results
        t = np.asarray(t.cpu() if torch.is_tensor(t) else t, dtype=np.float64)
    dev = _device()
    Z = torch.as_tensor(Z, dtype=torch.float64, device=dev).contiguous()
    V = torch.as_tensor(V, dtype=torch.float64, device=dev).contiguous()
    if Z.dim() != 2 or Z.shape != V.shape or Z.shape[1] != len(t):
        raise ValueError("Z and V must be [N, n_steps] with n_steps = len(t)")
    return t, Z, V


def _stats(Z, V, idx, r_alive):
    """[n_bins, 6]: count, mean z, mean v, var z, var v, mean v^2 (host array)."""
    dev = Z.device
    idx_d = torch.as_tensor(np.asarray(idx, dtype=np.int64), device=dev)
    out = torch.empty((len(idx), 6), dtype=torch.float64, device=dev)
    _lib.check(_lib.load().mm_ensemble_stats(_dptr(Z), _dptr(V), Z.shape[0], Z.shape[1], _dptr(idx_d),
                                             len(idx), float(r_alive), _dptr(out), _stream_handle(None)),
               "mm_ensemble_stats")
    return out.cpu().numpy()


def _bins(t, time_bins):
    edges = np.linspace(0, t[-1], time_bins + 1)
    centres = 0.5 * (edges[:-1] + edges[1:])
    idx = np.minimum(np.searchsorted(t, centres), len(t) - 1)
    return centres, idx


def sigma_vs_time(results, time_bins: int = 50):
    """Cloud size and velocity spread vs time over the molecules with
    |z| < 0.015 m: (t_centres, sigma_z, sigma_v, n_alive); NaN where at most
    one molecule remains (analysis.py:128-192)."""
    t, Z, V = _as_ensemble(results)
    centres, idx = _bins(t, time_bins)
    s = _stats(Z, V, idx, R_ESCAPE)
    n = s[:, 0]
    ok = n > 1
    sz = np.where(ok, np.sqrt(s[:, 3]), np.nan)
    sv = np.where(ok, np.sqrt(s[:, 4]), np.nan)
    return centres, sz, sv, n


def temperature_vs_time(results, mass: float, time_bins: int = 50):
    """T = m <v^2> / k_B vs time over the molecules with |z| < 0.015 m
    (analysis.py:195-246)."""
    t, Z, V = _as_ensemble(results)
    centres, idx = _bins(t, time_bins)
    s = _stats(Z, V, idx, R_ESCAPE)
    T = np.where(s[:, 0] > 1, mass * s[:, 5] / k_B, np.nan)
    return centres, T


def density_vs_time(results, N_total: int = 2000, time_bins: int = 50):
    """Peak density N_eff / (sigma^3 (2 pi)^1.5) vs time, N_eff = N_total times
    the surviving share (analysis.py:249-287)."""
    t, Z, V = _as_ensemble(results)
    centres, sz, _, n_alive = sigma_vs_time((t, Z, V), time_bins)
    n0 = np.zeros(time_bins)
    ok = np.isfinite(sz) & (sz > 0)
    n_eff = N_total * (n_alive / Z.shape[0])
    n0[ok] = n_eff[ok] / (sz[ok] ** 3 * (2 * np.pi) ** 1.5)
    return centres, n0


def survived(result, r_max: float = 3e-3) -> bool:
    """|z_final| < r_max for one trajectory (t_arr, z_arr, v_arr)
    (analysis.py:290-312).  For a whole ensemble see survived_mask."""
    _, z_arr, _ = result
    return bool(abs(float(z_arr[-1])) < r_max)


def survived_mask(results, r_max: float = 3e-3) -> np.ndarray:
    """survived() of every molecule of an ensemble."""
    _, Z, _ = _as_ensemble(results)
    return (Z[:, -1].abs() < r_max).cpu().numpy()


def capture_fraction(results, r_max: float = 3e-3, t_min: float = 1e-3) -> float:
    """Share of molecules with |z(t_min)| < r_max among the trajectories that
    run to t_min (analysis.py:315-355)."""
    t, Z, V = _as_ensemble(results)
    if Z.shape[0] == 0 or t[-1] < t_min:
        return 0.0
    j = min(int(np.searchsorted(t, t_min)), len(t) - 1)
    return float(_stats(Z, V, [j], r_max)[0, 0] / Z.shape[0])


def histogram(x, bins: int, lo: float, hi: float) -> Tuple[np.ndarray, np.ndarray]:
    """numpy.histogram(x, bins, range=(lo, hi)) computed on the device:
    (counts int64 [bins], edges [bins + 1])."""
    dev = _device()
    xd = torch.as_tensor(x, dtype=torch.float64, device=dev).contiguous().reshape(-1)
    counts = torch.empty(bins, dtype=torch.int64, device=dev)
    _lib.check(_lib.load().mm_histogram(_dptr(xd), xd.numel(), 1, float(lo), float(hi), int(bins),
                                        _dptr(counts), _stream_handle(None)), "mm_histogram")
    return counts.cpu().numpy(), np.linspace(lo, hi, bins + 1)


def _gauss(x, A, mu, sigma):
    return A * np.exp(-0.5 * ((x - mu) / sigma) ** 2)


def _fit_sigma(x, bins, lo, hi, sigma_floor):
    from scipy.optimize import curve_fit
    xd = torch.as_tensor(x, dtype=torch.float64, device=_device()).contiguous().reshape(-1)
    counts, edges = histogram(xd, bins, lo, hi)
    centres = 0.5 * (edges[:-1] + edges[1:])
    counts = counts.astype(float)
    if np.max(counts) < 1:
        return np.inf
    # the fit's starting point from numpy's mean and std, as the reference: the
    # fit can be ill-conditioned, and a start one rounding away may converge
    # to a different optimum
    xh = xd.cpu().numpy()
    p0 = [np.max(counts), np.mean(xh), np.std(xh)]
    if p0[2] < 1e-10:
        p0[2] = sigma_floor
    try:
        popt, _ = curve_fit(_gauss, centres, counts, p0=p0, maxfev=5000)
        return abs(popt[2])
    except (RuntimeError, ValueError):
        return np.inf


def gaussian_fit(positions, bins: int = 200, range_mm: Tuple[float, float] = (-2, 2)) -> float:
    """Sigma (m) of a Gaussian fitted to the position histogram; inf if the
    fit fails (analysis.py:28-71)."""
    return _fit_sigma(positions, bins, range_mm[0] * 1e-3, range_mm[1] * 1e-3, 1e-4)


def maxwell_boltzmann_fit_1d(velocities, mass: float, bins: int = 100,
                             range_ms: Tuple[float, float] = (-1, 1)) -> float:
    """Temperature m sigma_v^2 / k_B (K) of a Gaussian fitted to the velocity
    histogram; inf if the fit fails (analysis.py:74-125)."""
    s = _fit_sigma(velocities, bins, range_ms[0], range_ms[1], 0.01)
    return mass * s ** 2 / k_B if np.isfinite(s) else np.inf
