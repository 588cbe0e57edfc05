"""Simulator-taking GPU wrappers with the signatures of
molmot_cuda/force_scan_cuda.py:48-290, 533-843 (DC and RF simulators)."""
from __future__ import annotations

from typing import Dict

import numpy as np

from . import force_scan as _fs
from .simulator import as_gpu_simulator


def force_vs_z_cuda(simulator, z_arr: np.ndarray, v: float = 0.0):
    return _fs.force_vs_z(simulator, z_arr, v)


def force_vs_v_cuda(simulator, v_arr: np.ndarray, z: float = 0.0):
    return _fs.force_vs_v(simulator, v_arr, z)


def spring_constant_cuda(simulator, z0: float = 0.0, dz: float = 0.3e-3) -> float:
    return _fs.spring_constant(simulator, z0, dz)


def damping_coefficient_cuda(simulator, z0: float = 0.0, dv: float = 0.1) -> float:
    return _fs.damping_coefficient(simulator, z0, dv)


def capture_velocity_cuda(simulator, z_start=3e-3, v_max=15.0, dv=0.5, dt=1e-6, n_steps=5000,
                          z_escape=0.015) -> float:
    return _fs.capture_velocity(simulator, z_start, v_max, dv, dt, n_steps, z_escape)


def optimize_parameters_cuda(mol_data, param_ranges: Dict[str, np.ndarray], B_gradient: float,
                             mot_type: str = "dc", s0: float = 1.0, dz: float = 0.3e-3,
                             dv: float = 0.1, Gamma_eff_factor: float = 1.0,
                             verbose: bool = True) -> Dict:
    return _fs.optimize_parameters(mol_data, param_ranges, B_gradient, mot_type, s0, dz, dv,
                                   verbose, Gamma_eff_factor)


def force_map_2d_cuda(simulator, v_arr: np.ndarray, z_arr: np.ndarray):
    """F, populations, R on the v x z grid, shaped (Nv, Nz, ...)."""
    sim = as_gpu_simulator(simulator)
    v_arr = np.asarray(v_arr, dtype=np.float64)
    z_arr = np.asarray(z_arr, dtype=np.float64)
    V, Z = np.meshgrid(v_arr, z_arr, indexing="ij")
    F, P, R = sim.force_points(V.ravel(), Z.ravel())
    nv, nz = v_arr.size, z_arr.size
    return F.reshape(nv, nz), P.reshape(nv, nz, -1), R.reshape(nv, nz)
