"""GPU API twin of the reference's ``molmot_cuda`` package
(molmot_cuda/__init__.py:34-169, rate_equations_cuda.py:399-894,
trajectories_cuda.py:305-452), computed by molmot_b200's sm_100a kernels.

Semantics follow the reference's CUDA path: hbar = 1.0545718e-34 and, when
every population clamps to zero, uniform populations
(molmot_cuda/rate_equations_cuda.py:253-258).  All functions return numpy
arrays shaped as the reference's.
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np
import torch

from .constants import HBAR_JIT
from .engine import BeamSets, force_batch, pack_for
from .force_scan import optimize_parameters as _optimize_parameters
from .simulator import BeamListSimulator


def has_cuda() -> bool:
    """True when a CUDA GPU is visible and the native library loads."""
    from . import has_cuda as _h
    return _h()


def get_device_info() -> dict:
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    free, total = torch.cuda.mem_get_info()
    return {"name": p.name, "compute_capability": f"{p.major}.{p.minor}",
            "total_memory_MB": total / 2 ** 20, "free_memory_MB": free / 2 ** 20,
            "num_devices": torch.cuda.device_count()}


class CUDAMolData:
    """Device-resident molecule and beams for repeated calls
    (molmot_cuda/rate_equations_cuda.py:399-441)."""

    def __init__(self, mol_data, beams, Gamma_eff_factor: float = 1.0):
        self.mol_data = mol_data
        self.beams = list(beams)
        self.pack = pack_for(mol_data)
        self.n_ground, self.n_excited = mol_data.n_ground, mol_data.n_excited
        self.n_states = mol_data.n_ground + mol_data.n_excited
        self.n_beams = len(self.beams)
        self.Gamma, self.k = float(mol_data.Gamma), float(mol_data.k)
        self.Gamma_eff = float(Gamma_eff_factor)
        self.hbar_val = HBAR_JIT
        self.mass = float(mol_data.mass)
        self._bs = {}

    def beam_sets(self, B_gradient: float) -> BeamSets:
        key = float(B_gradient)
        if key not in self._bs:
            self._bs[key] = BeamSets.from_beams(self.beams, key, self.Gamma_eff)
        return self._bs[key]


def solve_rate_equations_batch(mol_data, beams, v_arr: np.ndarray, z_arr: np.ndarray,
                               B_gradient: float, Gamma_eff_factor: float = 1.0,
                               cuda_data: Optional[CUDAMolData] = None
                               ) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """F (Nv, Nz), populations (Nv, Nz, n_ground), R (Nv, Nz) on the v x z grid."""
    cd = cuda_data if cuda_data is not None else CUDAMolData(mol_data, beams, Gamma_eff_factor)
    v_arr = np.atleast_1d(np.asarray(v_arr, dtype=np.float64))
    z_arr = np.atleast_1d(np.asarray(z_arr, dtype=np.float64))
    out = force_batch(cd.pack, cd.beam_sets(B_gradient), v_arr, z_arr, grid=True,
                      hbar=HBAR_JIT, uniform_fallback=True, want_status=False)
    nv, nz = v_arr.size, z_arr.size
    return (out["F"].cpu().numpy().reshape(nv, nz), out["pop"].cpu().numpy().reshape(nv, nz, -1),
            out["R"].cpu().numpy().reshape(nv, nz))


def force_vs_z_cuda(mol_data, beams, z_arr, v, B_gradient, Gamma_eff_factor=1.0, cuda_data=None):
    F, P, R = solve_rate_equations_batch(mol_data, beams, np.array([v]), z_arr, B_gradient,
                                         Gamma_eff_factor, cuda_data)
    return F[0, :], P[0, :, :], R[0, :]


def force_vs_v_cuda(mol_data, beams, v_arr, z, B_gradient, Gamma_eff_factor=1.0, cuda_data=None):
    F, _, _ = solve_rate_equations_batch(mol_data, beams, v_arr, np.array([z]), B_gradient,
                                         Gamma_eff_factor, cuda_data)
    return F[:, 0]


def force_map_2d_cuda(mol_data, beams, v_arr, z_arr, B_gradient, Gamma_eff_factor=1.0,
                      cuda_data=None):
    return solve_rate_equations_batch(mol_data, beams, v_arr, z_arr, B_gradient,
                                      Gamma_eff_factor, cuda_data)


def spring_constant_cuda(mol_data, beams, B_gradient, z0=0.0, dz=0.3e-3, Gamma_eff_factor=1.0,
                         cuda_data=None) -> float:
    F, _, _ = solve_rate_equations_batch(mol_data, beams, np.array([0.0]),
                                         np.array([z0 - dz, z0 + dz]), B_gradient,
                                         Gamma_eff_factor, cuda_data)
    return -(F[0, 1] - F[0, 0]) / (2.0 * dz)


def damping_coefficient_cuda(mol_data, beams, B_gradient, z0=0.0, dv=0.1, Gamma_eff_factor=1.0,
                             cuda_data=None) -> float:
    F, _, _ = solve_rate_equations_batch(mol_data, beams, np.array([-dv, dv]), np.array([z0]),
                                         B_gradient, Gamma_eff_factor, cuda_data)
    return -(F[1, 0] - F[0, 0]) / (2.0 * dv)


def optimize_parameters_cuda(mol_data, delta_arr, split_arr, s0, B_gradient, dz=0.3e-3, dv=0.1,
                             Gamma_eff_factor=1.0, verbose=True) -> dict:
    """(delta, split) scan of the DC MOT in one launch
    (molmot_cuda/rate_equations_cuda.py:768-894)."""
    return _optimize_parameters(mol_data, {"delta": delta_arr, "split": split_arr}, B_gradient,
                                "dc", s0=s0, dz=dz, dv=dv, verbose=verbose,
                                Gamma_eff_factor=Gamma_eff_factor)


def simulate_trajectories_cuda(simulator, z0_arr, v0_arr, t_max, dt=1e-6, z_escape=0.015,
                               save_full=False, cuda_data=None, block_size=64):
    """(z_final, v_final, n_actual, z_traj, v_traj) for N particles
    (molmot_cuda/trajectories_cuda.py:305-426)."""
    from .trajectories import simulate_trajectories
    return simulate_trajectories(simulator, z0_arr, v0_arr, t_max, dt, z_escape, save_full)


def simulate_trajectory_cuda(simulator, z0, v0, t_max, dt=1e-6, z_escape=0.015, cuda_data=None):
    from .trajectories import simulate_trajectory
    return simulate_trajectory(simulator, z0, v0, t_max, dt, z_escape)


def capture_velocity_cuda(simulator, z_start=3e-3, v_max=15.0, dv=0.5, dt=1e-6, n_steps=5000,
                          z_escape=0.015) -> float:
    """All test velocities in one trajectory launch
    (molmot_cuda/force_scan_cuda.py:533-670); RF simulators included."""
    from .force_scan import capture_velocity
    return capture_velocity(simulator, z_start, v_max, dv, dt, n_steps, z_escape)


# ------------------------------------------------------------------ 3D twins
def rate_eq_force_3d_batch(mol_data, beams, r_arr, v_arr, B_gradient, Gamma_eff_factor=1.0):
    """(F [n, 3], R [n], pop [n, n_ground]) -- molmot_cuda/simulator_3d_cuda.py:666-754,
    with a correct eigensolver."""
    from .simulator_3d import rate_eq_force_3d_batch as f
    return f(mol_data, beams, r_arr, v_arr, B_gradient, Gamma_eff_factor)


def compute_3d_force_map_cuda(mol_data, beams, axes="xz", n_points=50, v=None, B_gradient=0.0,
                              extent=5e-3, Gamma_eff_factor=1.0):
    from .simulator_3d import MOTSimulator3D, compute_3d_force_map
    sim = MOTSimulator3D(mol_data, list(beams), B_gradient, Gamma_eff_factor=Gamma_eff_factor)
    return compute_3d_force_map(sim, axes, n_points, v, extent)


def simulate_ensemble_3d_cuda(mol_data, beams, r0_list, v0_list, t_max, dt=1e-6, B_gradient=0.0,
                              Gamma_eff_factor=1.0, r_escape=0.015):
    """(t [n_steps], r [N, n_steps, 3], v [N, n_steps, 3]) -- one launch for all steps
    (molmot_cuda/simulator_3d_cuda.py:890-973 launches once per step)."""
    from .simulator_3d import MOTSimulator3D
    sim = MOTSimulator3D(mol_data, list(beams), B_gradient, Gamma_eff_factor=Gamma_eff_factor)
    return sim.simulate_ensemble_arrays(r0_list, v0_list, t_max, dt, r_escape)


def simulate_trajectory_3d_cuda(mol_data, beams, r0, v0, t_max, dt=1e-6, B_gradient=0.0,
                                Gamma_eff_factor=1.0, r_escape=0.015):
    t, R, V = simulate_ensemble_3d_cuda(mol_data, beams, [r0], [v0], t_max, dt, B_gradient,
                                        Gamma_eff_factor, r_escape)
    return t, R[0], V[0]
