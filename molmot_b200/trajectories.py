"""Trajectory integration and particle sampling (drop-in for
molmot/propagation/trajectories.py and trajectories_jit.py).

All integrators run every particle and every step in one launch of the fused
trajectory kernel:

* simulate_trajectory / simulate_trajectory_jit -- one 1D Euler trajectory
  (trajectories.py:19-75, trajectories_jit.py:122-146)
* simulate_trajectories -- N 1D trajectories; (z_final, v_final, n_actual,
  z_traj, v_traj) like molmot_cuda's simulate_trajectories_cuda
* simulate_trajectories_3d -- the per-axis 3D model (trajectories.py:78-156)
* monte_carlo_temperature -- ensemble temperature (trajectories.py:159-229),
  with the reference's initial conditions (numpy default_rng(42) draws)
* samplers -- trajectories.py:236-442, on the host with numpy
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .constants import k_B
from .simulator import as_gpu_simulator


def simulate_trajectories(simulator, z0, v0, t_max: float, dt: float = 1e-6,
                          z_escape: float = 0.015, save_full: bool = False,
                          precision: str = "fp64"):
    """N independent 1D Euler trajectories.  Returns numpy arrays
    (z_final, v_final, n_actual, z_traj or None, v_traj or None)."""
    sim = as_gpu_simulator(simulator)
    n_steps = int(t_max / dt)
    o = sim.trajectories(np.atleast_1d(z0), np.atleast_1d(v0), dt, n_steps, ndim=1,
                         r_escape=z_escape, save_full=save_full, precision=precision)
    zt = o["r_traj"][..., 0].cpu().numpy() if save_full else None
    vt = o["v_traj"][..., 0].cpu().numpy() if save_full else None
    return (o["r_final"][:, 0].cpu().numpy(), o["v_final"][:, 0].cpu().numpy(),
            o["n_actual"].cpu().numpy(), zt, vt)


def simulate_trajectory(simulator, z0: float, v0: float, t_max: float, dt: float = 1e-6,
                        z_escape: float = 0.015) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(t, z, v) arrays of length int(t_max/dt); after an escape the last
    state repeats (trajectories.py:19-75)."""
    n_steps = int(t_max / dt)
    _, _, _, zt, vt = simulate_trajectories(simulator, [z0], [v0], t_max, dt, z_escape, True)
    return np.arange(n_steps) * dt, zt[0], vt[0]


simulate_trajectory_jit = simulate_trajectory


def simulate_trajectories_3d(simulator, r0_list: List[np.ndarray], v0_list: List[np.ndarray],
                             t_max: float, dt: float = 1e-6, r_escape: float = 0.015
                             ) -> List[Tuple[np.ndarray, np.ndarray, np.ndarray]]:
    """Per-axis 3D model: F_z = F(v_z, z), F_x = F(v_x, -x/2), F_y = F(v_y, -y/2);
    returns [(t, r (n, 3), v (n, 3))] per particle."""
    sim = as_gpu_simulator(simulator)
    n_steps = int(t_max / dt)
    r0 = np.asarray(r0_list, dtype=np.float64).reshape(-1, 3)
    v0 = np.asarray(v0_list, dtype=np.float64).reshape(-1, 3)
    o = sim.trajectories(r0, v0, dt, n_steps, ndim=3, r_escape=r_escape, save_full=True)
    rt = o["r_traj"].cpu().numpy()
    vt = o["v_traj"].cpu().numpy()
    t = np.arange(n_steps) * dt
    return [(t, rt[i], vt[i]) for i in range(r0.shape[0])]


def monte_carlo_temperature(simulator, n_particles: int = 100, t_max: float = 0.1,
                            dt: float = 1e-6, z_init_sigma: float = 1e-3,
                            v_init_sigma: float = 1.0, t_equilibrium: float = 0.05,
                            seed: int = 42) -> float:
    """T = m <v^2> / k_B over the post-equilibrium steps of an ensemble of 1D
    trajectories.  Initial conditions are the reference's: a
    numpy default_rng(seed) drawing z0 then v0 for each particle in turn."""
    sim = as_gpu_simulator(simulator)
    mass = sim.mol_data.mass
    n_steps = int(t_max / dt)
    i_eq = int(t_equilibrium / dt)
    rng = np.random.default_rng(seed)
    z0 = np.empty(n_particles)
    v0 = np.empty(n_particles)
    for i in range(n_particles):
        z0[i] = rng.normal(0, z_init_sigma)
        v0[i] = rng.normal(0, v_init_sigma)
    o = sim.trajectories(z0, v0, dt, n_steps, ndim=1, r_escape=0.015, i_eq=i_eq)
    vsq = o["vsq_sum"].cpu().numpy()
    ns = o["n_samp"].cpu().numpy()
    n_samples = ns.sum()
    if n_samples == 0:
        return float("inf")
    # the reference accumulates one running sum over particles in order
    total = 0.0
    for x in vsq:
        total += x
    return mass * (total / n_samples) / k_B


# ---------------------------------------------------------------- samplers
def sample_direction(rng=None) -> np.ndarray:
    """Unit vector uniform on the sphere (phi = 2 pi u1, cos(theta) = 2 u2 - 1)."""
    rng = np.random.default_rng() if rng is None else rng
    theta = 2.0 * math.pi * rng.random()
    z = 2.0 * rng.random() - 1.0
    rp = math.sqrt(max(0.0, 1.0 - z * z))
    return np.array([rp * math.cos(theta), rp * math.sin(theta), z])


def sample_maxwell_boltzmann(temperature, mass, n_particles=1, rng=None):
    """3D Maxwell-Boltzmann velocities: each component N(0, sqrt(k_B T / m))."""
    rng = np.random.default_rng() if rng is None else rng
    sigma = math.sqrt(k_B * temperature / mass) if temperature > 0 else 0.0
    v = rng.normal(0.0, sigma, size=(n_particles, 3)) if sigma > 0 else np.zeros((n_particles, 3))
    return v[0] if n_particles == 1 else v


def sample_maxwell_boltzmann_speed(temperature, mass, n_particles=1, rng=None):
    v = sample_maxwell_boltzmann(temperature, mass, n_particles, rng)
    return float(np.linalg.norm(v)) if n_particles == 1 else np.linalg.norm(v, axis=1)


def sample_gaussian_position(sigma, n_particles=1, rng=None):
    rng = np.random.default_rng() if rng is None else rng
    r = rng.normal(0.0, sigma, size=(n_particles, 3))
    return r[0] if n_particles == 1 else r


def sample_uniform_sphere(radius, n_particles=1, rng=None):
    """Positions uniform inside a sphere, by rejection from the enclosing cube."""
    rng = np.random.default_rng() if rng is None else rng
    out = np.zeros((n_particles, 3))
    for i in range(n_particles):
        while True:
            r = rng.uniform(-radius, radius, size=3)
            if np.linalg.norm(r) <= radius:
                out[i] = r
                break
    return out[0] if n_particles == 1 else out


def make_position_sampler(sigma=1e-3, method="gaussian"):
    rng = np.random.default_rng()
    if method == "gaussian":
        return lambda: sample_gaussian_position(sigma, 1, rng)
    if method == "uniform_sphere":
        return lambda: sample_uniform_sphere(sigma, 1, rng)
    raise ValueError(f"Unknown method: {method}")


def make_velocity_sampler(temperature, mass, method="maxwell_boltzmann"):
    """Callable returning one 3D velocity per call: Maxwell-Boltzmann at
    `temperature`, or zero ('fixed') (molmot/propagation/trajectories.py:413-446)."""
    rng = np.random.default_rng()
    if method == "maxwell_boltzmann":
        return lambda: sample_maxwell_boltzmann(temperature, mass, 1, rng)
    if method == "fixed":
        return lambda: np.zeros(3)
    raise ValueError(f"Unknown method: {method}")
