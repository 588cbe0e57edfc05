"""Force scans and MOT characterisation on the GPU (drop-in for
molmot/mot/force_scan.py:18-301).

Every function takes a simulator (molmot_b200's DCMOTSimulator /
RFMOTSimulator, or the reference's objects with the same attributes) and
evaluates all its points in one kernel launch instead of a Python loop:

* force_vs_z / force_vs_v             -- one launch over the scan
* spring_constant / damping_coefficient -- 2-point central differences
  k = -(F(z0+dz) - F(z0-dz)) / 2dz, alpha = -(F(dv) - F(-dv)) / 2dv
* capture_velocity                     -- every test velocity as one
  trajectory of the fused trajectory kernel; the answer is the last velocity
  before the first one that escapes, as the reference's sequential loop gives
* optimize_parameters                  -- all (delta, split) cells as parameter
  sets of one launch (4 finite-difference points per set)
* spring_constant_fit / damping_coefficient_fit -- least-squares slope over
  an n-point stencil (default 33), used by the gradient workload
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np

from .constants import k_B  # noqa: F401  (re-exported like the reference module)
from .engine import BeamSets, force_batch, pack_for
from .fields import make_dc_mot_beams, make_rf_mot_beams
from .simulator import as_gpu_simulator


def force_vs_z(simulator, z_arr: np.ndarray, v: float = 0.0
               ) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(F (Nz,), populations (Nz, n_ground), R (Nz,)) at velocity v."""
    sim = as_gpu_simulator(simulator)
    z_arr = np.asarray(z_arr, dtype=np.float64)
    return sim.force_points(np.full(z_arr.shape, float(v)), z_arr)


def force_vs_v(simulator, v_arr: np.ndarray, z: float = 0.0) -> np.ndarray:
    """F (Nv,) at position z."""
    sim = as_gpu_simulator(simulator)
    v_arr = np.asarray(v_arr, dtype=np.float64)
    return sim.force_points(v_arr, np.full(v_arr.shape, float(z)))[0]


def spring_constant(simulator, z0: float = 0.0, dz: float = 0.3e-3) -> float:
    """k = -dF/dz at z0 (N/m), central difference with step dz (v = 0)."""
    F = as_gpu_simulator(simulator).force_points([0.0, 0.0], [z0 + dz, z0 - dz])[0]
    return -(F[0] - F[1]) / (2.0 * dz)


def damping_coefficient(simulator, z0: float = 0.0, dv: float = 0.1) -> float:
    """alpha = -dF/dv at z0 (N s/m); divide by the mass for beta (1/s)."""
    F = as_gpu_simulator(simulator).force_points([dv, -dv], [z0, z0])[0]
    return -(F[0] - F[1]) / (2.0 * dv)


def _lsq_slope(x, F):
    x = np.asarray(x)
    xm = x.mean()
    return float(np.sum((x - xm) * (F - F.mean())) / np.sum((x - xm) ** 2))


def spring_constant_fit(simulator, z0: float = 0.0, half_width: float = 0.3e-3,
                        n: int = 33) -> float:
    """k = -slope of the least-squares line through F(z) at n points in
    z0 +- half_width (v = 0)."""
    z = z0 + np.linspace(-half_width, half_width, n)
    F = as_gpu_simulator(simulator).force_points(np.zeros(n), z)[0]
    return -_lsq_slope(z, F)


def damping_coefficient_fit(simulator, z0: float = 0.0, half_width: float = 0.1,
                            n: int = 33) -> float:
    """alpha = -slope of the least-squares line through F(v) at n points in
    +- half_width (z = z0)."""
    v = np.linspace(-half_width, half_width, n)
    F = as_gpu_simulator(simulator).force_points(v, np.full(n, z0))[0]
    return -_lsq_slope(v, F)


def capture_velocity(simulator, z_start: float = 3e-3, v_max: float = 15.0, dv: float = 0.5,
                     dt: float = 1e-6, n_steps: int = 5000, z_escape: float = 0.015) -> float:
    """Largest tested v0 (dv, 2 dv, ... <= v_max) such that a molecule starting
    at z_start with velocity -v0, and every slower one, stays within z_escape
    for n_steps Euler steps (molmot/mot/force_scan.py:130-190)."""
    sim = as_gpu_simulator(simulator)
    tests = []
    v_test = dv
    while v_test <= v_max:  # the same accumulation as the reference's loop
        tests.append(v_test)
        v_test += dv
    if not tests:
        return 0.0
    tests = np.array(tests)
    o = sim.trajectories(np.full(tests.size, float(z_start)), -tests, dt, n_steps + 1,
                         r_escape=z_escape)
    trapped = (o["n_actual"].cpu().numpy() == n_steps + 1)
    v_capture = 0.0
    for vt, ok in zip(tests, trapped):
        if not ok:
            break
        v_capture = float(vt)
    return v_capture


def optimize_parameters(mol_data, param_ranges: Dict[str, np.ndarray], B_gradient: float,
                        mot_type: str = "dc", s0: float = 1.0, dz: float = 0.3e-3,
                        dv: float = 0.1, verbose: bool = True, Gamma_eff_factor: float = 1.0
                        ) -> Dict:
    """Scan (detuning, split) for the DC MOT, or detuning for the RF MOT, and
    pick the largest spring constant with k > 0 and beta > 0
    (molmot/mot/force_scan.py:193-301).  One kernel launch for the whole scan."""
    delta_scan = np.asarray(param_ranges["delta"], dtype=np.float64)
    mass = mol_data.mass
    pack = pack_for(mol_data)
    # finite-difference points of every set: (v, z) = (0, +dz), (0, -dz), (+dv, 0), (-dv, 0)
    pv = np.array([0.0, 0.0, dv, -dv])
    pz = np.array([dz, -dz, 0.0, 0.0])
    if mot_type == "dc":
        split_scan = np.asarray(param_ranges.get("split", np.array([0.0])), dtype=np.float64)
        lists = [make_dc_mot_beams(mol_data, delta_Gamma=d, split_Gamma=sp, s0=s0)
                 for d in delta_scan for sp in split_scan]
        Bs = [B_gradient] * len(lists)
    elif mot_type == "rf":
        split_scan = None
        lists, Bs = [], []
        for d in delta_scan:
            lists += [make_rf_mot_beams(mol_data, delta_Gamma=d, s0=s0, phase=0),
                      make_rf_mot_beams(mol_data, delta_Gamma=d, s0=s0, phase=1)]
            Bs += [B_gradient, -B_gradient]
    else:
        raise ValueError(f"Unknown mot_type: {mot_type}")
    bs = BeamSets.from_beams(lists, Bs, Gamma_eff_factor)
    n = len(lists)
    out = force_batch(pack, bs, np.tile(pv, n), np.tile(pz, n), points_per_set=4,
                      want_pop=False, want_R=False)
    F = out["F"].cpu().numpy().reshape(n, 4)
    if mot_type == "rf":
        F = 0.5 * (F[0::2] + F[1::2])
    k = -(F[:, 0] - F[:, 1]) / (2.0 * dz)
    beta = -(F[:, 2] - F[:, 3]) / (2.0 * dv) / mass
    if mot_type == "dc":
        K_map = k.reshape(delta_scan.size, split_scan.size)
        beta_map = beta.reshape(delta_scan.size, split_scan.size)
        merit = K_map.copy()
        merit[K_map <= 0] = 0
        merit[beta_map <= 0] = 0
        ib = np.unravel_index(np.argmax(merit), merit.shape)
        if verbose:
            print(f"  scanned {n} (delta, split) cells in one launch; best delta="
                  f"{delta_scan[ib[0]]:.3f} split={split_scan[ib[1]]:.3f}")
        return {"delta_scan": delta_scan, "split_scan": split_scan, "K_map": K_map,
                "beta_map": beta_map, "delta_best": float(delta_scan[ib[0]]),
                "split_best": float(split_scan[ib[1]]), "k_best": float(K_map[ib]),
                "beta_best": float(beta_map[ib])}
    ib = int(np.argmax(k * (k > 0) * (beta > 0)))
    return {"delta_scan": delta_scan, "K_arr": k, "beta_arr": beta,
            "delta_best": float(delta_scan[ib]), "k_best": float(k[ib]),
            "beta_best": float(beta[ib])}
