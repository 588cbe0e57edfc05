"""3D MOT simulator on the GPU (drop-in for molmot/mot/simulator_3d.py).

``rate_eq_force_3d`` / ``MOTSimulator3D.force_3d`` evaluate the 3D
rate-equation force with the sm_100a kernel (quadrupole field, ground-state
Zeeman eigenbasis from a Jacobi eigensolver, per-beam local polarisation
weights, Gaussian beam profiles).  ``simulate_trajectory_3d`` and
``simulate_ensemble_3d`` run the leapfrog integrator for all particles and
all steps in one launch, optionally with photon-recoil kicks (seeded,
counter-based, resumable).  The reference's 3D path uses CODATA hbar; so do
these functions unless ``hbar`` is given.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np

from .constants import hbar as HBAR_CODATA
from .engine import beam_sets_3d, force3d_batch, pack_for, traj3d


class Beam3D:
    """One laser beam in 3D: unit k, absolute frequency (Hz), lab-frame
    polarisation index q_lab (0, 1, 2 = sigma-, pi, sigma+), s0, 1/e^2 radius
    (None: plane wave) -- molmot/mot/simulator_3d.py:32-56."""

    def __init__(self, k_hat, freq, q_lab, s0, beam_radius=None):
        self.k_hat = np.asarray(k_hat, dtype=float)
        self.k_hat = self.k_hat / np.linalg.norm(self.k_hat)
        self.freq = freq
        self.q_lab = q_lab
        self.s0 = s0
        self.beam_radius = beam_radius


_DIRS = [np.array([1, 0, 0]), np.array([-1, 0, 0]), np.array([0, 1, 0]), np.array([0, -1, 0]),
         np.array([0, 0, 1]), np.array([0, 0, -1])]


def make_6beam_config(mol_data, beam_pairs, beam_radius=10e-3) -> List[Beam3D]:
    """Each beam pair dict (freq, q_fwd, q_bwd, s0) becomes beams along
    +x, -x, +y, -y, +z, -z; forward (+) beams take q_fwd, backward ones q_bwd
    (simulator_3d.py:59-105)."""
    beams = []
    for bp in beam_pairs:
        for i, d in enumerate(_DIRS):
            beams.append(Beam3D(d, bp["freq"], bp["q_fwd"] if i % 2 == 0 else bp["q_bwd"],
                                bp["s0"], beam_radius))
    return beams


def make_beam_pairs_dc4(mol_data, delta_Gamma, split_Gamma, s0):
    """Four-frequency DC MOT pairs (molmot/obe/obe_subdoppler.py:308-323)."""
    G = mol_data.Gamma
    d = delta_Gamma * G / (2 * np.pi)
    sp = split_Gamma * G / (2 * np.pi)
    return [{"freq": mol_data.omega_J32 + d + sp, "q_fwd": 2, "q_bwd": 0, "s0": s0},
            {"freq": mol_data.omega_J32 + d - sp, "q_fwd": 0, "q_bwd": 2, "s0": s0},
            {"freq": mol_data.omega_J12 + d + sp, "q_fwd": 2, "q_bwd": 0, "s0": s0},
            {"freq": mol_data.omega_J12 + d - sp, "q_fwd": 0, "q_bwd": 2, "s0": s0}]


def make_beam_pairs_rf(mol_data, delta_Gamma, s0, phase=0):
    """RF MOT pairs of one switching phase (obe_subdoppler.py:289-305)."""
    d = delta_Gamma * mol_data.Gamma / (2 * np.pi)
    q32, q12 = (2, 0) if phase == 0 else (0, 2)
    return [{"freq": mol_data.omega_J32 + d, "q_fwd": q32, "q_bwd": 2 - q32, "s0": s0},
            {"freq": mol_data.omega_J12 + d, "q_fwd": q12, "q_bwd": 2 - q12, "s0": s0}]


def _beam_arrays(beams, beam_radius=None):
    kh = np.array([b.k_hat for b in beams])
    fq = np.array([b.freq for b in beams], dtype=float)
    q = np.array([b.q_lab for b in beams], dtype=np.int32)
    s0 = np.array([b.s0 for b in beams], dtype=float)
    rad = [beam_radius if beam_radius is not None else b.beam_radius for b in beams]
    return kh, fq, q, s0, rad


class _Beams3DCache:
    def __init__(self):
        self.key = None
        self.bs = None

    def get(self, beams, B, gef, beam_radius=None):
        kh, fq, q, s0, rad = _beam_arrays(beams, beam_radius)
        key = (kh.tobytes(), fq.tobytes(), q.tobytes(), s0.tobytes(), tuple(map(str, rad)), B, gef)
        if key != self.key:
            self.bs = beam_sets_3d(kh, fq, q, s0, rad, B, gef)
            self.key = key
        return self.bs


_cache = _Beams3DCache()


def rate_eq_force_3d_batch(mol_data, beams, r_arr, v_arr, B_gradient, Gamma_eff_factor=1.0,
                           beam_radius=None, hbar=None):
    """F [n, 3], R [n], populations [n, n_ground] at many points (one launch)."""
    bs = _cache.get(beams, float(B_gradient), float(Gamma_eff_factor), beam_radius)
    o = force3d_batch(pack_for(mol_data), bs, np.asarray(r_arr, dtype=float).reshape(-1, 3),
                      np.asarray(v_arr, dtype=float).reshape(-1, 3), hbar=hbar or HBAR_CODATA)
    return o["F"].cpu().numpy(), o["R"].cpu().numpy(), o["pop"].cpu().numpy()


def rate_eq_force_3d(mol_data, beams, r, v, B_gradient, Gamma_eff_factor=1.0, beam_radius=None):
    """(F (3,), R, populations) at one point -- simulator_3d.py:168-365."""
    F, R, P = rate_eq_force_3d_batch(mol_data, beams, [r], [v], B_gradient, Gamma_eff_factor,
                                     beam_radius)
    return F[0], float(R[0]), P[0]


class MOTSimulator3D:
    """3D MOT (simulator_3d.py:372-532) with GPU force and ensembles."""

    def __init__(self, mol_data, beam_config, B_gradient, s0=1.0, Gamma_eff_factor=1.0,
                 beam_radius=10e-3):
        self.mol_data = mol_data
        self.B_gradient = B_gradient
        self.Gamma_eff_factor = Gamma_eff_factor
        self.beam_radius = beam_radius
        self.mass = mol_data.mass
        if isinstance(beam_config, list) and beam_config:
            if isinstance(beam_config[0], dict):
                self.beams = make_6beam_config(mol_data, beam_config, beam_radius=beam_radius)
            elif hasattr(beam_config[0], "k_hat"):
                self.beams = beam_config
            else:
                raise ValueError("beam_config must be list of Beam3D or beam_pairs dicts")
        else:
            raise ValueError("beam_config must be a non-empty list")
        self._cache = _Beams3DCache()

    def _bs(self):
        return self._cache.get(self.beams, float(self.B_gradient), float(self.Gamma_eff_factor))

    def force_3d(self, r, v):
        """(F (3,), R_scatter, populations) -- the reference's return order."""
        o = force3d_batch(pack_for(self.mol_data), self._bs(), [r], [v], hbar=HBAR_CODATA)
        return o["F"][0].cpu().numpy(), float(o["R"][0].item()), o["pop"][0].cpu().numpy()

    def force_3d_batch(self, r_arr, v_arr):
        o = force3d_batch(pack_for(self.mol_data), self._bs(), r_arr, v_arr, hbar=HBAR_CODATA)
        return o["F"].cpu().numpy(), o["R"].cpu().numpy(), o["pop"].cpu().numpy()

    def run_ensemble(self, r0, v0, t_max, dt=1e-6, r_escape=0.015, kicks=False, seed=0,
                     save_full=False, step0=0):
        """Device-level ensemble run: dict of torch tensors (see engine.traj3d)."""
        n_steps = int(t_max / dt) if step0 == 0 else int(t_max)
        return traj3d(pack_for(self.mol_data), self._bs(), r0, v0, dt, n_steps, step0=step0,
                      r_escape=r_escape, kicks=kicks, seed=seed, hbar=HBAR_CODATA,
                      save_full=save_full)

    def simulate_trajectory_3d(self, r0, v0, t_max, dt=1e-6, r_escape=0.015, kicks=False, seed=0):
        """(t, r (n, 3), v (n, 3)) -- leapfrog, simulator_3d.py:443-504."""
        t, R, V = self.simulate_ensemble_arrays([r0], [v0], t_max, dt, r_escape, kicks, seed)
        return t, R[0], V[0]

    def simulate_ensemble_arrays(self, r0_list, v0_list, t_max, dt=1e-6, r_escape=0.015,
                                 kicks=False, seed=0):
        n_steps = int(t_max / dt)
        o = self.run_ensemble(np.asarray(r0_list, dtype=float), np.asarray(v0_list, dtype=float),
                              t_max, dt, r_escape, kicks, seed, save_full=True)
        return np.arange(n_steps) * dt, o["r_traj"].cpu().numpy(), o["v_traj"].cpu().numpy()

    def simulate_ensemble_3d(self, r0_list, v0_list, t_max, dt=1e-6, r_escape=0.015,
                             callback=None, kicks=False, seed=0):
        """[(t, r, v)] per particle, all integrated in one launch."""
        t, R, V = self.simulate_ensemble_arrays(r0_list, v0_list, t_max, dt, r_escape, kicks, seed)
        out = []
        for i in range(R.shape[0]):
            out.append((t, R[i], V[i]))
            if callback is not None:
                callback(i, t, R[i], V[i])
        return out


def compute_3d_force_map(simulator, axes="xz", n_points=50, v=None, extent=5e-3):
    """(coords1, coords2, F_a1, F_a2, R) on a plane through the trap
    (simulator_3d.py:539-595), one launch."""
    v = np.zeros(3) if v is None else np.asarray(v, dtype=float)
    a1, a2 = {"x": 0, "y": 1, "z": 2}[axes[0]], {"x": 0, "y": 1, "z": 2}[axes[1]]
    c1 = np.linspace(-extent, extent, n_points)
    c2 = np.linspace(-extent, extent, n_points)
    r = np.zeros((n_points, n_points, 3))
    r[:, :, a1] = c1[:, None]
    r[:, :, a2] = c2[None, :]
    F, R, _ = simulator.force_3d_batch(r.reshape(-1, 3), np.tile(v, (n_points * n_points, 1)))
    F = F.reshape(n_points, n_points, 3)
    return c1, c2, F[:, :, a1], F[:, :, a2], R.reshape(n_points, n_points)
