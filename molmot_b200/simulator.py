"""DC and RF MOT simulators backed by the GPU force kernels.

Mirror molmot/mot/simulator.py:17-162: ``force(v, z) -> (F, populations, R)``.
The RF MOT force is the average of its two half-cycles, phase 0 with +B' and
phase 1 with -B' (simulator.py:49-90).  ``force_points`` evaluates many
(v, z) points in one launch; the force-scan functions use it.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .constants import HBAR_JIT
from .engine import BeamSets, force_batch, pack_for, traj
from .fields import make_dc_mot_beams, make_rf_mot_beams


class _GPUSimulator:
    """Common machinery: the simulator is a weighted set of (beams, B') pairs."""

    hbar = HBAR_JIT
    uniform_fallback = False

    def param_sets(self) -> List[Tuple[list, float]]:
        raise NotImplementedError

    def _beam_sets(self) -> BeamSets:
        ps = self.param_sets()
        key = tuple((tuple((b.kdir_z, b.freq_offset, b.polarization, b.s0) for b in L), B)
                    for L, B in ps) + (self.Gamma_eff_factor,)
        if getattr(self, "_bs_key", None) != key:
            self._bs = BeamSets.from_beams([L for L, _ in ps], [B for _, B in ps],
                                           self.Gamma_eff_factor)
            self._bs_key = key
        return self._bs

    def force_points(self, v, z, precision="fp64"):
        """F, populations, R at points (v[i], z[i]) -- numpy arrays."""
        v = np.atleast_1d(np.asarray(v, dtype=np.float64))
        z = np.atleast_1d(np.asarray(z, dtype=np.float64))
        v, z = np.broadcast_arrays(v, z)
        n = v.size
        bs = self._beam_sets()
        ns = bs.n_sets
        out = force_batch(pack_for(self.mol_data), bs, np.tile(v.ravel(), ns),
                          np.tile(z.ravel(), ns), points_per_set=n, precision=precision,
                          hbar=self.hbar, uniform_fallback=self.uniform_fallback)
        F = out["F"].cpu().numpy().reshape(ns, n)
        P = out["pop"].cpu().numpy().reshape(ns, n, -1)
        R = out["R"].cpu().numpy().reshape(ns, n)
        if ns == 1:
            return F[0], P[0], R[0]
        return 0.5 * (F[0] + F[1]), 0.5 * (P[0] + P[1]), 0.5 * (R[0] + R[1])

    def force(self, v: float, z: float) -> Tuple[float, np.ndarray, float]:
        F, P, R = self.force_points([v], [z])
        return float(F[0]), P[0], float(R[0])

    def trajectories(self, r0, v0, dt, n_steps, ndim=1, r_escape=0.015, save_full=False,
                     i_eq=None, precision="fp64"):
        bs = self._beam_sets()
        return traj(pack_for(self.mol_data), bs, r0, v0, dt, n_steps, ndim=ndim,
                    n_avg=bs.n_sets, r_escape=r_escape, save_full=save_full, i_eq=i_eq,
                    precision=precision, hbar=self.hbar)


class RFMOTSimulator(_GPUSimulator):
    def __init__(self, mol_data, delta_Gamma: float = -1.0, s0: float = 1.0,
                 B_gradient: float = 0.16, Gamma_eff_factor: float = 1.0):
        self.mol_data = mol_data
        self.delta_Gamma = delta_Gamma
        self.s0 = s0
        self.B_gradient = B_gradient
        self.Gamma_eff_factor = Gamma_eff_factor

    def param_sets(self):
        b0 = make_rf_mot_beams(self.mol_data, delta_Gamma=self.delta_Gamma, s0=self.s0, phase=0)
        b1 = make_rf_mot_beams(self.mol_data, delta_Gamma=self.delta_Gamma, s0=self.s0, phase=1)
        return [(b0, self.B_gradient), (b1, -self.B_gradient)]


class DCMOTSimulator(_GPUSimulator):
    def __init__(self, mol_data, delta_Gamma: float = -0.20, split_Gamma: float = 0.70,
                 s0: float = 1.0, B_gradient: float = 0.16, Gamma_eff_factor: float = 1.0):
        self.mol_data = mol_data
        self.delta_Gamma = delta_Gamma
        self.split_Gamma = split_Gamma
        self.s0 = s0
        self.B_gradient = B_gradient
        self.Gamma_eff_factor = Gamma_eff_factor
        self._beams = make_dc_mot_beams(mol_data, delta_Gamma=delta_Gamma,
                                        split_Gamma=split_Gamma, s0=s0)

    def param_sets(self):
        return [(self._beams, self.B_gradient)]

    def update_beams(self):
        self._beams = make_dc_mot_beams(self.mol_data, delta_Gamma=self.delta_Gamma,
                                        split_Gamma=self.split_Gamma, s0=self.s0)


class BeamListSimulator(_GPUSimulator):
    """Any fixed beam list (for example a reference simulator's ``_beams``)."""

    def __init__(self, mol_data, beams, B_gradient, Gamma_eff_factor=1.0):
        self.mol_data = mol_data
        self._beams = list(beams)
        self.B_gradient = B_gradient
        self.Gamma_eff_factor = Gamma_eff_factor

    def param_sets(self):
        return [(self._beams, self.B_gradient)]


def as_gpu_simulator(sim) -> _GPUSimulator:
    """Accept molmot_b200 simulators and the reference's DC/RF simulator objects
    (same attributes) and return a GPU-backed equivalent."""
    if isinstance(sim, _GPUSimulator):
        return sim
    gef = getattr(sim, "Gamma_eff_factor", 1.0)
    if hasattr(sim, "_beams") and hasattr(sim, "B_gradient"):
        return BeamListSimulator(sim.mol_data, sim._beams, sim.B_gradient, gef)
    if all(hasattr(sim, a) for a in ("mol_data", "delta_Gamma", "s0", "B_gradient")):
        return RFMOTSimulator(sim.mol_data, sim.delta_Gamma, sim.s0, sim.B_gradient, gef)
    raise TypeError(f"cannot run simulator of type {type(sim).__name__} on the GPU: it needs "
                    "mol_data and either _beams + B_gradient (DC) or delta_Gamma + s0 + "
                    "B_gradient (RF)")
