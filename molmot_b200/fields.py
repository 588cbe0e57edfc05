"""Laser beams of the 1D rate-equation model and the MOT beam builders.

Mirrors molmot/obe/fields.py:22-58 (``LaserBeam``), :76-136
(``make_rf_mot_beams``) and :139-202 (``make_dc_mot_beams``).  Frequencies
are absolute (Hz); polarisation is the spherical index q = 0, 1, 2 for
sigma-, pi, sigma+.  A retro-reflected (-z) beam has its circular
polarisation mirrored (q -> 2 - q), pi stays pi.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List

import numpy as np


@dataclass
class LaserBeam:
    direction: np.ndarray
    freq_offset: float
    polarization: int
    s0: float

    def __post_init__(self):
        if isinstance(self.direction, (int, float)):
            self.direction = np.array([0.0, 0.0, float(self.direction)])
        self.direction = np.asarray(self.direction, dtype=float)

    @property
    def kdir_z(self) -> float:
        """z-projection of the propagation direction (the 1D model's k sign)."""
        return float(self.direction[2])


@dataclass
class MOTConfig:
    beams: List[LaserBeam] = field(default_factory=list)
    B_gradient: float = 0.0


def _retro(q: int) -> int:
    return 2 - q if q != 1 else 1


def _pair(freq: float, q_fwd: int, s0: float) -> List[LaserBeam]:
    return [LaserBeam(np.array([0.0, 0.0, 1.0]), freq, q_fwd, s0),
            LaserBeam(np.array([0.0, 0.0, -1.0]), freq, _retro(q_fwd), s0)]


def make_dc_mot_beams(mol_data, delta_Gamma: float = -0.20, split_Gamma: float = 0.70,
                      s0: float = 1.0, n_freq: int = 4) -> List[LaserBeam]:
    """Four-frequency DC MOT: for each spin-rotation manifold (J=3/2, J=1/2)
    a sigma+ component at detuning + split and a sigma- one at detuning -
    split, each as a +z/-z beam pair (8 beams)."""
    G = mol_data.Gamma
    d_hz = delta_Gamma * G / (2.0 * math.pi)
    s_hz = split_Gamma * G / (2.0 * math.pi)
    comps = [(mol_data.omega_J32 + d_hz + s_hz, 2),
             (mol_data.omega_J32 + d_hz - s_hz, 0),
             (mol_data.omega_J12 + d_hz + s_hz, 2),
             (mol_data.omega_J12 + d_hz - s_hz, 0)]
    beams: List[LaserBeam] = []
    for f, q in comps:
        beams += _pair(f, q, s0)
    return beams


def make_rf_mot_beams(mol_data, delta_Gamma: float = -1.0, s0: float = 1.0,
                      phase: int = 0, n_sidebands: int = 2) -> List[LaserBeam]:
    """RF MOT half-cycle: the J=3/2 and J=1/2 sidebands carry opposite
    circular polarisations, both flipped between phase 0 and phase 1."""
    d_hz = delta_Gamma * mol_data.Gamma / (2.0 * math.pi)
    f32 = mol_data.omega_J32 + d_hz
    f12 = mol_data.omega_J12 + d_hz
    q32, q12 = (2, 0) if phase == 0 else (0, 2)
    return _pair(f32, q32, s0) + _pair(f12, q12, s0)


def beam_arrays(beams: List[LaserBeam]):
    """Flat (kdir_z, freq, pol, s0) float64 arrays of a beam list."""
    return (np.array([b.kdir_z for b in beams], dtype=np.float64),
            np.array([b.freq_offset for b in beams], dtype=np.float64),
            np.array([b.polarization for b in beams], dtype=np.int32),
            np.array([b.s0 for b in beams], dtype=np.float64))
