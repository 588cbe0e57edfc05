"""SrOH molecular data: the ``MolecularData`` container and the CSV loader.

Mirrors molmot/molecules/sroh.py:87-174 (container and derived arrays) and
:486-592 (``load_sroh_from_julia``).  The nine CSV files under
``sroh_julia/`` are the reference's SrOH data (energies, transition dipoles,
Zeeman matrices) exactly as shipped in its julia_sim/ directory.

Derived quantities follow the reference bit for bit:
  d_squared[g, e, q] = |tdm[g, n_g + e, q]|**2          (numpy abs, then square)
  zeeman_z_diag      = Re diag(zeeman_z)
  omega_J32/J12      = mean(E_e) - mean(E_g[:8]) / mean(E_g[8:]) when n_g == 12,
                       otherwise both mean(E_e) - mean(E_g)
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from ..constants import amu, wavenumber

LAMBDA_NM = 687.0
LAMBDA_M = LAMBDA_NM * 1e-9
GAMMA_HZ = 6.4e6
GAMMA_RAD = 2.0 * math.pi * GAMMA_HZ
MASS_AMU = 105.0
MASS_KG = MASS_AMU * amu
K_WAVE = wavenumber(LAMBDA_M)

SROH_DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sroh_julia")


@dataclass
class MolecularData:
    """Level structure consumed by the rate-equation kernels.

    energies (n_states,) Hz; tdm (n_states, n_states, 3) complex with the
    polarisation index q = 0, 1, 2 for sigma-, pi, sigma+; zeeman_{x,y,z}
    (n_states, n_states) complex, scaled so that a field B (Gauss) shifts a
    level by B * Z * Gamma / (2 pi) Hz.  Ground states come first.
    """
    energies: np.ndarray
    tdm: np.ndarray
    zeeman_x: np.ndarray
    zeeman_y: np.ndarray
    zeeman_z: np.ndarray
    Gamma: float = GAMMA_RAD
    k: float = K_WAVE
    mass: float = MASS_KG
    wavelength: float = LAMBDA_M
    n_ground: int = 12
    n_excited: int = 4
    n_states: int = 16
    d_squared: Optional[np.ndarray] = field(default=None, repr=False)
    zeeman_z_diag: Optional[np.ndarray] = field(default=None, repr=False)
    omega_J12: float = 0.0
    omega_J32: float = 0.0
    omega_mean: float = 0.0

    def __post_init__(self):
        n_g, n_e = self.n_ground, self.n_excited
        if self.d_squared is None:
            block = np.asarray(self.tdm)[:n_g, n_g:n_g + n_e, :]
            self.d_squared = np.abs(block) ** 2
        if self.zeeman_z_diag is None:
            self.zeeman_z_diag = np.real(np.diag(self.zeeman_z))
        E_g = self.energies[:n_g]
        E_e_mean = np.mean(self.energies[n_g:])
        if n_g == 12:
            # ground ordering of the SrOH data: 8 J=3/2 levels, then 4 J=1/2
            E_J32, E_J12 = np.mean(E_g[:8]), np.mean(E_g[8:])
        else:
            E_J32 = E_J12 = np.mean(E_g)
        self.omega_J12 = E_e_mean - E_J12
        self.omega_J32 = E_e_mean - E_J32
        self.omega_mean = E_e_mean - np.mean(E_g)


def _read_table(path: str) -> np.ndarray:
    return np.loadtxt(path)


def load_sroh_from_julia(data_dir: Optional[str] = None, verbose: bool = False) -> MolecularData:
    """Load SrOH from the reference's CSV layout.

    sroh_energies.csv: 16 energies (Hz).  sroh_tdm_{re,im}.csv: 48 x 16,
    row 3*state + q holds tdm[state, :, q].  sroh_zeeman_{x,y,z}_{re,im}.csv:
    16 x 16.  ``data_dir`` defaults to the copy packaged with molmot_b200.
    """
    d = SROH_DATA_DIR if data_dir is None else data_dir
    n_s, n_g, n_e = 16, 12, 4
    E = _read_table(os.path.join(d, "sroh_energies.csv"))
    if E.shape != (n_s,):
        raise ValueError(f"expected {n_s} energies, got shape {E.shape}")
    t_re = _read_table(os.path.join(d, "sroh_tdm_re.csv"))
    t_im = _read_table(os.path.join(d, "sroh_tdm_im.csv"))
    if t_re.shape != (3 * n_s, n_s) or t_im.shape != t_re.shape:
        raise ValueError(f"TDM table shape {t_re.shape}, expected {(3 * n_s, n_s)}")
    flat = t_re + 1j * t_im
    # row 3*i + q -> tdm[i, :, q]
    tdm = flat.reshape(n_s, 3, n_s).transpose(0, 2, 1).copy()

    def zeeman(axis):
        re = _read_table(os.path.join(d, f"sroh_zeeman_{axis}_re.csv"))
        im = _read_table(os.path.join(d, f"sroh_zeeman_{axis}_im.csv"))
        if re.shape != (n_s, n_s) or im.shape != (n_s, n_s):
            raise ValueError(f"Zeeman {axis} shape {re.shape}")
        return re + 1j * im

    mol = MolecularData(energies=E, tdm=tdm, zeeman_x=zeeman("x"), zeeman_y=zeeman("y"),
                        zeeman_z=zeeman("z"), Gamma=GAMMA_RAD, k=K_WAVE, mass=MASS_KG,
                        wavelength=LAMBDA_M, n_ground=n_g, n_excited=n_e, n_states=n_s)
    if verbose:
        print(f"SrOH: {n_g} ground + {n_e} excited levels from {d}")
    return mol
