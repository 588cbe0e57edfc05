"""Seeded synthetic molecules for uneven batches and 3D tests.

Each molecule has n_ground ground and n_excited excited levels:
  * energies: ground hyperfine energies U[0, 200] MHz, excited ones
    U[0, 200] MHz above a fixed optical transition (SrOH's, 4.32e14 Hz);
  * transition dipoles: complex Gaussian tdm[g, n_g + e, q], rescaled per
    excited state so that its branching ratios over ground states follow a
    Dirichlet(1) draw;
  * Zeeman: a g-factor U[-1, 1] per level and a projection m from
    {-2 .. 2} give the z diagonal g m; the x and y ground blocks are random
    Hermitian matrices of the same scale, so B.Z has a non-degenerate
    spectrum for generic field directions (the 3D eigenbasis is unique).
"""
from __future__ import annotations

import numpy as np

from .sroh import GAMMA_RAD, K_WAVE, LAMBDA_M, MASS_KG, MolecularData

TRANSITION_HZ = 4.32035108e14


def synthetic_molecule(n_ground: int, n_excited: int, seed: int) -> MolecularData:
    rng = np.random.default_rng(seed)
    n_g, n_e = int(n_ground), int(n_excited)
    n_s = n_g + n_e
    E = np.concatenate([rng.uniform(0.0, 200e6, n_g),
                        TRANSITION_HZ + rng.uniform(0.0, 200e6, n_e)])
    tdm = np.zeros((n_s, n_s, 3), dtype=complex)
    for e in range(n_e):
        d = rng.normal(size=(n_g, 3)) + 1j * rng.normal(size=(n_g, 3))
        cur = np.sum(np.abs(d) ** 2, axis=1)
        target = rng.dirichlet(np.ones(n_g))
        d *= np.sqrt(target / cur)[:, None]
        tdm[:n_g, n_g + e, :] = d
        tdm[n_g + e, :n_g, :] = np.conj(d)
    gfac = rng.uniform(-1.0, 1.0, n_s)
    m = rng.integers(-2, 3, n_s).astype(float)
    Zz = np.diag(gfac * m).astype(complex)
    Zx = np.zeros((n_s, n_s), dtype=complex)
    Zy = np.zeros((n_s, n_s), dtype=complex)
    for Z in (Zx, Zy):
        A = rng.normal(size=(n_g, n_g)) + 1j * rng.normal(size=(n_g, n_g))
        Z[:n_g, :n_g] = 0.25 * (A + A.conj().T) / np.sqrt(n_g)
    Zz[:n_g, :n_g] += 0.1 * np.diag(rng.normal(size=n_g))
    return MolecularData(energies=E, tdm=tdm, zeeman_x=Zx, zeeman_y=Zy, zeeman_z=Zz,
                         Gamma=GAMMA_RAD, k=K_WAVE, mass=MASS_KG, wavelength=LAMBDA_M,
                         n_ground=n_g, n_excited=n_e, n_states=n_s)


def dc_beams_for(mol, detunings_hz=(-8e6, -4e6, -8e6, -4e6), s0=(2.0, 1.0, 2.0, 1.0)):
    """A 4-frequency pattern for any molecule: two frequencies below the mean
    transition of the lower half of the ground levels and two below that of
    the upper half, alternating sigma+/sigma-, each as a +z/-z pair (8 beams).
    Returns (kdir, freq, pol, s0) arrays of length 8."""
    n_g = mol.n_ground
    E = mol.energies
    Ee = np.mean(E[n_g:])
    lo = Ee - np.mean(E[: max(1, n_g // 2)])
    hi = Ee - np.mean(E[n_g // 2: n_g]) if n_g > 1 else lo
    refs = [lo, lo, hi, hi]
    pols = [2, 0, 2, 0]
    kdir, freq, pol, s0b = [], [], [], []
    for f0, d, q, s in zip(refs, detunings_hz, pols, s0):
        for k in (1.0, -1.0):
            kdir.append(k)
            freq.append(f0 + d)
            pol.append(q if k > 0 else 2 - q)
            s0b.append(s)
    return np.array(kdir), np.array(freq), np.array(pol, dtype=np.int32), np.array(s0b)
