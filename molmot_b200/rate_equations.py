"""Single-point rate-equation solvers with the reference's signatures.

``solve_rate_equations`` mirrors molmot/obe/rate_equations.py:24-191 (CODATA
hbar, uniform populations when every population clamps to zero),
``solve_rate_equations_jit`` mirrors molmot/obe/rate_equations_jit.py:148-165
(hbar = 1.0545718e-34, populations left at zero), and
``solve_rate_equations_auto`` mirrors :196-218, which dispatches to the JIT
form.  Each call is one GPU launch of one point; batched callers should use
``engine.force_batch`` or the simulators' ``force_points``.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .constants import HBAR_JIT, hbar as HBAR_CODATA
from .engine import BeamSets, force_batch, pack_for


def _one(mol_data, beams, v, z, B_gradient, Gamma_eff_factor, hbar, uniform):
    bs = BeamSets.from_beams(list(beams), float(B_gradient), Gamma_eff_factor)
    out = force_batch(pack_for(mol_data), bs, np.array([float(v)]), np.array([float(z)]),
                      hbar=hbar, uniform_fallback=uniform)
    return (float(out["F"][0].item()), out["pop"][0].cpu().numpy(), float(out["R"][0].item()))


def solve_rate_equations(mol_data, beams: List, v: float, z: float, B_gradient: float,
                         Gamma_eff_factor: float = 1.0) -> Tuple[float, np.ndarray, float]:
    """(force N, populations (n_ground,), scattering rate 1/s) -- Python-path semantics."""
    return _one(mol_data, beams, v, z, B_gradient, Gamma_eff_factor, HBAR_CODATA, True)


def solve_rate_equations_jit(mol_data, beams: List, v: float, z: float, B_gradient: float,
                             Gamma_eff_factor: float = 1.0) -> Tuple[float, np.ndarray, float]:
    """(force, populations, scattering rate) -- numba-core semantics."""
    return _one(mol_data, beams, v, z, B_gradient, Gamma_eff_factor, HBAR_JIT, False)


def solve_rate_equations_auto(mol_data, beams: List, v: float, z: float, B_gradient: float,
                              Gamma_eff_factor: float = 1.0) -> Tuple[float, np.ndarray, float]:
    """The reference dispatches to its JIT solver when numba is importable."""
    return solve_rate_equations_jit(mol_data, beams, v, z, B_gradient, Gamma_eff_factor)
