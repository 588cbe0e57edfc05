"""Algorithmic work per steady-state point, for roofline figures.

Convention: +, -, *, / each count as one FLOP, over the reference's numba
algorithm (molmot/obe/rate_equations_jit.py:18-145), with A the number of
active (beam, ground, excited) triples (d2 >= 1e-15 for the beam's
polarisation).  For SrOH with the 8-beam DC MOT, A = 96 and the total is
about 4.82 kFLOP per point.

The FP32-bulk form performs the per-triple rate work (18 A) and the
per-state shift/doppler prelude in FP32 and everything from the population
matrix on in FP64, plus the refinement step (residual 2 n_g^2 + triangular
solves n_g^2).
"""
from __future__ import annotations

import numpy as np


def active_triples(d_squared, pols) -> int:
    """A = number of (b, g, e) with d2[g, e, pol_b] >= 1e-15."""
    d2 = np.asarray(d_squared)
    return int(sum(int((d2[:, :, int(q)] >= 1e-15).sum()) for q in np.asarray(pols).ravel()))


def flops_per_point(n_g: int, n_e: int, n_b: int, A: int, refine: bool = False):
    """Returns (fp64_flops, fp32_flops) of one point.  With refine=False all
    work is FP64 (the plain form)."""
    n_s = n_g + n_e
    prelude = 3 * n_s + 3 * n_b
    rates = 18 * A
    sat = 2 * n_g + 2 * n_g * n_e
    build = n_g * n_e + 2 * n_g * n_g * n_e
    lu = sum(m * (2 * m + 5) for m in range(n_g))
    back = n_g * n_g
    tail = 2 * n_g + 4 * n_g * n_e
    if not refine:
        return float(prelude + rates + sat + build + lu + back + tail), 0.0
    fp32 = prelude + rates + sat
    fp64 = build + lu + back + tail + 3 * n_g * n_g
    return float(fp64), float(fp32)
