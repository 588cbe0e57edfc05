"""Algorithmic work per steady-state point, for roofline figures.

Convention: +, -, *, / each count as one FLOP, over the reference's numba
algorithm (molmot/obe/rate_equations_jit.py:18-145), with A the number of
active (beam, ground, excited) triples (d2 >= 1e-15 for the beam's
polarisation).  For SrOH with the 8-beam DC MOT, A = 96 and the total is
about 4.82 kFLOP per point.

flops_per_point counts the plain form (the reference's algorithm);
flops_reduced counts the FP32-bulk and FP64-reduced forms, which solve the
populations through the excited-state chain.
"""
from __future__ import annotations

import numpy as np


def active_triples(d_squared, pols) -> int:
    """A = number of (b, g, e) with d2[g, e, pol_b] >= 1e-15."""
    d2 = np.asarray(d_squared)
    return int(sum(int((d2[:, :, int(q)] >= 1e-15).sum()) for q in np.asarray(pols).ravel()))


def flops_per_point(n_g: int, n_e: int, n_b: int, A: int):
    """(fp64_flops, 0.0) of one point of the plain form (the reference's
    algorithm, all FP64)."""
    n_s = n_g + n_e
    prelude = 3 * n_s + 3 * n_b
    rates = 18 * A
    sat = 2 * n_g + 2 * n_g * n_e
    build = n_g * n_e + 2 * n_g * n_g * n_e
    lu = sum(m * (2 * m + 5) for m in range(n_g))
    back = n_g * n_g
    tail = 2 * n_g + 4 * n_g * n_e
    return float(prelude + rates + sat + build + lu + back + tail), 0.0


def flops_reduced(n_g: int, n_e: int, A: int):
    """(fp64_flops, fp32_flops) of one point of the FP32-bulk form, which
    solves the populations through the excited-state chain.

    Per active triple: FP32 u = u0 + uv v - uB B (2 FMA), 1 + u^2 (1 FMA),
    L = 1/(1 + u^2), rate = c1 L, s += c2 L (1 FMA): 10 FLOP; FP64 sums of the
    rate and of hk * rate: 3 FLOP.  Per ground state (FP64): r_g, 1/r_g, F_g/r_g,
    (1 + s_g)/r_g, R[g,e]/r_g, the K update (n_e^2 FMA) and two n_e-vector
    updates.  The chain solve (state reduction of n_e states) and the final
    three n_e dot products."""
    fp32 = 10 * A
    per_g = (n_e - 1) + 1 + 1 + 2 + n_e + 2 * n_e * n_e + 4 * n_e
    gth = sum((k - 1) + 1 + k + 2 * k * k for k in range(1, n_e)) + sum(2 * k for k in range(1, n_e))
    final = 3 * 2 * n_e + 3
    fp64 = 3 * A + n_g * per_g + gth + final
    return float(fp64), float(fp32)


def flops_reduced64(n_g: int, n_e: int, A: int) -> float:
    """FP64 FLOP of one point of the FP64-reduced form (the uneven batch's
    form for molecules the reduction covers): the plain form's rates
    (18 FLOP per active triple) and the excited-chain solve of
    flops_reduced."""
    fp64, _ = flops_reduced(n_g, n_e, A)
    return float(fp64 - 3 * A + 18 * A)


def reduction_covers(d_squared, pols) -> bool:
    """Host twin of the reduced form's structural check for one parameter
    set: every ground state has an active triple, and the excited-state chain
    (e' -> e when e' decays to a ground state that a beam excites to e) is
    strongly connected."""
    d2 = np.asarray(d_squared)
    n_g, n_e, _ = d2.shape
    act = np.zeros((n_g, n_e), dtype=bool)
    for q in np.asarray(pols).ravel():
        act |= d2[:, :, int(q)] >= 1e-15
    if not act.any(axis=1).all():
        return False
    decays = d2.sum(axis=2).T > 0  # [e, g]: e decays to g
    reach = np.eye(n_e, dtype=bool) | (decays.astype(int) @ act.astype(int) > 0)
    for k in range(n_e):
        reach |= reach[:, [k]] & reach[[k], :]
    return bool(reach.all())


def uneven_flops(mols, counts, pols) -> float:
    """Algorithmic FP64 FLOP of an uneven batch: per molecule its points times
    the FP64-reduced count, or the plain count where the reduction does not
    cover it (the elimination then runs)."""
    total = 0.0
    for m, c, p in zip(mols, counts, pols):
        A = active_triples(m.d_squared, p)
        if reduction_covers(m.d_squared, p):
            total += c * flops_reduced64(m.n_ground, m.n_excited, A)
        else:
            total += c * flops_per_point(m.n_ground, m.n_excited, len(np.asarray(p).ravel()), A)[0]
    return total
