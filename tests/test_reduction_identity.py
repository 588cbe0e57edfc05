"""The identity behind the reduced forms, checked on the CPU (numpy, FP64).

The reference's steady state solves M p = 0 with sum(p) = 1, where
M[g', g] = sum_e R[g, e] BR[e, g'] - delta_gg' r_g and r_g = sum_e R[g, e]
(molmot/obe/rate_equations_jit.py:92-136).  Every column of M sums to zero,
so with the excitation fluxes n_e = sum_g R[g, e] p_g the balance reads
r_g p_g = sum_e BR[e, g] n_e, and n is the stationary vector of the
column-stochastic excited chain K[e, e'] = sum_g (R[g, e] / r_g) BR[e', g].
Then p_g = (sum_e BR[e, g] n_e) / r_g, normalised, and F = sum_g p_g F_g.
Here the rates are restated from the reference's formulas, the chain is
solved by state reduction, and F and p are compared with the reference's own
outputs (tests/golden/random_points.npz, _rate_eq_core) on 384 points of 24
parameter sets: 1e-12 of max|F| per set, 1e-12 absolute on p.
"""
import math

import numpy as np

from conftest import golden

HBAR = 1.0545718e-34


def _rates(mol, kdir, freq, pol, s0, Bg, v, z):
    """Saturated rates R[g, e] and per-ground forces F_g at one point, in the
    reference's formulas (rate_equations_jit.py:58-90)."""
    n_g, n_e = mol.n_ground, mol.n_excited
    G, k = mol.Gamma, mol.k
    E, zd, d2 = np.asarray(mol.energies), np.asarray(mol.zeeman_z_diag), np.asarray(mol.d_squared)
    B = Bg * z * 1e4
    Es = E + B * zd * G / (2 * math.pi)
    gh2 = (G / 2) ** 2
    R = np.zeros((n_g, n_e))
    Fg = np.zeros(n_g)
    s = np.zeros(n_g)
    for b in range(len(kdir)):
        fd = freq[b] + (-k * kdir[b] * v) / (2 * math.pi)
        for g in range(n_g):
            for e in range(n_e):
                dd = d2[g, e, int(pol[b])]
                if dd < 1e-15:
                    continue
                de = (fd - (Es[n_g + e] - Es[g])) * 2 * math.pi
                L = gh2 / (de * de + gh2)
                ru = (G / 2) * s0[b] * dd * L
                R[g, e] += ru
                Fg[g] += HBAR * k * kdir[b] * ru
                s[g] += s0[b] * dd * L
    sat = 1.0 / (1.0 + s)
    return R * sat[:, None], Fg * sat


def _branching(mol):
    d2 = np.asarray(mol.d_squared)
    tot = d2.sum(axis=(0, 2))
    return (d2.sum(axis=2) / np.where(tot > 1e-30, tot, 1.0)).T  # BR[e, g]


def _chain_stationary(K):
    """Stationary vector of the column-stochastic K (K[to, from]) by state
    reduction (Grassmann, Taksar and Heyman, 1985)."""
    n = K.shape[0]
    Q = K.T.copy()  # Q[i, j]: probability i -> j
    for m in range(n - 1, 0, -1):
        S = Q[m, :m].sum()
        Q[:m, m] /= S
        Q[:m, :m] += np.outer(Q[:m, m], Q[m, :m])
    pi = np.zeros(n)
    pi[0] = 1.0
    for m in range(1, n):
        pi[m] = pi[:m] @ Q[:m, m]
    return pi


def test_excited_chain_reduction_reproduces_reference(mol):
    g = golden("random_points.npz")
    BR = _branching(mol)
    n_sets, npt = int(g["n_sets"]), int(g["n_pts"])
    F = np.zeros(n_sets * npt)
    P = np.zeros((n_sets * npt, mol.n_ground))
    for i in range(n_sets * npt):
        R, Fg = _rates(mol, g["kdir"][i], g["freq"][i], g["pol"][i], g["s0"][i], g["B"][i],
                       g["v"][i], g["z"][i])
        r = R.sum(axis=1)
        K = (R / r[:, None]).T @ BR.T  # K[e, e'] = sum_g a[g, e] BR[e', g]
        n = _chain_stationary(K)
        p = (BR.T @ n) / r
        p /= p.sum()
        F[i], P[i] = p @ Fg, p
    Fr = g["F_jit"].reshape(n_sets, npt)
    err = np.abs(F.reshape(n_sets, npt) - Fr).max(axis=1) / np.abs(Fr).max(axis=1)
    assert err.max() < 1e-12, err.max()
    assert np.abs(P - g["p_jit"]).max() < 1e-12


def _reduced_force_and_grad(mol, kdir, freq, pol, s0, Bg, v, z):
    """F and dF/dfreq_b by the reduced adjoint, restated in numpy: with
    u = (cf - F cw) / norm and lambda solving (I - K)^T lambda = u on the
    excited states 1.. (lambda_0 = 0), dF = sum_g [y_g sum_e lambda_e da_ge
    + (y_g / norm) dphi_g - (F y_g / norm) dw_g], through the unsaturated rate
    sums of each (g, e), the force sums f_g and the saturation sums s_g."""
    n_g, n_e = mol.n_ground, mol.n_excited
    G, k = mol.Gamma, mol.k
    E, zd, d2 = np.asarray(mol.energies), np.asarray(mol.zeeman_z_diag), np.asarray(mol.d_squared)
    BR = _branching(mol)
    Es = E + Bg * z * 1e4 * zd * G / (2 * math.pi)
    gh2 = (G / 2) ** 2
    nb = len(kdir)
    trips = []  # (g, e, b, c1, c2, hk, L, dL/dfreq)
    Ru = np.zeros((n_g, n_e)); f = np.zeros(n_g); s = np.zeros(n_g)
    for b in range(nb):
        fd = freq[b] + (-k * kdir[b] * v) / (2 * math.pi)
        for g in range(n_g):
            for e in range(n_e):
                dd = d2[g, e, int(pol[b])]
                if dd < 1e-15:
                    continue
                de = (fd - (Es[n_g + e] - Es[g])) * 2 * math.pi
                den = de * de + gh2
                L = gh2 / den
                dL = -2 * de * L / den * 2 * math.pi
                c1, c2, hk = (G / 2) * s0[b] * dd, s0[b] * dd, HBAR * k * kdir[b]
                trips.append((g, e, b, c1, c2, hk, L, dL))
                Ru[g, e] += c1 * L; f[g] += hk * c1 * L; s[g] += c2 * L
    r = Ru.sum(axis=1)
    a = Ru / r[:, None]
    phi, w = f / r, (1 + s) / r
    K = a.T @ BR.T
    cw, cf = BR @ w, BR @ phi
    pi = _chain_stationary(K)
    nrm = cw @ pi
    F = (cf @ pi) / nrm
    u = (cf - F * cw) / nrm
    lam = np.zeros(n_e)
    A = np.eye(n_e) - K.T
    lam[1:] = np.linalg.solve(A[1:, 1:], u[1:])
    y = BR.T @ pi
    Lam = a @ lam
    grad = np.zeros(nb)
    for g, e, b, c1, c2, hk, L, dL in trips:
        alpha = y[g] / r[g] * (lam[e] - Lam[g] - phi[g] / nrm + w[g] * F / nrm)
        beta = y[g] / (nrm * r[g])
        gamma = -F * y[g] / (nrm * r[g])
        grad[b] += (alpha * c1 + beta * hk * c1 + gamma * c2) * dL
    return F, grad


def test_reduced_adjoint_matches_central_differences(mol):
    """The adjoint of the chain reduction (the formulas of the FP64-reduced
    adjoint kernel) against central differences of the same numpy model,
    with frequency steps of 10 kHz: 2e-5 of the largest component.  The
    difference quotient itself is good to about (h / linewidth)^2 ~ 8e-6,
    and smaller steps meet the model's 1/16 Hz resolution of the
    Doppler-shifted frequency (~4.3e14 Hz); an error in the formulas shows at
    order one."""
    import bench
    kd, fr, po, s0, B = bench.make_params(mol, 3, 21)
    rng = np.random.default_rng(22)
    for i in range(3):
        v, z = rng.uniform(-5, 5), rng.uniform(-5e-3, 5e-3)
        F, grad = _reduced_force_and_grad(mol, kd[i], fr[i], po[i], s0[i], B[i], v, z)
        fd = np.zeros_like(grad)
        for b in range(len(grad)):
            fp, fm = fr[i].copy(), fr[i].copy()
            fp[b] += 1e4
            fm[b] -= 1e4
            h2 = fp[b] - fm[b]
            fd[b] = (_reduced_force_and_grad(mol, kd[i], fp, po[i], s0[i], B[i], v, z)[0]
                     - _reduced_force_and_grad(mol, kd[i], fm, po[i], s0[i], B[i], v, z)[0]) / h2
        assert np.abs(grad - fd).max() <= 2e-5 * np.abs(fd).max(), (grad, fd)
