"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the reference's 3D
rate-equation force and leapfrog integrator, plus the counter-based RNG and
photon-recoil kick model of molmot_b200's 3D trajectory kernel.

Reference (paths within the molmot project):
  molmot/mot/simulator_3d.py:112-165  _decompose_polarization_local
  molmot/mot/simulator_3d.py:168-365  rate_eq_force_3d
  molmot/mot/simulator_3d.py:443-504  MOTSimulator3D.simulate_trajectory_3d
The eigen-decomposition uses numpy.linalg.eigh as the reference does.  Pinned
against the reference's own outputs (tests/golden/force3d_golden.npz,
traj3d_golden.npz, generated by tests/golden/make_golden.py).

Recoil kicks (not in the reference's rate-equation integrators; the
B200 build's model): after each velocity update, N ~ Poisson(R dt)
scattering events, R the local scattering rate; the velocity receives
v_rec * (sum of 2N isotropic unit vectors) -- one absorption fluctuation and
one spontaneous emission per event, zero mean.  Random numbers:
Philox4x32-10 (Salmon et al., SC'11) keyed by the seed, counter
(particle, step, draw, 0).
"""
from __future__ import annotations

import math

import numpy as np

HBAR_CODATA = 1.054571817e-34


def pol_weights(q_lab: int, B_hat: np.ndarray) -> np.ndarray:
    """|d^1_{m' m}(theta)|^2 column for m = q_lab - 1, normalised (simulator_3d.py:112-165)."""
    n = np.linalg.norm(B_hat)
    if n < 1e-15:
        return np.array([1.0 / 3.0] * 3)
    Bh = B_hat / n
    ct = np.clip(Bh[2], -1.0, 1.0)
    st = np.sin(np.arccos(ct))
    m = np.array([[((1 + ct) / 2) ** 2, (st / np.sqrt(2)) ** 2, ((1 - ct) / 2) ** 2],
                  [(st / np.sqrt(2)) ** 2, ct ** 2, (st / np.sqrt(2)) ** 2],
                  [((1 - ct) / 2) ** 2, (st / np.sqrt(2)) ** 2, ((1 + ct) / 2) ** 2]])
    w = m[:, q_lab].copy()
    s = w.sum()
    if s > 1e-15:
        w /= s
    return w


def force3d(mol, khat, freq, q_lab, s0, radius, r, v, B_gradient, Gamma_eff=1.0,
            hbar=HBAR_CODATA, want_rates=False):
    """(F (3,), R, p (n_g,)) at one point; khat [n_b, 3], radius [n_b] (<= 0 or
    nan: plane wave)."""
    r = np.asarray(r, dtype=float)
    v = np.asarray(v, dtype=float)
    G, k = mol.Gamma, mol.k
    n_g, n_e = mol.n_ground, mol.n_excited
    B = np.array([-B_gradient * r[0] / 2.0 * 1e4, -B_gradient * r[1] / 2.0 * 1e4,
                  B_gradient * r[2] * 1e4])
    Bm = np.linalg.norm(B)
    B_hat = B / Bm if Bm > 1e-10 else np.array([0.0, 0.0, 1.0])
    H = (B[0] * mol.zeeman_x[:n_g, :n_g] + B[1] * mol.zeeman_y[:n_g, :n_g]
         + B[2] * mol.zeeman_z[:n_g, :n_g])
    lam, U = np.linalg.eigh(0.5 * (H + H.conj().T))
    Es_g = mol.energies[:n_g] + lam * G / (2 * np.pi)
    Es_e = mol.energies[n_g:] + B[2] * np.real(np.diag(mol.zeeman_z[n_g:, n_g:])) * G / (2 * np.pi)
    d_bare = np.abs(mol.tdm[:n_g, n_g:n_g + n_e, :])          # [g, e, q]
    d_sq = np.abs(np.einsum("ga,geq->aeq", U.conj(), d_bare)) ** 2
    BR = np.zeros((n_e, n_g))
    for ie in range(n_e):
        tot = np.sum(d_sq[:, ie, :])
        if tot > 1e-30:
            BR[ie] = np.sum(d_sq[:, ie, :], axis=1) / tot
    gh = G / 2.0
    n_b = len(freq)
    s_tot = np.zeros(n_g)
    Rb = np.zeros((n_b, n_g, n_e))
    mask = d_sq >= 1e-15
    om = Es_e[None, :] - Es_g[:, None]                        # [g, e]
    for b in range(n_b):
        dop = -k * np.dot(khat[b], v) / (2 * np.pi)
        gf = 1.0
        if radius[b] is not None and np.isfinite(radius[b]) and radius[b] > 0:
            rp = np.dot(r, khat[b])
            rps = max(np.dot(r, r) - rp ** 2, 0.0)
            gf = np.exp(-2.0 * rps / radius[b] ** 2)
        w = pol_weights(int(q_lab[b]), B_hat)
        de = (freq[b] + dop - om) * 2 * np.pi
        L = gh ** 2 / (de ** 2 + gh ** 2)
        rs = np.sum(np.where(mask, w[None, None, :] * d_sq * L[:, :, None], 0.0), axis=2)
        s_tot += s0[b] * gf * rs.sum(axis=1)
        Rb[b] = rs * s0[b] * gf
    rate = gh * Rb * Gamma_eff / (1.0 + s_tot)[None, :, None]
    Rs = rate.sum(axis=0)
    M = np.zeros((n_g, n_g))
    for ig in range(n_g):
        M[ig, ig] -= Rs[ig].sum()
        M[ig, :] += Rs @ BR[:, ig]
    M[-1, :] = 1.0
    rhs = np.zeros(n_g)
    rhs[-1] = 1.0
    try:
        p = np.linalg.solve(M, rhs)
    except np.linalg.LinAlgError:
        p = np.ones(n_g) / n_g
    p = np.maximum(p, 0.0)
    ps = p.sum()
    p = p / ps if ps > 0 else np.ones(n_g) / n_g
    per_beam = np.einsum("bge,g->b", rate, p)
    F = hbar * k * np.einsum("b,bx->x", per_beam, np.asarray(khat))
    Rsc = float(per_beam.sum())
    if want_rates:
        return F, Rsc, p, lam, U
    return F, Rsc, p


# ------------------------------------------------------------------ Philox
_M0, _M1 = 0xD2511F53, 0xCD9E8D57
_W0, _W1 = 0x9E3779B9, 0xBB67AE85
_MASK = 0xFFFFFFFF


def philox4x32_10(counter, key):
    """Philox4x32 with 10 rounds on python ints; counter 4 words, key 2 words."""
    c0, c1, c2, c3 = [int(x) & _MASK for x in counter]
    k0, k1 = [int(x) & _MASK for x in key]
    for _ in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & _MASK, p1 & _MASK, ((p0 >> 32) ^ c3 ^ k1) & _MASK, p0 & _MASK
        k0 = (k0 + _W0) & _MASK
        k1 = (k1 + _W1) & _MASK
    return c0, c1, c2, c3


def uniforms(seed, particle, step, draw):
    """Four uniforms in (0, 1) for (particle, step, draw): (x + 0.5) 2^-32."""
    key = (seed & _MASK, (seed >> 32) & _MASK)
    x = philox4x32_10((particle, step, draw, 0), key)
    return [(xi + 0.5) * 2.0 ** -32 for xi in x]


def poisson_inversion(lam, u, kmax=256):
    """Smallest n with CDF(n) >= u for Poisson(lam), by sequential search."""
    p = math.exp(-lam)
    F = p
    n = 0
    while u > F and n < kmax:
        n += 1
        p *= lam / n
        F += p
    return n


def recoil_kick(seed, particle, step, R, dt, v_rec):
    """Velocity kick of one step: (kick (3,), n_events)."""
    u = uniforms(seed, particle, step, 0)
    n = poisson_inversion(R * dt, u[0])
    kick = np.zeros(3)
    for i in range(2 * n):
        w = uniforms(seed, particle, step, 1 + i // 2)
        a, b = (w[0], w[1]) if i % 2 == 0 else (w[2], w[3])
        cz = 2.0 * a - 1.0
        phi = 2.0 * math.pi * b
        sp = math.sqrt(max(0.0, 1.0 - cz * cz))
        kick += v_rec * np.array([sp * math.cos(phi), sp * math.sin(phi), cz])
    return kick, n


def leapfrog3d(mol, beams3, B_gradient, r0, v0, t_max, dt=1e-6, r_escape=0.015, Gamma_eff=1.0,
               hbar=HBAR_CODATA, kicks=False, seed=0, particle=0):
    """MOTSimulator3D.simulate_trajectory_3d (simulator_3d.py:443-504): returns
    (t, r [n, 3], v [n, 3]); with kicks, adds the recoil model after each
    velocity update.  beams3 = (khat, freq, q_lab, s0, radius)."""
    khat, freq, ql, s0, rad = beams3
    mass = mol.mass
    v_rec = hbar * mol.k / mass
    n = int(t_max / dt)
    t = np.arange(n) * dt
    R_ = np.zeros((n, 3))
    V_ = np.zeros((n, 3))
    R_[0] = r0
    V_[0] = v0
    F0, Rs0, _ = force3d(mol, khat, freq, ql, s0, rad, R_[0], V_[0], B_gradient, Gamma_eff, hbar)
    vh = V_[0] + 0.5 * dt * F0 / mass
    for j in range(1, n):
        R_[j] = R_[j - 1] + dt * vh
        if np.linalg.norm(R_[j]) > r_escape:
            R_[j:] = R_[j]
            V_[j:] = vh
            break
        F, Rs, _ = force3d(mol, khat, freq, ql, s0, rad, R_[j], vh, B_gradient, Gamma_eff, hbar)
        vn = vh + dt * F / mass
        if kicks:
            kick, _ = recoil_kick(seed, particle, j, Rs, dt, v_rec)
            vn = vn + kick
        V_[j] = 0.5 * (vh + vn)
        vh = vn
    return t, R_, V_
