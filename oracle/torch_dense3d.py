"""TEST INFRASTRUCTURE ONLY -- a dense FP64 torch restatement of the
reference's 3D rate-equation force (molmot/mot/simulator_3d.py:168-365,
rate_eq_force_3d) and of its leapfrog (:443-504), batched over points and
differentiable with torch autograd: torch.linalg.eigh for the ground Zeeman
eigenbasis (its derivative is defined for a non-degenerate spectrum),
torch.linalg.solve for the populations.  Used to check the 3D trajectory
tangents of molmot_b200 (derivatives with respect to beam frequencies,
saturation parameters and B', through positions and velocities).

Follows oracle/force3d.py (numpy), which is pinned to the reference's own
outputs; tests/test_force3d_oracle.py checks this restatement against it.
"""
from __future__ import annotations

import math

import numpy as np
import torch

HBAR_CODATA = 1.054571817e-34


def _pol_weights(q_lab, ct):
    """Normalised |d^1_{m' m}(theta)|^2 column of each beam (q_lab [n_b]) at
    cos(theta) = ct [n]: returns [n, n_b, 3] (simulator_3d.py:112-165)."""
    st2 = (1.0 - ct * ct).clamp(min=0.0)  # sin^2 theta
    d = ((1 + ct) / 2) ** 2
    o = ((1 - ct) / 2) ** 2
    m = st2 / 2
    c = ct * ct
    cols = []
    for q in q_lab:
        q = int(q)
        if q == 0:
            w = torch.stack([d, m, o], dim=-1)
        elif q == 1:
            w = torch.stack([m, c, m], dim=-1)
        else:
            w = torch.stack([o, m, d], dim=-1)
        cols.append(w / w.sum(-1, keepdim=True))
    return torch.stack(cols, dim=1)


def force3d(mol, khat, freq, q_lab, s0, radius, r, v, B_gradient, Gamma_eff=1.0, hbar=HBAR_CODATA):
    """F [n, 3], R [n], p [n, n_g] at points r, v [n, 3] (torch float64; may
    require grad); freq, s0 [n_b] and B_gradient (scalar) may be tensors that
    require grad.  khat [n_b, 3], q_lab [n_b], radius [n_b] are constants."""
    f64 = dict(dtype=torch.float64, device=r.device)
    c128 = dict(dtype=torch.complex128, device=r.device)
    n_g, n_e = int(mol.n_ground), int(mol.n_excited)
    G, k = float(mol.Gamma), float(mol.k)
    khat = torch.as_tensor(np.array(khat, dtype=float), **f64)
    radius = np.asarray(radius, dtype=float)
    freq = torch.as_tensor(freq, **f64)
    s0 = torch.as_tensor(s0, **f64)
    Bg = torch.as_tensor(B_gradient, **f64)
    n = r.shape[0]
    B = torch.stack([-Bg * r[:, 0] / 2.0 * 1e4, -Bg * r[:, 1] / 2.0 * 1e4, Bg * r[:, 2] * 1e4], dim=1)
    Bm = B.norm(dim=1)
    ct = torch.where(Bm > 1e-10, B[:, 2] / Bm.clamp(min=1e-300), torch.ones_like(Bm))
    Z = [torch.as_tensor(np.array(getattr(mol, f"zeeman_{a}"))[:n_g, :n_g], **c128) for a in "xyz"]
    H = sum(B[:, c, None, None].to(torch.complex128) * Z[c][None] for c in range(3))
    H = 0.5 * (H + H.conj().transpose(1, 2))
    lam, U = torch.linalg.eigh(H)
    E = torch.as_tensor(np.array(mol.energies, dtype=float), **f64)
    Es_g = E[None, :n_g] + lam * G / (2 * math.pi)
    Ze = torch.as_tensor(np.real(np.diag(np.asarray(mol.zeeman_z)[n_g:, n_g:])).copy(), **f64)
    Es_e = E[None, n_g:] + B[:, 2:3] * Ze[None] * G / (2 * math.pi)
    d_bare = torch.as_tensor(np.abs(np.asarray(mol.tdm)[:n_g, n_g:n_g + n_e, :]), **c128)
    x = torch.einsum("nga,geq->naeq", U.conj(), d_bare)
    d_sq = (x.real ** 2 + x.imag ** 2)                          # [n, a, e, q]
    mask = (d_sq >= 1e-15).to(torch.float64)
    tot = d_sq.sum(dim=(1, 3))                                  # [n, e]
    BR = d_sq.sum(dim=3) / tot[:, None, :]                      # [n, g, e]
    gh = G / 2.0
    om = Es_e[:, None, :] - Es_g[:, :, None]                    # [n, g, e]
    w = _pol_weights(q_lab, ct)                                 # [n, b, 3]
    rows = []
    s_tot = torch.zeros((n, n_g), **f64)
    for b in range(khat.shape[0]):
        dop = -k * (v @ khat[b]) / (2 * math.pi)
        gf = torch.ones(n, **f64)
        if np.isfinite(radius[b]) and radius[b] > 0:
            rp = r @ khat[b]
            rps = ((r * r).sum(1) - rp * rp).clamp(min=0.0)
            gf = torch.exp(-2.0 * rps / radius[b] ** 2)
        de = (freq[b] + dop[:, None, None] - om) * 2 * math.pi
        L = gh ** 2 / (de * de + gh ** 2)
        rs = (w[:, b, None, None, :] * d_sq * mask).sum(-1) * L   # [n, g, e]
        s_tot = s_tot + s0[b] * gf[:, None] * rs.sum(-1)
        rows.append(rs * (s0[b] * gf)[:, None, None])
    Rb = torch.stack(rows, dim=1)                               # [n, b, g, e]
    rate = gh * Rb * Gamma_eff / (1.0 + s_tot)[:, None, :, None]
    Rs = rate.sum(1)                                            # [n, g, e]
    M = torch.einsum("nke,nge->ngk", Rs, BR) - torch.diag_embed(Rs.sum(-1))
    M = torch.cat([M[:, :-1, :], torch.ones((n, 1, n_g), **f64)], dim=1)
    rhs = torch.zeros((n, n_g, 1), **f64)
    rhs[:, -1, 0] = 1.0
    p = torch.linalg.solve(M, rhs)[..., 0]
    per_beam = torch.einsum("nbge,ng->nb", rate, p)
    F = hbar * k * per_beam @ khat
    return F, per_beam.sum(1), p


def leapfrog(mol, beams3, B_gradient, r0, v0, n_steps, dt=1e-6, kicks=None, hbar=HBAR_CODATA):
    """The reference's leapfrog (simulator_3d.py:443-504) for particles r0, v0
    [n, 3] over n_steps samples (n_steps - 1 updates), differentiable; kicks
    (optional) [n_steps, n, 3] velocity increments added after each velocity
    update (held fixed: the derivative at fixed noise).  No escape test (the
    particles must stay inside).  Returns the synchronised velocity of the
    last sample [n, 3] and the final position."""
    khat, freq, q, s0, rad = beams3
    m = float(mol.mass)
    F0 = force3d(mol, khat, freq, q, s0, rad, r0, v0, B_gradient, hbar=hbar)[0]
    vh = v0 + 0.5 * dt * F0 / m
    r = r0
    vs = v0
    for j in range(1, n_steps):
        r = r + dt * vh
        F = force3d(mol, khat, freq, q, s0, rad, r, vh, B_gradient, hbar=hbar)[0]
        vn = vh + dt * F / m
        if kicks is not None:
            vn = vn + kicks[j]
        vs = 0.5 * (vh + vn)
        vh = vn
    return vs, r
