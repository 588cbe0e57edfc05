"""TEST INFRASTRUCTURE ONLY -- a dense FP64 torch restatement of the 1D
rate-equation force (molmot/obe/rate_equations_jit.py:18-145), vectorised
over points and differentiable with torch autograd (torch.linalg.solve for
the population system).  Used to check the adjoint kernel's gradients."""
from __future__ import annotations

import math

import numpy as np
import torch


def force(mol, kdir, pol, freq, s0, bgrad, v, z, pps, gamma_eff=1.0, hbar=1.0545718e-34):
    """F for points (v[i], z[i]) of set i // pps; freq, s0 [n_sets, n_b] and
    bgrad [n_sets] are torch float64 tensors (may require grad)."""
    dev = freq.device
    f64 = dict(dtype=torch.float64, device=dev)
    n_g, n_e = mol.n_ground, mol.n_excited
    E = torch.as_tensor(mol.energies, **f64)
    zd = torch.as_tensor(mol.zeeman_z_diag, **f64)
    d2 = np.asarray(mol.d_squared)
    BR = np.zeros((n_e, n_g))
    for e in range(n_e):
        tot = d2[:, e, :].sum()
        if tot > 1e-30:
            BR[e] = d2[:, e, :].sum(1) / tot
    BR = torch.as_tensor(BR, **f64)
    G, k = float(mol.Gamma), float(mol.k)
    gh = G / 2.0
    # v, z: arrays, or torch tensors (which may require grad)
    v = v.to(**f64) if torch.is_tensor(v) else torch.as_tensor(np.asarray(v), **f64)
    z = z.to(**f64) if torch.is_tensor(z) else torch.as_tensor(np.asarray(z), **f64)
    n = v.numel()
    sid = torch.arange(n, device=dev) // pps
    B = bgrad[sid]
    Es = E[None, :] + (B * z * 1e4)[:, None] * zd[None, :] * G / (2 * math.pi)
    R = torch.zeros((n, n_g, n_e), **f64)
    Fg = torch.zeros((n, n_g), **f64)
    s = torch.zeros((n, n_g), **f64)
    kdir = np.asarray(kdir)
    pol = np.asarray(pol)
    for b in range(kdir.shape[1]):
        dop = -k * torch.as_tensor(kdir[:, b], **f64)[sid] * v / (2 * math.pi)
        fb = freq[sid, b]
        sb = s0[sid, b]
        for g in range(n_g):
            for e in range(n_e):
                q = pol[:, b]
                dd = torch.as_tensor(d2[g, e, q], **f64)[sid]
                if not torch.any(dd >= 1e-15):
                    continue
                dd = torch.where(dd >= 1e-15, dd, torch.zeros_like(dd))
                de = (fb + dop - (Es[:, n_g + e] - Es[:, g])) * 2 * math.pi
                L = gh ** 2 / (de * de + gh ** 2)
                ru = gh * sb * dd * L * gamma_eff
                R[:, g, e] = R[:, g, e] + ru
                Fg[:, g] = Fg[:, g] + hbar * k * torch.as_tensor(kdir[:, b], **f64)[sid] * ru
                s[:, g] = s[:, g] + sb * dd * L
    sat = 1.0 / (1.0 + s)
    R = R * sat[:, :, None]
    Fg = Fg * sat
    M = torch.einsum("nke,eg->ngk", R, BR) - torch.diag_embed(R.sum(2))
    M = torch.cat([M[:, :-1, :], torch.ones((n, 1, n_g), **f64)], dim=1)
    rhs = torch.zeros((n, n_g, 1), **f64)
    rhs[:, -1, 0] = 1.0
    p = torch.linalg.solve(M, rhs)[..., 0]
    return (p * Fg).sum(1)
