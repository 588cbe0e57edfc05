"""Differentiable steady-state force (torch.autograd) and MOT coefficients.

``SteadyStateForce`` runs the fused force + adjoint kernel in the forward
pass (mm_force_adjoint: one transposed solve per point with the
elimination's own factors, or, with precision="fp64_reduced", with the
excited-chain solve's matrix) and keeps the per-point gradients; its backward
pass contracts them with the incoming gradient.  Gradients flow to the beam
frequencies (so to detunings), to the saturation parameters (so to powers,
s0 being proportional to power) and to B'.

``mot_coefficients`` gives, per parameter set, the spring constant
k = -dF/dz and damping beta = -(dF/dv)/m as least-squares slopes over
n-point stencils (default 33 points in z0 +- 0.3 mm at v = 0 and in
+- 0.1 m/s at z = z0), differentiable with respect to the detunings, the
powers (through s0) and B'.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import BeamSets, force_adjoint, pack_for


class SteadyStateForce(torch.autograd.Function):
    @staticmethod
    def forward(ctx, freq, s0, bgrad, v, z, pack, kdir, pol, gamma_eff, points_per_set, hbar,
                precision):
        bs = BeamSets(kdir, freq.detach().cpu().numpy(), pol, s0.detach().cpu().numpy(),
                      bgrad.detach().cpu().numpy(), gamma_eff)
        F, G = force_adjoint(pack, bs, v, z, points_per_set=points_per_set, hbar=hbar,
                             precision=precision)
        ctx.save_for_backward(G)
        ctx.shape = (freq.shape[0], freq.shape[1], points_per_set)
        return F.to(freq.device)

    @staticmethod
    def backward(ctx, gF):
        (G,) = ctx.saved_tensors
        n_sets, nb, pps = ctx.shape
        J = G.view(n_sets, pps, 2 * nb + 1)
        tot = (J * gF.reshape(n_sets, pps, 1).to(J.device)).sum(1)
        return (tot[:, :nb], tot[:, nb:2 * nb], tot[:, 2 * nb],
                None, None, None, None, None, None, None, None, None)


def steady_state_force(mol, kdir, pol, freq, s0, bgrad, v, z, points_per_set, gamma_eff=1.0,
                       hbar=None, precision="fp64"):
    """F at points (v, z) ([n_sets * points_per_set]) for parameter sets with
    beam frequencies freq [n_sets, n_b], saturation parameters s0 [n_sets, n_b]
    and gradients bgrad [n_sets] (torch float64 tensors, may require grad).
    precision: "fp64" or "fp64_reduced" (the two adjoint forms)."""
    return SteadyStateForce.apply(freq, s0, bgrad, v, z, pack_for(mol), np.asarray(kdir),
                                  np.asarray(pol), gamma_eff, int(points_per_set), hbar, precision)


def stencil_weights(x: np.ndarray) -> np.ndarray:
    """Weights c with slope = sum c_i F_i of the least-squares line through (x_i, F_i)."""
    xm = x - x.mean()
    return xm / np.sum(xm ** 2)


def mot_coefficients(mol, kdir, pol, freq, s0, bgrad, n: int = 33, z0: float = 0.0,
                     dz: float = 0.3e-3, dv: float = 0.1, gamma_eff: float = 1.0, hbar=None,
                     precision: str = "fp64"):
    """(k [n_sets], beta [n_sets]) -- differentiable (torch)."""
    n_sets = freq.shape[0]
    zs = z0 + np.linspace(-dz, dz, n)
    vs = np.linspace(-dv, dv, n)
    v = np.tile(np.concatenate([np.zeros(n), vs]), n_sets)
    z = np.tile(np.concatenate([zs, np.full(n, z0)]), n_sets)
    F = steady_state_force(mol, kdir, pol, freq, s0, bgrad, v, z, 2 * n, gamma_eff, hbar, precision)
    F = F.view(n_sets, 2 * n)
    cz = torch.as_tensor(stencil_weights(zs), dtype=F.dtype, device=F.device)
    cv = torch.as_tensor(stencil_weights(vs), dtype=F.dtype, device=F.device)
    k = -(F[:, :n] * cz).sum(1)
    beta = -(F[:, n:] * cv).sum(1) / mol.mass
    return k, beta
