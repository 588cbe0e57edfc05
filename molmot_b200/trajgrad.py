"""Gradients of trajectory ensembles: the per-axis 3D MOT model
(molmot/propagation/trajectories.py:78-156, the model of ``engine.traj`` with
ndim = 3) carried with its tangents d(r, v)/d theta in one launch
(mm_traj_grad_run).

Parameters theta_k add to beam frequencies (``freq_par[b] = k``), to
saturation parameters (``s0_par[b] = k``) or to B' (``bprime_par = k``).  The
tangents are propagated forward (forward mode): each step takes the force's
gradient from the FP64-reduced adjoint, so one force solve per axis and step
gives every parameter's derivative.  Photon-recoil kicks (N ~ Poisson(R dt)
events per step, R the sum of the three axes' scattering rates, 2N isotropic
kicks of hbar k / m) are held fixed under differentiation: the derivative at
fixed noise.

``mean_kinetic_energy`` wraps the ensemble-mean final kinetic energy
<m |v|^2 / 2> as a ``torch.autograd.Function`` of theta.  A run can be split
into checkpointed segments: every ``ckpt_every`` steps the state with its
tangents is saved, and a run resumed from a checkpoint gives the same bits as
the unbroken run.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .constants import HBAR_JIT
from .engine import BeamSets, MoleculePack, _dptr, _stream_handle, _to_dev


def _param_map(idx: Optional[Sequence[int]], n_b: int, n_par: int, what: str):
    arr = (ctypes.c_int32 * _lib.MM_MAX_BEAMS)(*([-1] * _lib.MM_MAX_BEAMS))
    if idx is None:
        return arr
    idx = [int(i) for i in idx]
    if len(idx) != n_b:
        raise ValueError(f"{what} has {len(idx)} entries for {n_b} beams")
    for b, k in enumerate(idx):
        if k < -1 or k >= n_par:
            raise ValueError(f"{what}[{b}] = {k} is outside [-1, {n_par})")
        arr[b] = k
    return arr


def pack_state(r, v, dr=None, dv=None, n_par: int = 1) -> torch.Tensor:
    """State rows [N, 6 + 6 n_par]: r[3], v[3], dr[3][n_par], dv[3][n_par]."""
    r = _to_dev(r).reshape(-1, 3)
    v = _to_dev(v).reshape(-1, 3)
    N = r.shape[0]
    st = torch.zeros((N, 6 + 6 * n_par), dtype=torch.float64, device=r.device)
    st[:, 0:3] = r
    st[:, 3:6] = v
    if dr is not None:
        st[:, 6:6 + 3 * n_par] = _to_dev(dr).reshape(N, 3 * n_par)
    if dv is not None:
        st[:, 6 + 3 * n_par:] = _to_dev(dv).reshape(N, 3 * n_par)
    return st


def unpack_state(st: torch.Tensor, n_par: int) -> dict:
    N = st.shape[0]
    return {"r": st[:, 0:3], "v": st[:, 3:6],
            "dr": st[:, 6:6 + 3 * n_par].reshape(N, 3, n_par),
            "dv": st[:, 6 + 3 * n_par:].reshape(N, 3, n_par)}


def traj_grad(pack: MoleculePack, beams: BeamSets, r0, v0, dt: float, n_steps: int, *,
              n_par: int, freq_par=None, s0_par=None, bprime_par: int = -1,
              r_escape: float = 0.015, kicks: bool = False, seed: int = 0, hbar=None,
              step0: int = 0, state=None, n_actual=None, ckpt_every: int = 0, stream=None) -> dict:
    """Run n_steps Euler steps of the per-axis model with tangents.

    r0, v0: (N, 3) for a new run (tangents start at zero), or ``state``
    ([N, 6 + 6 n_par], e.g. a checkpoint) with ``step0`` its absolute step and
    ``n_actual`` the previous call's stop steps.  Returns a dict of device
    tensors: r, v (N, 3), dr, dv (N, 3, n_par), n_actual (N,), state, and
    ckpt ([n_steps // ckpt_every, N, 6 + 6 n_par]) when ckpt_every > 0.
    """
    if state is None:
        state = pack_state(r0, v0, n_par=n_par)
    else:
        state = _to_dev(state).reshape(-1, 6 + 6 * n_par).clone()
    N = state.shape[0]
    dev = state.device
    if n_actual is None:
        n_actual = torch.zeros(N, dtype=torch.int32, device=dev)
    else:
        n_actual = torch.as_tensor(n_actual, dtype=torch.int32, device=dev).clone()
    o = _lib.TgradOpts()
    o.n_steps, o.step0 = int(n_steps), int(step0)
    o.ckpt_every = int(ckpt_every)
    o.dt, o.r_escape = float(dt), float(r_escape)
    o.hbar = float(hbar) if hbar else HBAR_JIT
    o.seed, o.kicks, o.n_par = int(seed), 1 if kicks else 0, int(n_par)
    o.freq_par = _param_map(freq_par, beams.n_beams, n_par, "freq_par")
    o.s0_par = _param_map(s0_par, beams.n_beams, n_par, "s0_par")
    o.bprime_par = int(bprime_par)
    ck = None
    if ckpt_every > 0:
        ck = torch.empty((n_steps // ckpt_every, N, 6 + 6 * n_par), dtype=torch.float64, device=dev)
    rc = _lib.load().mm_traj_grad_run(pack.handle, beams.handle, ctypes.byref(o), N, _dptr(state),
                                      _dptr(n_actual), _dptr(ck), _stream_handle(stream))
    _lib.check(rc, "mm_traj_grad_run")
    out = unpack_state(state, n_par)
    out.update(state=state, n_actual=n_actual)
    if ck is not None:
        out["ckpt"] = ck
    return out


class MeanKineticEnergy(torch.autograd.Function):
    """<m |v_final|^2 / 2> over the ensemble as a function of theta [n_par]."""

    @staticmethod
    def forward(ctx, theta, pack, base, maps, r0, v0, dt, n_steps, run_kw):
        kdir, freq, pol, s0, bgrad, geff = base
        freq_par, s0_par, bprime_par = maps
        th = theta.detach().cpu().numpy().astype(np.float64)
        f = np.array(freq, dtype=np.float64).copy()
        s = np.array(s0, dtype=np.float64).copy()
        for b in range(len(f)):
            if freq_par is not None and freq_par[b] >= 0:
                f[b] += th[freq_par[b]]
            if s0_par is not None and s0_par[b] >= 0:
                s[b] += th[s0_par[b]]
        bg = float(bgrad) + (th[bprime_par] if bprime_par >= 0 else 0.0)
        bs = BeamSets(np.asarray(kdir)[None], f[None], np.asarray(pol)[None], s[None], [bg], geff)
        out = traj_grad(pack, bs, r0, v0, dt, n_steps, n_par=len(th), freq_par=freq_par,
                        s0_par=s0_par, bprime_par=bprime_par, **run_kw)
        m = pack.mass
        E = 0.5 * m * (out["v"] ** 2).sum(1).mean()
        G = m * (out["v"][:, :, None] * out["dv"]).sum(1).mean(0)
        ctx.save_for_backward(G)
        return E.to(theta.device)

    @staticmethod
    def backward(ctx, gE):
        (G,) = ctx.saved_tensors
        return (gE.to(G.device) * G).to(gE.device), None, None, None, None, None, None, None, None


def mean_kinetic_energy(theta: torch.Tensor, pack: MoleculePack, kdir, freq, pol, s0, bgrad, r0, v0,
                        dt: float, n_steps: int, *, freq_par=None, s0_par=None, bprime_par: int = -1,
                        gamma_eff: float = 1.0, **run_kw) -> torch.Tensor:
    """Ensemble-mean final kinetic energy (J) of the per-axis 3D model for one
    beam set (kdir, freq, pol, s0 [n_beams], bgrad) whose parameters are
    shifted by theta ([n_par] float64 tensor) through the maps; differentiable
    with respect to theta.  run_kw: r_escape, kicks, seed, hbar (traj_grad)."""
    return MeanKineticEnergy.apply(theta, pack, (kdir, freq, pol, s0, bgrad, gamma_eff),
                                   (freq_par, s0_par, bprime_par), r0, v0, dt, n_steps, run_kw)


class DegenerateSpectrum(RuntimeError):
    """A 3D tangent step met a degenerate ground Zeeman spectrum, where the
    eigenbasis -- and with it d(force)/d(position) -- is not defined."""


def traj3d_grad(pack: MoleculePack, beams: BeamSets, r0, v0, dt: float, n_steps: int, *,
                n_par: int, freq_par=None, s0_par=None, bprime_par: int = -1,
                r_escape: float = 0.015, kicks: bool = False, seed: int = 0, hbar=None,
                gap_tol: float = 0.0, step0: int = 0, state=None, n_actual=None,
                ckpt_every: int = 0, allow_degenerate: bool = False, stream=None) -> dict:
    """The 3D leapfrog ensemble of ``engine.traj3d`` (24-beam force, beam set
    0 of 3D beam sets) with its tangents d(r, v)/d theta (mm_traj3d_grad_run),
    through the field dependence of the ground Zeeman eigenbasis.

    r0, v0: (N, 3) for a new run (tangents start at zero), or ``state``
    ([N, 6 + 6 n_par]: r, v_half and their tangents, e.g. a checkpoint) with
    ``step0`` the next update's absolute index and ``n_actual`` the previous
    call's stop steps.  Returns device tensors r, vh (N, 3), dr, dvh
    (N, 3, n_par), v and dv (the synchronised velocity of the last update and
    its tangent), n_actual, status, n_events, state and, with ckpt_every > 0,
    ckpt.  Raises DegenerateSpectrum when a step met a degenerate spectrum
    (status bit MM_ST_DEGENERATE), unless allow_degenerate.
    """
    from .constants import hbar as HBAR_CODATA
    if state is None:
        state = pack_state(r0, v0, n_par=n_par)
    else:
        state = _to_dev(state).reshape(-1, 6 + 6 * n_par).clone()
    N = state.shape[0]
    dev = state.device
    if n_actual is None:
        n_actual = torch.zeros(N, dtype=torch.int32, device=dev)
    else:
        n_actual = torch.as_tensor(n_actual, dtype=torch.int32, device=dev).clone()
    o = _lib.T3gradOpts()
    o.n_steps, o.step0, o.ckpt_every = int(n_steps), int(step0), int(ckpt_every)
    o.dt, o.r_escape = float(dt), float(r_escape)
    o.hbar = float(hbar) if hbar else HBAR_CODATA
    o.gap_tol = float(gap_tol)
    o.seed, o.kicks, o.n_par = int(seed), 1 if kicks else 0, int(n_par)
    o.freq_par = _param_map(freq_par, beams.n_beams, n_par, "freq_par")
    o.s0_par = _param_map(s0_par, beams.n_beams, n_par, "s0_par")
    o.bprime_par = int(bprime_par)
    L = _lib.load()
    vsync = torch.empty((N, 3 + 3 * n_par), dtype=torch.float64, device=dev)
    status = torch.empty(N, dtype=torch.int32, device=dev)
    n_ev = torch.empty(N, dtype=torch.int32, device=dev)
    ck = None
    if ckpt_every > 0:
        n_ck = int(L.mm_traj3d_grad_checkpoints(int(step0), int(n_steps), int(ckpt_every)))
        ck = torch.empty((n_ck, N, 6 + 6 * n_par), dtype=torch.float64, device=dev)
    rc = L.mm_traj3d_grad_run(pack.handle, beams.handle, ctypes.byref(o), N, _dptr(state), _dptr(vsync),
                              _dptr(n_actual), _dptr(status), _dptr(n_ev), _dptr(ck), _stream_handle(stream))
    _lib.check(rc, "mm_traj3d_grad_run")
    if not allow_degenerate and bool((status & _lib.MM_ST_DEGENERATE).any()):
        raise DegenerateSpectrum(
            "the ground Zeeman spectrum is degenerate on this trajectory (e.g. SrOH's 6 + 6 "
            "clusters): the eigenbasis, and with it d(force)/d(position), is not defined")
    out = unpack_state(state, n_par)
    out["vh"], out["dvh"] = out.pop("v"), out.pop("dv")
    out.update(v=vsync[:, :3], dv=vsync[:, 3:].reshape(N, 3, n_par), state=state, n_actual=n_actual,
               status=status, n_events=n_ev)
    if ck is not None:
        out["ckpt"] = ck
    return out
