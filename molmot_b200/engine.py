"""Device handles and batched calls over the C ABI.

``MoleculePack`` and ``BeamSets`` own the library's immutable device copies
of a molecule and of parameter sets of beams (the B200 counterpart of
molmot_cuda's ``CUDAMolData``, molmot_cuda/rate_equations_cuda.py:399-441).
``force_batch`` and ``traj1d`` launch the CUDA kernels on torch's current
stream with torch-owned device tensors.  Inputs may be numpy arrays or
torch tensors; numpy inputs are copied to the device first.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .constants import HBAR_JIT

PRECISIONS = {"fp64": _lib.MM_PREC_FP64, "fp32": _lib.MM_PREC_FP32_REFINE,
              "fp32_refine": _lib.MM_PREC_FP32_REFINE, "fp64_reduced": _lib.MM_PREC_FP64_REDUCED}


def _np(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _dptr(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("molmot_b200 needs a CUDA device (there is no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def _to_dev(x, dtype=torch.float64) -> torch.Tensor:
    dev = _device()
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype).to(dev)


def _stream_handle(stream: Optional[torch.cuda.Stream]):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def molecule_arrays(mol):
    """Flat host arrays of a MolecularData-like object for the pack."""
    n_g, n_e = int(mol.n_ground), int(mol.n_excited)
    out = dict(n_g=n_g, n_e=n_e, E=_np(mol.energies, np.float64),
               d2=_np(mol.d_squared, np.float64).reshape(-1),
               zd=_np(mol.zeeman_z_diag, np.float64))
    if getattr(mol, "zeeman_x", None) is not None and getattr(mol, "tdm", None) is not None:
        Z = [np.asarray(getattr(mol, f"zeeman_{a}"))[:n_g, :n_g] for a in "xyz"]
        out["Zre"] = _np(np.stack([z.real for z in Z]), np.float64).reshape(-1)
        out["Zim"] = _np(np.stack([z.imag for z in Z]), np.float64).reshape(-1)
        out["Ze"] = _np(np.real(np.diag(np.asarray(mol.zeeman_z)[n_g:, n_g:])), np.float64)
        tdm = np.asarray(mol.tdm)
        out["tdm_abs"] = _np(np.abs(tdm[:n_g, n_g:n_g + n_e, :]), np.float64).reshape(-1)
    return out


class MoleculePack:
    """Device copy of a molecule (energies, |d|^2, Zeeman diagonal, branching
    ratios; plus ground Zeeman blocks and |tdm| for the 3D model)."""

    def __init__(self, mol):
        self.mol = mol
        a = molecule_arrays(mol)
        self.n_ground, self.n_excited = a["n_g"], a["n_e"]
        self.Gamma, self.k, self.mass = float(mol.Gamma), float(mol.k), float(mol.mass)
        self._keep = a
        d = _lib.MolDesc()
        d.n_ground, d.n_excited = self.n_ground, self.n_excited
        d.energies, d.d_squared, d.zeeman_z_diag = _ptr(a["E"]), _ptr(a["d2"]), _ptr(a["zd"])
        d.Gamma, d.k, d.mass = self.Gamma, self.k, self.mass
        if "Zre" in a:
            d.zeeman_ground_re, d.zeeman_ground_im = _ptr(a["Zre"]), _ptr(a["Zim"])
            d.zeeman_excited_z, d.tdm_abs = _ptr(a["Ze"]), _ptr(a["tdm_abs"])
        _device()
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mm_pack_create(ctypes.byref(d), ctypes.byref(h)), "mm_pack_create")
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.load().mm_pack_destroy(h)
            except Exception:
                pass
            self.handle = None


class BeamSets:
    """Device copy of ``n_sets`` parameter sets of ``n_beams`` beams.

    kdir, freq, s0: [n_sets, n_beams] float; pol: [n_sets, n_beams] int in
    {0, 1, 2}; b_gradient: [n_sets] (T/m).  khat [n_sets, n_beams, 3] and
    radius [n_sets, n_beams] are for the 3D model.
    """

    def __init__(self, kdir, freq, pol, s0, b_gradient, gamma_eff: float = 1.0,
                 khat=None, radius=None):
        kdir = np.atleast_2d(_np(kdir, np.float64))
        n_sets, n_b = kdir.shape
        freq = _np(freq, np.float64).reshape(n_sets, n_b)
        pol = _np(pol, np.int32).reshape(n_sets, n_b)
        s0 = _np(s0, np.float64).reshape(n_sets, n_b)
        bg = _np(np.broadcast_to(np.asarray(b_gradient, dtype=np.float64), (n_sets,)), np.float64)
        self.n_sets, self.n_beams = n_sets, n_b
        self.gamma_eff = float(gamma_eff)
        self._keep = [kdir, freq, pol, s0, bg]
        d = _lib.BeamDesc()
        d.n_beams = n_b
        d.kdir, d.freq, d.pol, d.s0, d.b_gradient = (_ptr(kdir), _ptr(freq), _ptr(pol), _ptr(s0),
                                                     _ptr(bg))
        d.gamma_eff = self.gamma_eff
        if khat is not None:
            kh = _np(khat, np.float64).reshape(n_sets, n_b, 3)
            rad = _np(radius if radius is not None else np.zeros((n_sets, n_b)), np.float64)
            rad = rad.reshape(n_sets, n_b)
            self._keep += [kh, rad]
            d.khat, d.radius = _ptr(kh), _ptr(rad)
        _device()
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mm_beams_create(ctypes.byref(d), n_sets, ctypes.byref(h)),
                   "mm_beams_create")
        self.handle = h

    @classmethod
    def from_beams(cls, beam_lists: Sequence, b_gradient, gamma_eff: float = 1.0):
        """From one LaserBeam list or a list of lists (one per set)."""
        if len(beam_lists) and not isinstance(beam_lists[0], (list, tuple)):
            beam_lists = [beam_lists]
        kdir = [[b.kdir_z for b in L] for L in beam_lists]
        freq = [[b.freq_offset for b in L] for L in beam_lists]
        pol = [[b.polarization for b in L] for L in beam_lists]
        s0 = [[b.s0 for b in L] for L in beam_lists]
        return cls(kdir, freq, pol, s0, b_gradient, gamma_eff)

    def view(self, first_set: int, n_sets: int) -> "BeamSets":
        """Sets [first_set, first_set + n_sets) as a handle sharing this one's
        device arrays (mm_beams_view; no device allocation or copy)."""
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mm_beams_view(self.handle, int(first_set), int(n_sets), ctypes.byref(h)),
                   "mm_beams_view")
        v = BeamSets.__new__(BeamSets)
        v.n_sets, v.n_beams, v.gamma_eff = int(n_sets), self.n_beams, self.gamma_eff
        v._keep = [self]  # the parent's arrays must outlive the view
        v.handle = h
        return v

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.load().mm_beams_destroy(h)
            except Exception:
                pass
            self.handle = None


def _opts(precision, layout, pps=0, nv=0, nz=0, hbar=None, uniform_fallback=False):
    o = _lib.BatchOpts()
    o.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    o.layout = layout
    o.points_per_set = int(pps)
    o.nv, o.nz = int(nv), int(nz)
    o.hbar = float(hbar) if hbar else HBAR_JIT
    o.uniform_fallback = 1 if uniform_fallback else 0
    return o


def force_batch(pack: MoleculePack, beams: BeamSets, v, z, *, grid: bool = False,
                points_per_set: Optional[int] = None, precision="fp64", hbar=None,
                uniform_fallback: bool = False, want_pop: bool = True, want_R: bool = True,
                want_status: bool = True, out=None, stream=None):
    """Steady-state force for a batch of points (one kernel launch).

    grid=True: per set, the outer product of v (nv,) and z (nz,), results
    shaped [n_sets, nv, nz].  Otherwise v and z are per point and point i
    belongs to set i // points_per_set; results are flat [n].
    Returns a dict of device tensors F, R, pop, status.
    """
    v = _to_dev(v)
    z = _to_dev(z)
    if grid:
        nv, nz = v.numel(), z.numel()
        n = beams.n_sets * nv * nz
        opts = _opts(precision, _lib.MM_LAYOUT_GRID, nv=nv, nz=nz, hbar=hbar,
                     uniform_fallback=uniform_fallback)
        shape = (beams.n_sets, nv, nz)
    else:
        if v.numel() != z.numel():
            raise ValueError("points layout needs v and z of the same length")
        n = v.numel()
        pps = points_per_set if points_per_set else n
        opts = _opts(precision, _lib.MM_LAYOUT_POINTS, pps=pps, hbar=hbar,
                     uniform_fallback=uniform_fallback)
        shape = (n,)
    dev = v.device
    if out is None:
        out = {"F": torch.empty(shape, dtype=torch.float64, device=dev)}
        if want_R:
            out["R"] = torch.empty(shape, dtype=torch.float64, device=dev)
        if want_pop:
            out["pop"] = torch.empty(shape + (pack.n_ground,), dtype=torch.float64, device=dev)
        if want_status:
            out["status"] = torch.empty(shape, dtype=torch.int32, device=dev)
    rc = _lib.load().mm_force_batch(pack.handle, beams.handle, _dptr(v), _dptr(z), n,
                                    ctypes.byref(opts), _dptr(out["F"]), _dptr(out.get("R")),
                                    _dptr(out.get("pop")), _dptr(out.get("status")),
                                    _stream_handle(stream))
    _lib.check(rc, "mm_force_batch")
    return out


_COPY_STREAMS = {}


def force_maps_to_host(pack: MoleculePack, beams: BeamSets, v, z, out=None, *, precision="fp32",
                       hbar=None, chunk_sets: int = 64, sync: bool = True):
    """Force maps F[n_sets, nv, nz] of every parameter set (grid layout) in
    host memory.

    The sets are computed in chunks of ``chunk_sets`` on the current stream,
    alternating between two device buffers; each chunk's device->host copy runs
    on a second stream while the next chunk is computed, so the transfer of
    the maps hides the computation.  Only the first chunk's computation is
    not hidden: 64-set chunks (the default) took 39.0 ms for 4096 SrOH sets x
    256 x 256 against 40.2 ms with 256-set chunks, where one 2.15 GB copy
    alone takes 37.6 ms.  ``out``: a host float64 tensor of that shape
    (page-locked for overlapped copies; allocated page-locked if None).
    With sync=False the call returns once everything is enqueued and the maps
    are complete when the current stream reaches that point.
    """
    v = _to_dev(v)
    z = _to_dev(z)
    dev = v.device
    nv, nz, n_sets = v.numel(), z.numel(), beams.n_sets
    if out is None:
        out = torch.empty((n_sets, nv, nz), dtype=torch.float64, pin_memory=True)
    if tuple(out.shape) != (n_sets, nv, nz) or out.dtype != torch.float64 or out.is_cuda:
        raise ValueError(f"out must be a host float64 tensor of shape {(n_sets, nv, nz)}")
    chunk = max(1, min(int(chunk_sets), n_sets))
    comp = torch.cuda.current_stream(dev)
    copy = _COPY_STREAMS.get(dev.index)
    if copy is None:
        copy = _COPY_STREAMS[dev.index] = torch.cuda.Stream(device=dev)
    bufs = [torch.empty((chunk, nv, nz), dtype=torch.float64, device=dev) for _ in range(2)]
    free = [None, None]  # event: the copy out of buffer b has finished
    for i, first in enumerate(range(0, n_sets, chunk)):
        n = min(chunk, n_sets - first)
        b = i % 2
        if free[b] is not None:
            comp.wait_event(free[b])
        force_batch(pack, beams.view(first, n), v, z, grid=True, precision=precision, hbar=hbar,
                    want_pop=False, want_R=False, want_status=False, out={"F": bufs[b][:n]},
                    stream=comp)
        done = torch.cuda.Event()
        done.record(comp)
        copy.wait_event(done)
        with torch.cuda.stream(copy):
            out[first:first + n].copy_(bufs[b][:n], non_blocking=True)
        free[b] = torch.cuda.Event()
        free[b].record(copy)
    for t in bufs:
        t.record_stream(copy)
    comp.wait_stream(copy)
    if sync:
        comp.synchronize()
    return out


def traj(pack: MoleculePack, beams: BeamSets, r0, v0, dt: float, n_steps: int, *, ndim: int = 1,
         n_avg: int = 1, r_escape: float = 0.015, save_full: bool = False, i_eq: Optional[int] = None,
         precision="fp64", hbar=None, stream=None):
    """Independent trajectories on the GPU, all steps in one launch.

    ndim = 1: Euler along z; r0, v0 are (N,).  ndim = 3: the per-axis model;
    r0, v0 are (N, 3).  n_avg = 2 averages beam sets 0 and 1 (RF MOT).
    i_eq: also return per-particle sums of v^2 and sample counts over steps
    j >= i_eq (monte_carlo_temperature).  Returns a dict of device tensors
    r_final, v_final, n_actual and optionally r_traj, v_traj, vsq_sum, n_samp.
    """
    r0 = _to_dev(r0).reshape(-1, ndim)
    v0 = _to_dev(v0).reshape(-1, ndim)
    N = r0.shape[0]
    dev = r0.device
    out = {"r_final": torch.empty((N, ndim), dtype=torch.float64, device=dev),
           "v_final": torch.empty((N, ndim), dtype=torch.float64, device=dev),
           "n_actual": torch.empty(N, dtype=torch.int32, device=dev)}
    if save_full:
        out["r_traj"] = torch.empty((N, n_steps, ndim), dtype=torch.float64, device=dev)
        out["v_traj"] = torch.empty((N, n_steps, ndim), dtype=torch.float64, device=dev)
    if i_eq is not None:
        out["vsq_sum"] = torch.empty(N, dtype=torch.float64, device=dev)
        out["n_samp"] = torch.empty(N, dtype=torch.float64, device=dev)
    o = _lib.TrajOpts()
    o.ndim, o.n_avg, o.n_steps = int(ndim), int(n_avg), int(n_steps)
    o.dt, o.r_escape = float(dt), float(r_escape)
    o.i_eq = int(i_eq) if i_eq is not None else -1
    o.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    o.hbar = float(hbar) if hbar else HBAR_JIT
    rc = _lib.load().mm_traj_run(pack.handle, beams.handle, ctypes.byref(o), _dptr(r0), _dptr(v0), N,
                                 _dptr(out["r_final"]), _dptr(out["v_final"]),
                                 _dptr(out["n_actual"]), _dptr(out.get("r_traj")),
                                 _dptr(out.get("v_traj")), _dptr(out.get("vsq_sum")),
                                 _dptr(out.get("n_samp")), _stream_handle(stream))
    _lib.check(rc, "mm_traj_run")
    return out


def traj1d(pack: MoleculePack, beams: BeamSets, z0, v0, dt: float, n_steps: int, *,
           z_escape: float = 0.015, save_full: bool = False, precision="fp64", hbar=None,
           stream=None):
    """N independent 1D Euler trajectories (beam set 0).
    Returns device tensors (z_final, v_final, n_actual, z_traj, v_traj)."""
    o = traj(pack, beams, np.atleast_1d(z0) if not isinstance(z0, torch.Tensor) else z0,
             np.atleast_1d(v0) if not isinstance(v0, torch.Tensor) else v0, dt, n_steps, ndim=1,
             r_escape=z_escape, save_full=save_full, precision=precision, hbar=hbar, stream=stream)
    zt = o["r_traj"][..., 0] if save_full else None
    vt = o["v_traj"][..., 0] if save_full else None
    return o["r_final"][:, 0], o["v_final"][:, 0], o["n_actual"], zt, vt


_PACKS = {}


def pack_for(mol) -> MoleculePack:
    """Cached MoleculePack of a molecule object (rebuilt when its arrays change)."""
    key = id(mol)
    a = molecule_arrays(mol)
    fp = hash((a["E"].tobytes(), a["d2"].tobytes(), a["zd"].tobytes(), float(mol.Gamma),
               float(mol.k), float(mol.mass)))
    hit = _PACKS.get(key)
    if hit is not None and hit[0] is mol and hit[1] == fp:
        return hit[2]
    p = MoleculePack(mol)
    _PACKS[key] = (mol, fp, p)
    return p


def beam_sets_3d(khat, freq, q_lab, s0, radius, b_gradient, gamma_eff: float = 1.0) -> BeamSets:
    """BeamSets carrying unit k vectors and 1/e^2 radii (radius <= 0 or None:
    plane wave) for the 3D kernels; arrays [n_sets, n_beams(, 3)]."""
    kh = np.asarray(khat, dtype=np.float64)
    if kh.ndim == 2:
        kh = kh[None]
    n_sets, n_b = kh.shape[:2]
    rad = np.array([[0.0 if (x is None or not np.isfinite(x)) else float(x) for x in row]
                    for row in np.asarray(radius, dtype=object).reshape(n_sets, n_b)])
    return BeamSets(kh[..., 2], np.asarray(freq).reshape(n_sets, n_b),
                    np.asarray(q_lab).reshape(n_sets, n_b), np.asarray(s0).reshape(n_sets, n_b),
                    b_gradient, gamma_eff, khat=kh, radius=rad)


def force3d_batch(pack: MoleculePack, beams: BeamSets, r, v, *, points_per_set=None,
                  hbar=None, want_pop=True, stream=None):
    """3D force at points r[i], v[i] ([n, 3]); dict of device tensors F [n, 3], R, pop, status."""
    r = _to_dev(r).reshape(-1, 3)
    v = _to_dev(v).reshape(-1, 3)
    n = r.shape[0]
    dev = r.device
    out = {"F": torch.empty((n, 3), dtype=torch.float64, device=dev),
           "R": torch.empty(n, dtype=torch.float64, device=dev),
           "status": torch.empty(n, dtype=torch.int32, device=dev)}
    if want_pop:
        out["pop"] = torch.empty((n, pack.n_ground), dtype=torch.float64, device=dev)
    rc = _lib.load().mm_force3d_batch(pack.handle, beams.handle, _dptr(r), _dptr(v), n,
                                      int(points_per_set or n), float(hbar or 0.0),
                                      _dptr(out["F"]), _dptr(out["R"]), _dptr(out.get("pop")),
                                      _dptr(out["status"]), _stream_handle(stream))
    _lib.check(rc, "mm_force3d_batch")
    return out


def traj3d(pack: MoleculePack, beams: BeamSets, r0, v0, dt: float, n_steps: int, *, step0: int = 0,
           r_escape: float = 0.015, kicks: bool = False, seed: int = 0, hbar=None,
           save_full: bool = False, stream=None):
    """3D leapfrog ensemble (beam set 0), all steps in one launch.  Returns a
    dict of device tensors r, vh (half-step velocity; pass both back with
    step0 to resume), v (synchronised), n_actual, ke, n_events and, with
    save_full, r_traj / v_traj [N, n_steps, 3]."""
    r0 = _to_dev(r0).reshape(-1, 3)
    v0 = _to_dev(v0).reshape(-1, 3)
    N = r0.shape[0]
    dev = r0.device
    f64 = dict(dtype=torch.float64, device=dev)
    out = {"r": torch.empty((N, 3), **f64), "vh": torch.empty((N, 3), **f64),
           "v": torch.empty((N, 3), **f64),
           "n_actual": torch.empty(N, dtype=torch.int32, device=dev),
           "ke": torch.empty(N, **f64),
           "n_events": torch.empty(N, dtype=torch.int32, device=dev)}
    if save_full:
        out["r_traj"] = torch.empty((N, n_steps, 3), **f64)
        out["v_traj"] = torch.empty((N, n_steps, 3), **f64)
    rc = _lib.load().mm_traj3d_run(pack.handle, beams.handle, _dptr(r0), _dptr(v0), N, int(step0),
                                   int(n_steps), float(dt), float(r_escape), 1 if kicks else 0,
                                   int(seed) & 0xFFFFFFFFFFFFFFFF, float(hbar or 0.0),
                                   _dptr(out["r"]), _dptr(out["vh"]), _dptr(out["v"]),
                                   _dptr(out["n_actual"]), _dptr(out.get("r_traj")),
                                   _dptr(out.get("v_traj")), _dptr(out["ke"]),
                                   _dptr(out["n_events"]), _stream_handle(stream))
    _lib.check(rc, "mm_traj3d_run")
    return out


def force_adjoint(pack: MoleculePack, beams: BeamSets, v, z, *, grid: bool = False,
                  points_per_set: Optional[int] = None, hbar=None, precision: str = "fp64",
                  stream=None):
    """Force and its gradient: returns (F [n], grad [n, 2 n_beams + 1]) device
    tensors; grad rows are (dF/dfreq_b..., dF/ds0_b..., dF/dB').  precision:
    "fp64" (the elimination adjoint) or "fp64_reduced" (the adjoint of the
    excited-chain solve; batches with a set that fails its structural checks
    run the elimination adjoint)."""
    if precision not in ("fp64", "fp64_reduced"):
        raise ValueError(f"the adjoint runs in the fp64 and fp64_reduced forms, not {precision!r}")
    v = _to_dev(v)
    z = _to_dev(z)
    nb = beams.n_beams
    if grid:
        nv, nz = v.numel(), z.numel()
        n = beams.n_sets * nv * nz
        opts = _opts(precision, _lib.MM_LAYOUT_GRID, nv=nv, nz=nz, hbar=hbar)
    else:
        n = v.numel()
        opts = _opts(precision, _lib.MM_LAYOUT_POINTS, pps=points_per_set or n, hbar=hbar)
    F = torch.empty(n, dtype=torch.float64, device=v.device)
    G = torch.empty((n, 2 * nb + 1), dtype=torch.float64, device=v.device)
    rc = _lib.load().mm_force_adjoint(pack.handle, beams.handle, _dptr(v), _dptr(z), n,
                                      ctypes.byref(opts), _dptr(F), _dptr(G), _stream_handle(stream))
    _lib.check(rc, "mm_force_adjoint")
    return F, G
