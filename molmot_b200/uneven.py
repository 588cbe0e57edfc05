"""Uneven batches: many different molecules, each with its own beams and
number of points, in one persistent launch per size class (C ABI:
mm_bank_*, mm_uneven_plan_*, mm_uneven_force).

``UnevenBatch.force`` runs the persistent kernels; ``UnevenBatch.graph``
captures the whole call (counter reset + launches) in a CUDA graph for
replay; ``UnevenBatch.autotune`` times warps-per-CTA candidates for every
size class present and keeps the fastest (cached per GPU name and size-class
occupancy).  ``make_uneven_workload`` builds the seeded synthetic batch:
molecules with n_ground in {4..48} and n_excited in {4..16}, 64..4096
random (v, z) points each.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .constants import HBAR_JIT
from .engine import BeamSets, _device, _dptr, _stream_handle, _to_dev, molecule_arrays

_TUNE_CACHE: Dict[tuple, tuple] = {}


class MoleculeBank:
    """Device copy of many molecules (1D fields)."""

    def __init__(self, mols: Sequence):
        self.mols = list(mols)
        arrs = [molecule_arrays(m) for m in self.mols]
        self._keep = arrs
        descs = (_lib.MolDesc * len(arrs))()
        for d, a, m in zip(descs, arrs, self.mols):
            d.n_ground, d.n_excited = a["n_g"], a["n_e"]
            d.energies = ctypes.c_void_p(a["E"].ctypes.data)
            d.d_squared = ctypes.c_void_p(a["d2"].ctypes.data)
            d.zeeman_z_diag = ctypes.c_void_p(a["zd"].ctypes.data)
            d.Gamma, d.k, d.mass = float(m.Gamma), float(m.k), float(m.mass)
        _device()
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mm_bank_create(descs, len(arrs), ctypes.byref(h)), "mm_bank_create")
        self.handle = h
        self.n_ground = np.array([a["n_g"] for a in arrs])
        self.n_excited = np.array([a["n_e"] for a in arrs])

    def size_class(self) -> np.ndarray:
        return np.where(self.n_ground <= 16, 0, np.where(self.n_ground <= 32, 1, 2))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.load().mm_bank_destroy(h)
            except Exception:
                pass
            self.handle = None


class UnevenBatch:
    """Forces at (v[i], z[i]) for points grouped by molecule:
    molecule m owns points [offsets[m], offsets[m+1])."""

    def __init__(self, bank: MoleculeBank, point_counts: Sequence[int], beams: BeamSets,
                 warps_per_cta=(0, 0, 0), chunk_groups: int = 8, hbar: float = HBAR_JIT):
        if beams.n_sets != len(bank.mols):
            raise ValueError("one beam set per molecule is required")
        self.bank, self.beams, self.hbar = bank, beams, hbar
        self.offsets = np.concatenate([[0], np.cumsum(np.asarray(point_counts, dtype=np.int64))])
        self.n_points = int(self.offsets[-1])
        self._off_c = np.ascontiguousarray(self.offsets, dtype=np.int64)
        self.chunk_groups = chunk_groups
        self._plan(tuple(warps_per_cta))

    def _plan(self, wpc):
        old = getattr(self, "plan", None)
        o = _lib.UnevenOpts()
        for i in range(3):
            o.warps_per_cta[i] = int(wpc[i])
        o.chunk_groups = int(self.chunk_groups)
        off = np.ascontiguousarray(self.offsets, dtype=np.int64)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mm_uneven_plan_create(self.bank.handle,
                                                     off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                                     ctypes.byref(o), ctypes.byref(h)),
                   "mm_uneven_plan_create")
        self.plan = h
        self.wpc = tuple(wpc)
        if old is not None and old.value:
            _lib.load().mm_uneven_plan_destroy(old)

    def force(self, v, z, persistent: bool = True, out=None, stream=None, uniform_fallback=False):
        v = _to_dev(v)
        z = _to_dev(z)
        if v.numel() != self.n_points or z.numel() != self.n_points:
            raise ValueError(f"expected {self.n_points} points")
        if out is None:
            out = {"F": torch.empty(self.n_points, dtype=torch.float64, device=v.device),
                   "R": torch.empty(self.n_points, dtype=torch.float64, device=v.device),
                   "status": torch.empty(self.n_points, dtype=torch.int32, device=v.device)}
        rc = _lib.load().mm_uneven_force(self.plan, self.beams.handle, _dptr(v), _dptr(z),
                                         float(self.hbar), 1 if uniform_fallback else 0,
                                         1 if persistent else 0, _dptr(out["F"]),
                                         _dptr(out.get("R")), _dptr(out.get("status")),
                                         _stream_handle(stream))
        _lib.check(rc, "mm_uneven_force")
        return out

    def force_static(self, v, z, out, stream=None, uniform_fallback=False):
        """The same forces through mm_uneven_force_static, which allocates
        nothing: the caller passes `out` (F, and optionally R and status) and
        the work list lives in the library's fixed device array.  Two calls
        race on that array unless the second is ordered after the first on
        the GPU (the same stream, or a wait on an event recorded after the
        first).  v and z that are not float64, contiguous and on the current
        CUDA device are converted (a copy, which allocates); `out` must
        already be in that form."""
        v = _to_dev(v)
        z = _to_dev(z)
        if v.numel() != self.n_points or z.numel() != self.n_points:
            raise ValueError(f"expected {self.n_points} points")
        check_static_out(out, self.n_points, v.device)
        o = _lib.UnevenOpts()
        for i in range(3):
            o.warps_per_cta[i] = int(self.wpc[i])
        o.chunk_groups = int(self.chunk_groups)
        rc = _lib.load().mm_uneven_force_static(
            self.bank.handle, self.beams.handle,
            self._off_c.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(o),
            _dptr(v), _dptr(z), float(self.hbar), 1 if uniform_fallback else 0,
            _dptr(out["F"]), _dptr(out.get("R")), _dptr(out.get("status")), _stream_handle(stream))
        _lib.check(rc, "mm_uneven_force_static")
        return out

    def graph(self, v, z):
        """Capture one persistent call in a CUDA graph; returns (graph, out, v, z)
        -- replay with graph.replay() after writing new points into v and z."""
        v = _to_dev(v).clone()
        z = _to_dev(z).clone()
        out = self.force(v, z)  # warm-up outside capture (kernel attributes, module load)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.force(v, z, out=out, stream=s)
        torch.cuda.current_stream().wait_stream(s)
        return g, out, v, z

    def autotune(self, v, z, candidates=(2, 4, 8), reps: int = 3):
        """Pick warps per CTA for every size class present by timing the full
        batch with one class varied at a time (the others at their current
        choice).  Results are cached per GPU and class mix."""
        cls = self.bank.size_class()
        present = tuple(int((cls == c).any()) for c in range(3))
        key = (torch.cuda.get_device_name(), present, self.n_points, self.chunk_groups)
        if key in _TUNE_CACHE:
            self._plan(_TUNE_CACHE[key])
            return self.wpc
        v = _to_dev(v)
        z = _to_dev(z)
        best = list(self.wpc if all(self.wpc) else (4, 2, 2))
        for c in range(3):
            if not present[c]:
                continue
            times = {}
            for w in candidates:
                trial = list(best)
                trial[c] = w
                self._plan(tuple(trial))
                try:  # a shape whose shared memory exceeds the SM's is refused, not run
                    self.force(v, z)
                except RuntimeError:
                    continue
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    self.force(v, z)
                e1.record()
                torch.cuda.synchronize()
                times[w] = e0.elapsed_time(e1) / reps
            best[c] = min(times, key=times.get)
        self._plan(tuple(best))
        _TUNE_CACHE[key] = tuple(best)
        return self.wpc

    def __del__(self):
        h = getattr(self, "plan", None)
        if h is not None and h.value:
            try:
                _lib.load().mm_uneven_plan_destroy(h)
            except Exception:
                pass
            self.plan = None


def sample_molecules(n_ground, n_excited, counts, per_class: int = 4, seed: int = 0):
    """Indices of a parity sample of an uneven batch: per size class
    (n_ground <= 16, <= 32, <= 48) the molecule with the most points, the
    one with the most ground states, the one with the most excited states,
    and random others of the class up to ``per_class`` (fewer if the class
    is smaller), in ascending order."""
    ng = np.asarray(n_ground)
    ne = np.asarray(n_excited)
    cnt = np.asarray(counts)
    cls = np.where(ng <= 16, 0, np.where(ng <= 32, 1, 2))
    rng = np.random.default_rng(seed)
    picked = []
    for c in range(3):
        idx = np.flatnonzero(cls == c)
        if idx.size == 0:
            continue
        chosen = []
        for key in (cnt, ng, ne):
            i = int(idx[np.argmax(key[idx])])
            if i not in chosen:
                chosen.append(i)
        rest = [int(i) for i in rng.permutation(idx) if int(i) not in chosen]
        chosen += rest[:max(0, per_class - len(chosen))]
        picked += chosen[:max(per_class, 3)]
    return sorted(picked)


_STATIC_OUT = {"F": torch.float64, "R": torch.float64, "status": torch.int32}


def check_static_out(out, n_points: int, device: torch.device) -> None:
    """Checks the caller's output buffers of ``UnevenBatch.force_static``
    before their addresses go to the kernels: F is required, R and status
    optional; each must have its dtype (float64, float64, int32), be
    contiguous, hold n_points elements and live on ``device``.  Raises
    ValueError otherwise (a host tensor or a short buffer would make the
    kernels write outside it)."""
    if not isinstance(out, dict) or out.get("F") is None:
        raise ValueError("out must be a dict holding at least the 'F' tensor")
    for key in out:
        if key not in _STATIC_OUT:
            raise ValueError(f"unknown output {key!r}; expected F, R or status")
    for key, dtype in _STATIC_OUT.items():
        t = out.get(key)
        if t is None:
            continue
        if not isinstance(t, torch.Tensor):
            raise ValueError(f"out[{key!r}] must be a torch tensor")
        if t.dtype != dtype:
            raise ValueError(f"out[{key!r}] must be {dtype}, got {t.dtype}")
        if t.device != device:
            raise ValueError(f"out[{key!r}] must be on {device}, got {t.device}")
        if not t.is_contiguous():
            raise ValueError(f"out[{key!r}] must be contiguous")
        if t.numel() != n_points:
            raise ValueError(f"out[{key!r}] must hold {n_points} elements, got {t.numel()}")


def make_uneven_workload(n_mol: int = 2048, seed: int = 20261203, min_pts: int = 64,
                         max_pts: int = 4096, ng_range=(4, 48), ne_range=(4, 16)):
    """Seeded synthetic batch: (molecules, point counts, beam arrays
    (kdir, freq, pol, s0) [n_mol, 8], B' [n_mol], v, z)."""
    from .molecules.synthetic import synthetic_molecule, dc_beams_for
    rng = np.random.default_rng(seed)
    ng = rng.integers(ng_range[0], ng_range[1] + 1, n_mol)
    ne = rng.integers(ne_range[0], ne_range[1] + 1, n_mol)
    counts = rng.integers(min_pts, max_pts + 1, n_mol)
    mols = [synthetic_molecule(int(a), int(b), seed * 7919 + i) for i, (a, b) in enumerate(zip(ng, ne))]
    beams = [dc_beams_for(m) for m in mols]
    kdir = np.stack([b[0] for b in beams])
    freq = np.stack([b[1] for b in beams])
    pol = np.stack([b[2] for b in beams])
    s0 = np.stack([b[3] for b in beams])
    B = rng.uniform(5, 40, n_mol) * 1e-2
    n = int(counts.sum())
    v = rng.uniform(-10.0, 10.0, n)
    z = rng.uniform(-1e-2, 1e-2, n)
    return mols, counts, (kdir, freq, pol, s0), B, v, z
