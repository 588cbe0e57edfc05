"""TEST INFRASTRUCTURE ONLY -- ctypes binding of oracle/rate_eq_oracle.c.

Functions take a duck-typed molecule (attributes ``energies``,
``d_squared``, ``zeeman_z_diag``, ``Gamma``, ``k``, ``n_ground``,
``n_excited``; both molmot's ``MolecularData`` and molmot_b200's qualify)
and beams as flat arrays ``(kdir, freq, pol, s0)``.

Reference functions restated (paths within the molmot project):
  molmot/obe/rate_equations_jit.py:18-145 (_rate_eq_core, default flags)
  molmot/obe/rate_equations.py:24-191 (solve_rate_equations, TWO_PASS)
  molmot/propagation/trajectories_jit.py:18-58 (_trajectory_1d_jit)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc_rate_eq.so")

#: hbar hard-coded by the reference's numba core and CUDA kernels
HBAR_JIT = 1.0545718e-34
#: CODATA hbar of molmot/constants.py:18, used by the pure-Python path
HBAR_CODATA = 1.054571817e-34

UNIFORM_FALLBACK = 1
TWO_PASS = 2

_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


def build() -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_rate_eq_point.restype = ctypes.c_int
        L.orc_rate_eq_point.argtypes = [
            ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
            ctypes.c_int, _dp, _dp, _dp, _dp,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
            _dp, _dp, _dp]
        L.orc_force_batch.restype = ctypes.c_int
        L.orc_force_batch.argtypes = [
            ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp,
            ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
            _dp, _dp, ctypes.c_int,
            _dp, _dp, _dp, _ip]
        L.orc_traj1d.restype = ctypes.c_int
        L.orc_traj1d.argtypes = [
            ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
            ctypes.c_int, _dp, _dp, _dp, _dp,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
            ctypes.c_double, ctypes.c_int64, _dp, _dp,
            ctypes.c_int, _dp, _dp, _ip, _dp, _dp]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_max_threads.argtypes = []
        _lib = L
    return _lib


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _mol_arrays(mol):
    return (int(mol.n_ground), int(mol.n_excited), _c(mol.energies),
            _c(mol.d_squared).reshape(-1), _c(mol.zeeman_z_diag))


def beam_arrays(beams):
    """(kdir_z, freq, pol-as-float, s0) arrays from a LaserBeam list."""
    return (np.array([b.kdir_z for b in beams], dtype=np.float64),
            np.array([b.freq_offset for b in beams], dtype=np.float64),
            np.array([b.polarization for b in beams], dtype=np.float64),
            np.array([b.s0 for b in beams], dtype=np.float64))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def point(mol, beams, v, z, B_gradient, Gamma_eff=1.0, hbar=HBAR_JIT, flags=0):
    """One point; returns (F, p, R, status) like _rate_eq_core (+ status)."""
    n_g, n_e, E, d2, zd = _mol_arrays(mol)
    kdir, freq, pol, s0 = [_c(a) for a in (beams if isinstance(beams, tuple) else beam_arrays(beams))]
    F = np.zeros(1)
    R = np.zeros(1)
    p = np.zeros(n_g)
    st = lib().orc_rate_eq_point(n_g, n_e, _p(E), _p(d2), _p(zd), len(kdir), _p(kdir), _p(freq),
                                 _p(pol), _p(s0), float(v), float(z), float(B_gradient),
                                 float(mol.Gamma), float(mol.k), float(Gamma_eff), float(hbar),
                                 int(flags), _p(F), _p(p), _p(R))
    if st < 0:
        raise ValueError("oracle: invalid sizes")
    return float(F[0]), p, float(R[0]), int(st)


def force_batch(mol, kdir, freq, pol, s0, B_gradient, v, z, *, grid=False,
                points_per_set=None, Gamma_eff=1.0, hbar=HBAR_JIT, flags=0,
                n_threads=0, want_pop=True):
    """Batch over parameter sets.

    ``kdir, freq, pol, s0`` are [n_sets, n_b]; ``B_gradient`` is [n_sets].
    With ``grid=True`` the points are the per-set outer product of ``v``
    (nv,) and ``z`` (nz,), flattened as (set, iv, iz).  Otherwise ``v`` and
    ``z`` are per-point arrays and point i belongs to set i // points_per_set.
    Returns (F, pop, R, status) flattened over points.
    """
    n_g, n_e, E, d2, zd = _mol_arrays(mol)
    kdir, freq, pol, s0 = [np.atleast_2d(_c(a)) for a in (kdir, freq, pol, s0)]
    n_sets, n_b = kdir.shape
    Bg = _c(np.broadcast_to(np.asarray(B_gradient, dtype=np.float64), (n_sets,)))
    v = _c(v)
    z = _c(z)
    if grid:
        nv, nz = v.size, z.size
        n = n_sets * nv * nz
        pps = nv * nz
    else:
        nv = nz = 0
        n = v.size
        pps = int(points_per_set) if points_per_set else n
    F = np.zeros(n)
    R = np.zeros(n)
    st = np.zeros(n, dtype=np.int32)
    pop = np.zeros((n, n_g)) if want_pop else None
    rc = lib().orc_force_batch(n_g, n_e, _p(E), _p(d2), _p(zd), float(mol.Gamma), float(mol.k),
                               float(Gamma_eff), float(hbar), int(flags), n_b, n_sets,
                               _p(kdir), _p(freq), _p(pol), _p(s0), _p(Bg), n, pps, nv, nz,
                               _p(v), _p(z), int(n_threads), _p(F), _p(pop), _p(R),
                               st.ctypes.data_as(_ip))
    if rc != 0:
        raise ValueError("oracle: invalid arguments")
    return F, pop, R, st


def traj1d(mol, beams, B_gradient, z0, v0, dt, n_steps, *, Gamma_eff=1.0, hbar=HBAR_JIT,
           z_escape=0.015, save_full=False, n_threads=0, flags=0):
    """N 1D Euler trajectories.  Returns (z_f, v_f, n_actual, z_traj, v_traj)."""
    n_g, n_e, E, d2, zd = _mol_arrays(mol)
    kdir, freq, pol, s0 = [_c(a) for a in (beams if isinstance(beams, tuple) else beam_arrays(beams))]
    z0 = _c(np.atleast_1d(z0))
    v0 = _c(np.atleast_1d(v0))
    N = z0.size
    zf = np.zeros(N)
    vf = np.zeros(N)
    na = np.zeros(N, dtype=np.int32)
    zt = np.zeros((N, n_steps)) if save_full else None
    vt = np.zeros((N, n_steps)) if save_full else None
    rc = lib().orc_traj1d(n_g, n_e, _p(E), _p(d2), _p(zd), float(mol.Gamma), float(mol.k),
                          float(Gamma_eff), float(hbar), int(flags), len(kdir), _p(kdir),
                          _p(freq), _p(pol), _p(s0), float(B_gradient), float(mol.mass),
                          float(dt), int(n_steps), float(z_escape), N, _p(z0), _p(v0),
                          int(n_threads), _p(zf), _p(vf), na.ctypes.data_as(_ip), _p(zt), _p(vt))
    if rc != 0:
        raise ValueError("oracle: invalid arguments")
    return zf, vf, na, zt, vt
