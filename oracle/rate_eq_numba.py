"""TEST INFRASTRUCTURE / CPU BASELINE ONLY -- numba restatement of the
reference's rate-equation core, driven by a parallel harness over points.

The reference's CPU hot path is numba-compiled Python
(molmot/obe/rate_equations_jit.py:18-145, _rate_eq_core).  This module
restates that algorithm (same operation order, JIT hbar by default) so the
CPU baseline of bench.py runs the reference's own technology on every host
core (``prange`` over points).  It is checked bit for bit against
oracle/rate_eq_oracle.c in tests/test_oracle_numba.py.
"""
from __future__ import annotations

import os

os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/molmot_b200_numba_cache")

import numpy as np  # noqa: E402
from numba import njit, prange  # noqa: E402
import numba  # noqa: E402


@njit(cache=True)
def _branching(d2, n_g, n_e):
    BR = np.zeros((n_e, n_g))
    for ie in range(n_e):
        total = 0.0
        for ig in range(n_g):
            for q in range(3):
                total += d2[ig, ie, q]
        if total > 1e-30:
            for ig in range(n_g):
                s = 0.0
                for q in range(3):
                    s += d2[ig, ie, q]
                BR[ie, ig] = s / total
    return BR


@njit(cache=True)
def core(E, d2, zd, BR, kdir, freq, pol, s0, v, z, Bg, Gamma, k_wave, Geff, hbar_val, n_g, n_e):
    """One point; returns F (the populations and rate are computed but only
    the force is returned, as the force-map workload needs)."""
    n_b = kdir.shape[0]
    B_gauss = Bg * z * 1e4
    gh = Gamma / 2.0
    gh2 = gh * gh
    Es = np.empty(n_g + n_e)
    for i in range(n_g + n_e):
        Es[i] = E[i] + B_gauss * zd[i] * Gamma / (2.0 * np.pi)
    R = np.zeros((n_g, n_e))
    Ft = np.zeros((n_g, n_e))
    st = np.zeros(n_g)
    for ib in range(n_b):
        kd = kdir[ib]
        q = pol[ib]
        dop = -k_wave * kd * v / (2.0 * np.pi)
        for ig in range(n_g):
            for ie in range(n_e):
                dd = d2[ig, ie, q]
                if dd < 1e-15:
                    continue
                om = Es[n_g + ie] - Es[ig]
                de = (freq[ib] + dop - om) * 2.0 * np.pi
                L = gh2 / (de * de + gh2)
                ru = gh * s0[ib] * dd * L * Geff
                R[ig, ie] += ru
                Ft[ig, ie] += hbar_val * k_wave * kd * ru
                st[ig] += s0[ib] * dd * L
    for ig in range(n_g):
        sc = 1.0 / (1.0 + st[ig])
        for ie in range(n_e):
            R[ig, ie] *= sc
            Ft[ig, ie] *= sc
    n = n_g
    A = np.zeros((n, n))
    for ig in range(n_g):
        for ie in range(n_e):
            A[ig, ig] -= R[ig, ie]
        for ik in range(n_g):
            for ie in range(n_e):
                A[ig, ik] += R[ik, ie] * BR[ie, ig]
    for j in range(n):
        A[n - 1, j] = 1.0
    b = np.zeros(n)
    b[n - 1] = 1.0
    for col in range(n):
        mx = abs(A[col, col])
        mr = col
        for row in range(col + 1, n):
            if abs(A[row, col]) > mx:
                mx = abs(A[row, col])
                mr = row
        if mr != col:
            for j in range(n):
                t = A[col, j]
                A[col, j] = A[mr, j]
                A[mr, j] = t
            t = b[col]
            b[col] = b[mr]
            b[mr] = t
        for row in range(col + 1, n):
            if abs(A[col, col]) < 1e-30:
                continue
            f = A[row, col] / A[col, col]
            for j in range(col, n):
                A[row, j] -= f * A[col, j]
            b[row] -= f * b[col]
    p = np.zeros(n)
    for i in range(n - 1, -1, -1):
        s = b[i]
        for j in range(i + 1, n):
            s -= A[i, j] * p[j]
        if abs(A[i, i]) > 1e-30:
            p[i] = s / A[i, i]
    tot = 0.0
    for i in range(n):
        if p[i] < 0:
            p[i] = 0.0
        tot += p[i]
    if tot > 0:
        for i in range(n):
            p[i] /= tot
    F = 0.0
    for ig in range(n_g):
        for ie in range(n_e):
            F += p[ig] * Ft[ig, ie]
    return F


@njit(parallel=True, cache=True)
def grid_harness(E, d2, zd, kdir, freq, pol, s0, Bg, v, z, Gamma, k_wave, Geff, hbar_val,
                 n_g, n_e, out):
    """out[s, iv, iz] = F for every set s (beam rows kdir[s] ...) and grid point."""
    BR = _branching(d2, n_g, n_e)
    n_sets = kdir.shape[0]
    nv = v.shape[0]
    nz = z.shape[0]
    total = n_sets * nv * nz
    for i in prange(total):
        s = i // (nv * nz)
        r = i - s * nv * nz
        out[i] = core(E, d2, zd, BR, kdir[s], freq[s], pol[s], s0[s], v[r // nz], z[r % nz],
                      Bg[s], Gamma, k_wave, Geff, hbar_val, n_g, n_e)


def force_grid(mol, kdir, freq, pol, s0, Bg, v, z, Geff=1.0, hbar=1.0545718e-34, n_threads=None):
    """F[n_sets, nv, nz] on the CPU with numba threads."""
    if n_threads:
        numba.set_num_threads(int(n_threads))
    kdir = np.atleast_2d(np.asarray(kdir, dtype=np.float64))
    n_sets = kdir.shape[0]
    out = np.empty(n_sets * len(v) * len(z))
    grid_harness(np.ascontiguousarray(mol.energies, dtype=np.float64),
                 np.ascontiguousarray(mol.d_squared, dtype=np.float64),
                 np.ascontiguousarray(mol.zeeman_z_diag, dtype=np.float64), kdir,
                 np.atleast_2d(np.asarray(freq, dtype=np.float64)),
                 np.atleast_2d(np.asarray(pol, dtype=np.int64)),
                 np.atleast_2d(np.asarray(s0, dtype=np.float64)),
                 np.broadcast_to(np.asarray(Bg, dtype=np.float64), (n_sets,)).copy(),
                 np.asarray(v, dtype=np.float64), np.asarray(z, dtype=np.float64),
                 float(mol.Gamma), float(mol.k), float(Geff), float(hbar),
                 int(mol.n_ground), int(mol.n_excited), out)
    return out.reshape(n_sets, len(v), len(z))


def threads() -> int:
    return int(numba.get_num_threads())
