"""The numba CPU-baseline restatement equals the C oracle bit for bit."""
import numpy as np

from conftest import golden
from oracle import rate_eq as orc


def test_numba_grid_equals_c_oracle(mol):
    from oracle import rate_eq_numba as nb
    g = golden("random_points.npz")
    ns, npts = int(g["n_sets"]), int(g["n_pts"])
    sel = lambda a: a.reshape(ns, npts, *a.shape[1:])[:, 0][:4]
    kd, fr, po, s0, B = sel(g["kdir"]), sel(g["freq"]), sel(g["pol"]), sel(g["s0"]), sel(g["B"])
    v = np.linspace(-10, 10, 9)
    z = np.linspace(-1e-2, 1e-2, 11)
    Fn = nb.force_grid(mol, kd, fr, po, s0, B, v, z, n_threads=2)
    Fc = orc.force_batch(mol, kd, fr, po, s0, B, v, z, grid=True, want_pop=False)[0]
    assert np.array_equal(Fn.ravel(), Fc)
