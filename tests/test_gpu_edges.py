"""Edge cases of the force entry points, every form against the oracle:
  * the maximum beam count (32 beams with random polarisations, directions,
    frequencies and intensities);
  * non-finite inputs: a NaN or infinite velocity or position gives F = NaN
    with the non-finite status bit in every form, and the finite points of
    the same batch are unaffected (the reference's elimination returns NaN
    for NaN inputs and F = 0 for infinite ones, through IEEE 1/inf; these
    kernels' reciprocals do not define 1/inf, so the point is flagged);
  * empty batches (zero points or particles) return without work in every
    entry point, with null arrays allowed.
"""
import numpy as np
import pytest
import torch

from oracle import rate_eq as orc

pytestmark = pytest.mark.gpu

FORMS = [("fp64", 1e-10), ("fp64_reduced", 1e-10), ("fp32", 1e-6)]


@pytest.fixture(scope="module")
def pack(mol, gpu):
    from molmot_b200.engine import MoleculePack
    return MoleculePack(mol)


def _max_beam_sets(mol, n_sets, seed):
    from molmot_b200 import _lib
    rng = np.random.default_rng(seed)
    nb = _lib.MM_MAX_BEAMS
    E = mol.energies
    refs = np.array([E[15] - E[0], E[15] - E[9], E[14] - E[2], E[13] - E[8]])
    freq = refs[rng.integers(0, 4, (n_sets, nb))] + rng.uniform(-30e6, 5e6, (n_sets, nb))
    pol = rng.integers(0, 3, (n_sets, nb)).astype(np.int32)
    kdir = rng.choice([-1.0, 1.0], (n_sets, nb)) * rng.uniform(0.3, 1.0, (n_sets, nb))
    s0 = 10 ** rng.uniform(-1.5, 0.5, (n_sets, nb))
    B = rng.uniform(0.05, 0.4, n_sets)
    return kdir, freq, pol, s0, B


@pytest.mark.parametrize("precision,tol", FORMS)
def test_maximum_beam_count(mol, pack, precision, tol):
    from molmot_b200.engine import BeamSets, force_batch
    params = _max_beam_sets(mol, 4, 17)
    rng = np.random.default_rng(18)
    npt = 48
    v = rng.uniform(-10, 10, 4 * npt)
    z = rng.uniform(-1e-2, 1e-2, 4 * npt)
    out = force_batch(pack, BeamSets(*params), v, z, points_per_set=npt, precision=precision)
    Fo, popo, Ro, sto = orc.force_batch(mol, *params, v, z, points_per_set=npt)
    F = out["F"].cpu().numpy().reshape(4, -1)
    err = np.abs(F - Fo.reshape(4, -1)).max(1) / np.abs(Fo.reshape(4, -1)).max(1)
    assert err.max() < tol, err
    assert np.abs(out["R"].cpu().numpy() - Ro).max() / np.abs(Ro).max() < tol


@pytest.mark.parametrize("precision", ["fp64", "fp64_reduced", "fp32"])
def test_nonfinite_inputs_follow_reference(mol, pack, precision):
    import bench
    from molmot_b200.engine import BeamSets, force_batch
    params = bench.make_params(mol, 1, 5)
    # five non-finite points among finite ones spanning the map (the finite
    # points set the scale max|F| of the tolerance, as in every map test)
    v = np.concatenate([[np.nan, np.inf, -np.inf, 1.0, 0.5], np.linspace(-8, 8, 27)])
    z = np.concatenate([[0.0, 1e-3, -2e-3, np.nan, np.inf], np.linspace(-8e-3, 8e-3, 27)])
    n = v.size
    out = force_batch(pack, BeamSets(*params), v, z, points_per_set=n, precision=precision)
    Fo, popo, Ro, sto = orc.force_batch(mol, *params, v, z, points_per_set=n)
    F = out["F"].cpu().numpy()
    st = out["status"].cpu().numpy()
    bad = ~(np.isfinite(v) & np.isfinite(z))
    assert np.all(np.isnan(F[bad])) and np.all(st[bad] & 2)
    assert np.all(np.isnan(Fo[np.isnan(v) | np.isnan(z)]))  # the reference agrees on NaN inputs
    scale = np.abs(Fo[~bad]).max()
    assert np.abs(F[~bad] - Fo[~bad]).max() <= (1e-6 if precision == "fp32" else 1e-10) * scale
    assert np.array_equal(st[~bad], sto[~bad])


def test_empty_batches(mol, pack):
    from molmot_b200.engine import BeamSets, force_adjoint, force_batch, traj
    from molmot_b200.trajgrad import traj_grad
    import bench
    bs = BeamSets(*bench.make_params(mol, 2, 3))
    e = np.zeros(0)
    for precision in ("fp64", "fp64_reduced", "fp32"):
        out = force_batch(pack, bs, e, e, precision=precision)
        assert out["F"].numel() == 0 and out["pop"].shape == (0, 12)
    for precision in ("fp64", "fp64_reduced"):
        F, G = force_adjoint(pack, bs, e, e, precision=precision)
        assert F.numel() == 0 and G.shape == (0, 17)
    for ndim in (1, 3):
        o = traj(pack, bs, np.zeros((0, ndim)), np.zeros((0, ndim)), 1e-6, 10, ndim=ndim)
        assert o["r_final"].shape == (0, ndim)
    g = traj_grad(pack, bs, np.zeros((0, 3)), np.zeros((0, 3)), 1e-6, 10, n_par=1, bprime_par=0)
    assert g["dv"].shape == (0, 3, 1)
    torch.cuda.synchronize()
