"""CaF and CaOH (12 ground + 4 excited levels, 30 active couplings against
SrOH's 39) through every 1D force form, against the reference's
_rate_eq_core outputs in tests/golden/molecules_golden.npz:
plain FP64 and FP64-reduced to 1e-10 of max|F| per parameter set, FP32-bulk
to 1e-6; the two adjoints agree to 1e-9 of the largest gradient component;
plain FP64 trajectories equal the C oracle's."""
import numpy as np
import pytest
import torch

from molecules_fixture import NAMES, load, points, set_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp64_reduced", 1e-10), ("fp32", 1e-6)])
def test_forces_match_reference(gpu, name, precision, tol):
    from molmot_b200.engine import BeamSets, MoleculePack, force_batch
    mol, g = load(name)
    ns, npt, sets, v, z, F, p, R = points(g, name)
    out = force_batch(MoleculePack(mol), BeamSets(*sets), v, z, points_per_set=npt, precision=precision)
    assert set_err(out["F"].cpu().numpy(), F, ns).max() < tol
    assert np.max(np.abs(out["R"].cpu().numpy() - R)) / np.abs(R).max() < tol
    assert np.max(np.abs(out["pop"].cpu().numpy().reshape(-1, 12) - p)) < 10 * tol


@pytest.mark.parametrize("name", NAMES)
def test_adjoint_forms_agree(gpu, name):
    from molmot_b200.engine import BeamSets, MoleculePack, force_adjoint
    mol, g = load(name)
    ns, npt, sets, v, z, F, _, _ = points(g, name)
    pk, bs = MoleculePack(mol), BeamSets(*sets)
    Fp, Gp = force_adjoint(pk, bs, v, z, points_per_set=npt, precision="fp64")
    Fr, Gr = force_adjoint(pk, bs, v, z, points_per_set=npt, precision="fp64_reduced")
    assert set_err(Fp.cpu().numpy(), F, ns).max() < 1e-10
    scale = Gp.view(ns, npt, -1).abs().amax(dim=1, keepdim=True)
    err = ((Gr - Gp).view(ns, npt, -1).abs() / scale).nan_to_num(0.0)
    assert float(err.max()) < 1e-9


@pytest.mark.parametrize("name", NAMES)
def test_trajectories_match_oracle(gpu, name):
    from molmot_b200.engine import BeamSets, MoleculePack, traj1d
    from molmot_b200.fields import beam_arrays, make_dc_mot_beams
    from oracle import rate_eq as orc
    mol, _ = load(name)
    kd, fr, po, s0 = beam_arrays(make_dc_mot_beams(mol, delta_Gamma=-0.25, split_Gamma=0.6, s0=1.5))
    rng = np.random.default_rng(9)
    z0, v0 = rng.normal(0, 2e-3, 16), rng.normal(0, 1.0, 16)
    zf, vf, na, _, _ = traj1d(MoleculePack(mol), BeamSets(kd[None], fr[None], po[None], s0[None], [0.16]),
                              z0, v0, 1e-6, 400)
    zo, vo, nao, _, _ = orc.traj1d(mol, (kd, fr, po, s0), 0.16, z0, v0, 1e-6, 400)
    assert np.array_equal(na.cpu().numpy(), nao)
    assert np.max(np.abs(zf.cpu().numpy() - zo)) < 1e-12
    assert np.max(np.abs(vf.cpu().numpy() - vo)) < 1e-9
