"""CaF and CaOH through the host side and the oracle: the molecule container's
derived fields and the DC MOT beam builder equal the reference's, and the C
oracle reproduces the reference's _rate_eq_core forces (the fixtures were
made by the reference itself, tests/golden/make_golden.py molecules)."""
import numpy as np
import pytest

from molecules_fixture import NAMES, load, points, set_err


@pytest.mark.parametrize("name", NAMES)
def test_derived_fields_and_beams(name):
    from molmot_b200.fields import beam_arrays, make_dc_mot_beams
    mol, g = load(name)
    assert (mol.n_ground, mol.n_excited) == (12, 4)
    assert np.array_equal(mol.d_squared, g[f"{name}_d_squared"])
    assert np.array_equal(mol.zeeman_z_diag, g[f"{name}_zeeman_z_diag"])
    for key in ("omega_J12", "omega_J32", "omega_mean"):
        assert getattr(mol, key) == float(g[f"{name}_{key}"]), key
    kd, fr, po, s0 = beam_arrays(make_dc_mot_beams(mol, delta_Gamma=-0.25, split_Gamma=0.6, s0=1.5))
    assert np.array_equal(kd, g[f"{name}_dc_kdir"]) and np.array_equal(fr, g[f"{name}_dc_freq"])
    assert np.array_equal(po, g[f"{name}_dc_pol"]) and np.array_equal(s0, g[f"{name}_dc_s0"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_core(name):
    from oracle import rate_eq as orc
    mol, g = load(name)
    ns, npt, (kd, fr, po, s0, B), v, z, F, p, R = points(g, name)
    Fo, popo, Ro, _ = orc.force_batch(mol, kd, fr, po, s0, B, v, z, points_per_set=npt)
    assert set_err(Fo, F, ns).max() < 1e-12
    assert np.max(np.abs(popo.reshape(-1, 12) - p)) < 1e-12
    assert np.max(np.abs(Ro - R) / np.abs(R).max()) < 1e-12
