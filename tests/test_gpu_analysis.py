"""Ensemble post-processing on the GPU (molmot_b200.analysis: mm_ensemble_stats
and mm_histogram) against the reference's outputs (tests/golden/
analysis_golden.npz) and the CPU restatement, for the reference's
list-of-tuples input, array input, and a GPU trajectory ensemble."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import analysis as oa

pytestmark = pytest.mark.gpu


def test_analysis_vs_reference_outputs(gpu):
    from molmot_b200 import analysis as an
    g = golden("analysis_golden.npz")
    mass = float(g["mass"])
    for e in ("e0", "e1"):
        t, Z, V = oa.synthetic_ensemble(int(g[f"{e}_seed"]), int(g[f"{e}_n"]), int(g[f"{e}_steps"]))
        res = [(t, Z[i], V[i]) for i in range(Z.shape[0])]
        c, sz, sv, na = an.sigma_vs_time(res, time_bins=40)
        assert np.array_equal(c, g[f"{e}_t"]) and np.array_equal(na, g[f"{e}_na"])
        assert np.allclose(sz, g[f"{e}_sz"], rtol=1e-12, atol=0, equal_nan=True)
        assert np.allclose(sv, g[f"{e}_sv"], rtol=1e-12, atol=0, equal_nan=True)
        arrays = (t, torch.as_tensor(Z, device=gpu), torch.as_tensor(V, device=gpu))
        assert np.allclose(an.temperature_vs_time(arrays, mass, time_bins=40)[1], g[f"{e}_T"],
                           rtol=1e-12, equal_nan=True)
        assert np.allclose(an.density_vs_time(arrays, N_total=2000, time_bins=40)[1], g[f"{e}_n0"],
                           rtol=1e-11)
        assert an.capture_fraction(res, r_max=3e-3, t_min=1e-3) == float(g[f"{e}_capture"])
        assert an.capture_fraction(arrays, r_max=5e-3, t_min=0.0) == float(g[f"{e}_capture_t0"])
        assert np.array_equal(an.survived_mask(arrays), g[f"{e}_survived"])
        assert [an.survived(r) for r in res] == list(g[f"{e}_survived"])
        S = Z.shape[1]
        assert an.gaussian_fit(Z[:, S // 2]) == pytest.approx(float(g[f"{e}_gfit"]), rel=1e-8)
        assert an.gaussian_fit(Z[:, -1], bins=80, range_mm=(-5, 5)) == \
            pytest.approx(float(g[f"{e}_gfit_final"]), rel=1e-8)
        assert an.maxwell_boltzmann_fit_1d(V[:, -1], mass) == pytest.approx(float(g[f"{e}_mbfit"]),
                                                                            rel=1e-8)


def test_histogram_matches_numpy_bin_for_bin(gpu):
    """Edges, the upper bound (last bin), values outside the range and NaN."""
    from molmot_b200.analysis import histogram
    rng = np.random.default_rng(3)
    for bins, lo, hi in [(200, -2e-3, 2e-3), (100, -1.0, 1.0), (7, 0.1, 0.7), (1, -1.0, 3.0)]:
        edges = np.linspace(lo, hi, bins + 1)
        x = np.concatenate([rng.uniform(lo - 0.3 * (hi - lo), hi + 0.3 * (hi - lo), 20000), edges,
                            np.nextafter(edges, -np.inf), np.nextafter(edges, np.inf), [np.nan, hi, lo]])
        c, e = histogram(x, bins, lo, hi)
        ref_c, ref_e = np.histogram(x, bins=bins, range=(lo, hi))
        assert np.array_equal(c, ref_c), (bins, lo, hi)
        assert np.array_equal(e, ref_e)


def test_analysis_of_gpu_trajectory_ensemble(mol, gpu):
    """The reductions applied to a GPU-integrated 1D ensemble (saved
    trajectories, escapes included) equal the CPU restatement's."""
    from molmot_b200 import analysis as an
    from molmot_b200.engine import BeamSets, traj
    from molmot_b200.fields import make_dc_mot_beams
    bs = BeamSets.from_beams(make_dc_mot_beams(mol, -0.20, 0.70, 1.0), 0.16)
    rng = np.random.default_rng(9)
    from molmot_b200.engine import pack_for
    out = traj(pack_for(mol), bs, rng.normal(0, 3e-3, 512), rng.normal(0, 3.0, 512), 1e-6, 3000,
               save_full=True)
    t, Zd, Vd = an.ensemble_from_traj(out, 1e-6)
    Z, V = Zd.cpu().numpy(), Vd.cpu().numpy()
    assert (np.abs(Z[:, -1]) > oa.R_ESCAPE).any()  # some molecules escaped
    c, sz, sv, na = an.sigma_vs_time((t, Zd, Vd), time_bins=30)
    c2, sz2, sv2, na2 = oa.sigma_vs_time(t, Z, V, 30)
    assert np.array_equal(na, na2)
    assert np.allclose(sz, sz2, rtol=1e-12, equal_nan=True) and np.allclose(sv, sv2, rtol=1e-12, equal_nan=True)
    assert np.allclose(an.temperature_vs_time((t, Zd, Vd), mol.mass, 30)[1],
                       oa.temperature_vs_time(t, Z, V, mol.mass, 30)[1], rtol=1e-12, equal_nan=True)
    assert an.capture_fraction((t, Zd, Vd), 3e-3, 1e-3) == oa.capture_fraction(t, Z, 3e-3, 1e-3)
