"""The CPU restatement of molmot/mot/analysis.py (oracle/analysis.py) against
the reference's own outputs on seeded synthetic ensembles
(tests/golden/analysis_golden.npz)."""
import numpy as np

from conftest import golden
from oracle import analysis as oa


def test_oracle_matches_reference_analysis():
    g = golden("analysis_golden.npz")
    mass = float(g["mass"])
    for e in ("e0", "e1"):
        t, Z, V = oa.synthetic_ensemble(int(g[f"{e}_seed"]), int(g[f"{e}_n"]), int(g[f"{e}_steps"]))
        c, sz, sv, na = oa.sigma_vs_time(t, Z, V, 40)
        assert np.array_equal(c, g[f"{e}_t"]) and np.array_equal(na, g[f"{e}_na"])
        assert np.allclose(sz, g[f"{e}_sz"], rtol=1e-14, atol=0, equal_nan=True)
        assert np.allclose(sv, g[f"{e}_sv"], rtol=1e-14, atol=0, equal_nan=True)
        assert np.allclose(oa.temperature_vs_time(t, Z, V, mass, 40)[1], g[f"{e}_T"], rtol=1e-14,
                           equal_nan=True)
        assert np.allclose(oa.density_vs_time(t, Z, V, 2000, 40)[1], g[f"{e}_n0"], rtol=1e-13)
        assert oa.capture_fraction(t, Z, 3e-3, 1e-3) == float(g[f"{e}_capture"])
        assert oa.capture_fraction(t, Z, 5e-3, 0.0) == float(g[f"{e}_capture_t0"])
        assert np.array_equal(oa.survived(Z), g[f"{e}_survived"])
        S = Z.shape[1]
        assert oa.gaussian_fit(Z[:, S // 2]) == float(g[f"{e}_gfit"])
        assert oa.gaussian_fit(Z[:, -1], bins=80, range_mm=(-5, 5)) == float(g[f"{e}_gfit_final"])
        assert oa.maxwell_boltzmann_fit_1d(V[:, -1], mass) == float(g[f"{e}_mbfit"])
