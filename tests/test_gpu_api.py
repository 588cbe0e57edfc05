"""The drop-in API (simulators, force scans, trajectories, the molmot_cuda twin)
against values the reference computed (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def rel_to_max(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(a)), np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def sims(mol, gpu):
    from molmot_b200.simulator import DCMOTSimulator, RFMOTSimulator
    return (DCMOTSimulator(mol, delta_Gamma=-0.30, split_Gamma=0.40, s0=1.0, B_gradient=0.16),
            RFMOTSimulator(mol, delta_Gamma=-1.0, s0=1.0, B_gradient=0.16))


def test_force_scan_dc_rf(sims):
    from molmot_b200 import force_scan as fs
    g = golden("force_scan_api.npz")
    dc, rf = sims
    F, P, R = fs.force_vs_z(dc, g["zs"])
    assert rel_to_max(F, g["F_dc_z"]) < 1e-10
    assert np.max(np.abs(P - g["P_dc_z"])) < 1e-10
    assert rel_to_max(R, g["R_dc_z"]) < 1e-10
    assert rel_to_max(fs.force_vs_v(dc, g["vs"]), g["F_dc_v"]) < 1e-10
    F, P, R = fs.force_vs_z(rf, g["zs"])
    assert rel_to_max(F, g["F_rf_z"]) < 1e-10
    assert rel_to_max(fs.force_vs_v(rf, g["vs"]), g["F_rf_v"]) < 1e-10
    for key, fn, sim in [("k_dc", fs.spring_constant, dc), ("a_dc", fs.damping_coefficient, dc),
                         ("k_rf", fs.spring_constant, rf), ("a_rf", fs.damping_coefficient, rf)]:
        assert abs(fn(sim) - g[key]) < 1e-8 * abs(g[key]), key
    assert fs.spring_constant(dc) > 0 and fs.damping_coefficient(dc) > 0


def test_single_point_solvers(mol, sims):
    from molmot_b200.rate_equations import solve_rate_equations_jit, solve_rate_equations
    g = golden("random_points.npz")
    from molmot_b200.fields import LaserBeam
    for i in range(0, 40, 7):
        beams = [LaserBeam(np.array([0, 0, g["kdir"][i][b]]), g["freq"][i][b], int(g["pol"][i][b]),
                           g["s0"][i][b]) for b in range(8)]
        F, p, R = solve_rate_equations_jit(mol, beams, g["v"][i], g["z"][i], g["B"][i])
        assert abs(F - g["F_jit"][i]) <= 1e-12 * abs(g["F_jit"][i]) + 1e-36
        assert np.max(np.abs(p - g["p_jit"][i])) < 1e-12
        F, p, R = solve_rate_equations(mol, beams, g["v"][i], g["z"][i], g["B"][i])
        assert abs(F - g["F_py"][i]) <= 1e-10 * abs(g["F_py"][i]) + 1e-36


def test_simulator_force_types(sims):
    dc, rf = sims
    F, p, R = dc.force(0.0, 1e-3)
    assert isinstance(F, float) and F < 0
    assert abs(p.sum() - 1.0) < 1e-12 and R > 0
    F, p, R = rf.force(0.0, 1e-3)
    assert F < 0


def test_capture_velocity(sims):
    from molmot_b200 import force_scan as fs
    g = golden("force_scan_api.npz")
    assert fs.capture_velocity(sims[0], v_max=6.0, dv=0.5, n_steps=3000) == float(g["vcap_dc"])


def test_optimize_parameters(mol, gpu):
    from molmot_b200 import force_scan as fs
    g = golden("optimize_parameters.npz")
    o = fs.optimize_parameters(mol, {"delta": g["delta"], "split": g["split"]}, 0.16, verbose=False)
    assert rel_to_max(o["K_map"], g["K_map"]) < 1e-8
    assert rel_to_max(o["beta_map"], g["beta_map"]) < 1e-8
    assert o["delta_best"] == float(g["delta_best"]) and o["split_best"] == float(g["split_best"])


def test_trajectories_api(mol, gpu):
    from molmot_b200.simulator import DCMOTSimulator, RFMOTSimulator
    from molmot_b200 import trajectories as tr
    g = golden("trajectory_api_golden.npz")
    dc = DCMOTSimulator(mol, delta_Gamma=-0.20, split_Gamma=0.70, s0=1.0, B_gradient=0.16)
    out = tr.simulate_trajectories_3d(dc, list(g["r0"]), list(g["v0"]), float(g["t_max3"]))
    for i, (t, r, v) in enumerate(out):
        assert np.max(np.abs(r - g["r3"][i])) < 1e-12
        assert np.max(np.abs(v - g["v3"][i])) < 1e-9
    rf = RFMOTSimulator(mol, delta_Gamma=-1.0, s0=1.0, B_gradient=0.16)
    t, z, v = tr.simulate_trajectory(rf, 2e-3, -1.0, float(g["t_max_rf"]))
    assert np.max(np.abs(z - g["z_rf"])) < 1e-12
    assert np.max(np.abs(v - g["v_rf"])) < 1e-9
    T = tr.monte_carlo_temperature(dc, n_particles=int(g["mc_n"]), t_max=float(g["mc_t_max"]),
                                   t_equilibrium=float(g["mc_t_eq"]))
    assert abs(T - float(g["T_mc"])) < 1e-9 * float(g["T_mc"])


def test_reference_objects_accepted(mol, gpu):
    """A simulator object with the reference's attributes (DC: _beams) runs on the GPU."""
    from molmot_b200 import force_scan as fs
    from molmot_b200.fields import make_dc_mot_beams
    g = golden("force_scan_api.npz")

    class RefLikeDC:
        pass

    s = RefLikeDC()
    s.mol_data = mol
    s._beams = make_dc_mot_beams(mol, delta_Gamma=-0.30, split_Gamma=0.40, s0=1.0)
    s.B_gradient = 0.16
    s.Gamma_eff_factor = 1.0
    assert rel_to_max(fs.force_vs_z(s, g["zs"])[0], g["F_dc_z"]) < 1e-10


def test_molmot_cuda_twin(mol, gpu):
    from molmot_b200 import cuda as mc
    g = golden("three_way_golden.npz")
    from molmot_b200.fields import LaserBeam
    beams = [LaserBeam(np.array([0, 0, g["kdir"][b]]), g["freq"][b], int(g["pol"][b]), g["s0"][b])
             for b in range(8)]
    B = float(g["B_gradient"])
    F, P, R = mc.force_vs_z_cuda(mol, beams, g["z_arr"], 0.0, B)
    assert rel_to_max(F / g["F_unit"], g["Fz_gpu"]) < 1e-10
    assert np.max(np.abs(P - g["Pz_gpu"])) < 1e-10
    Fv = mc.force_vs_v_cuda(mol, beams, g["v_arr"], 0.0, B)
    assert rel_to_max(Fv / g["F_unit"], g["Fv_gpu"]) < 1e-10
    k = mc.spring_constant_cuda(mol, beams, B)
    assert abs(k - float(g["k_gpu"])) < 1e-9 * abs(float(g["k_gpu"]))
    beta = mc.damping_coefficient_cuda(mol, beams, B) / mol.mass
    assert abs(beta - float(g["beta_gpu"])) < 1e-9 * abs(float(g["beta_gpu"]))
    Fm, Pm, Rm = mc.force_map_2d_cuda(mol, beams, g["v_arr"][:7], g["z_arr"][:9], B)
    assert Fm.shape == (7, 9) and Pm.shape == (7, 9, 12)
    info = mc.get_device_info()
    assert "compute_capability" in info
