"""The CPU oracle against the reference's golden vectors (no GPU needed).

Pins oracle/rate_eq_oracle.c to:
  * validation/three_way_results.npz (config 1, Hallas ratios): the reference
    GPU arrays (JIT hbar) and its pure-Python arrays (CODATA hbar);
  * seeded random points run through the reference's numba core and its
    Python solver (tests/golden/random_points.npz);
  * the reference's 1D trajectory endpoints and short JIT trajectories.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import rate_eq as orc


def rel_to_max(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(a)), np.max(np.abs(b)), 1e-300)


def test_three_way_jit_golden_bitlevel(mol):
    g = golden("three_way_golden.npz")
    beams = (g["kdir"], g["freq"], g["pol"].astype(float), g["s0"])
    Fz = np.array([orc.point(mol, beams, 0.0, z, float(g["B_gradient"]))[0] for z in g["z_arr"]])
    Pz = np.array([orc.point(mol, beams, 0.0, z, float(g["B_gradient"]))[1] for z in g["z_arr"]])
    Fv = np.array([orc.point(mol, beams, v, 0.0, float(g["B_gradient"]))[0] for v in g["v_arr"]])
    # the reference GPU kernel runs the JIT algorithm (same hbar, two-pass order)
    assert rel_to_max(Fz / g["F_unit"], g["Fz_gpu"]) < 1e-14
    assert rel_to_max(Fv / g["F_unit"], g["Fv_gpu"]) < 1e-14
    assert np.max(np.abs(Pz - g["Pz_gpu"])) < 1e-14


def test_three_way_python_golden(mol):
    g = golden("three_way_golden.npz")
    beams = (g["kdir"], g["freq"], g["pol"].astype(float), g["s0"])
    fl = orc.TWO_PASS | orc.UNIFORM_FALLBACK
    B = float(g["B_gradient"])
    Fz = np.array([orc.point(mol, beams, 0.0, z, B, hbar=orc.HBAR_CODATA, flags=fl)[0]
                   for z in g["z_arr"]])
    Fv = np.array([orc.point(mol, beams, v, 0.0, B, hbar=orc.HBAR_CODATA, flags=fl)[0]
                   for v in g["v_arr"]])
    assert rel_to_max(Fz / g["F_unit"], g["Fz_cpu_s"]) < 1e-13
    assert rel_to_max(Fv / g["F_unit"], g["Fv_cpu_s"]) < 1e-13
    # spring constant and damping (molmot/mot/force_scan.py:84-127)
    dz, dv = 0.3e-3, 0.1
    Fp = orc.point(mol, beams, 0.0, dz, B, hbar=orc.HBAR_CODATA, flags=fl)[0]
    Fm = orc.point(mol, beams, 0.0, -dz, B, hbar=orc.HBAR_CODATA, flags=fl)[0]
    k = -(Fp - Fm) / (2 * dz)
    assert abs(k - g["k_cpu_s"]) < 1e-12 * abs(g["k_cpu_s"])
    Fvp = orc.point(mol, beams, dv, 0.0, B, hbar=orc.HBAR_CODATA, flags=fl)[0]
    Fvm = orc.point(mol, beams, -dv, 0.0, B, hbar=orc.HBAR_CODATA, flags=fl)[0]
    beta = -(Fvp - Fvm) / (2 * dv * mol.mass)
    assert abs(beta - g["beta_cpu_s"]) < 1e-10 * abs(g["beta_cpu_s"])
    # the two hbar values explain the reference's documented 1.6e-8 CPU/GPU gap
    assert 1e-9 < rel_to_max(g["Fz_cpu_s"], g["Fz_gpu"]) < 1e-7


def test_random_points_jit_bitwise(mol):
    g = golden("random_points.npz")
    n = g["F_jit"].size
    for i in range(n):
        beams = (g["kdir"][i], g["freq"][i], g["pol"][i].astype(float), g["s0"][i])
        F, p, R, st = orc.point(mol, beams, g["v"][i], g["z"][i], g["B"][i])
        assert F == g["F_jit"][i]
        assert R == g["R_jit"][i]
        assert np.array_equal(p, g["p_jit"][i])


def test_random_points_python_path(mol):
    g = golden("random_points.npz")
    fl = orc.TWO_PASS | orc.UNIFORM_FALLBACK
    worst = 0.0
    for i in range(g["F_py"].size):
        beams = (g["kdir"][i], g["freq"][i], g["pol"][i].astype(float), g["s0"][i])
        F = orc.point(mol, beams, g["v"][i], g["z"][i], g["B"][i], hbar=orc.HBAR_CODATA, flags=fl)[0]
        worst = max(worst, abs(F - g["F_py"][i]) / max(abs(g["F_py"][i]), 1e-300))
    assert worst < 1e-12


def test_batch_matches_point(mol):
    g = golden("random_points.npz")
    ns, npts = int(g["n_sets"]), int(g["n_pts"])
    kd = g["kdir"].reshape(ns, npts, -1)[:, 0]
    fr = g["freq"].reshape(ns, npts, -1)[:, 0]
    po = g["pol"].reshape(ns, npts, -1)[:, 0]
    s0 = g["s0"].reshape(ns, npts, -1)[:, 0]
    B = g["B"].reshape(ns, npts)[:, 0]
    F, pop, R, st = orc.force_batch(mol, kd, fr, po, s0, B, g["v"], g["z"], points_per_set=npts,
                                    n_threads=4)
    assert np.array_equal(F, g["F_jit"])
    assert np.array_equal(pop, g["p_jit"])


def test_grid_layout(mol):
    g = golden("config1_equal_split.npz")
    F, pop, R, st = orc.force_batch(mol, g["kdir"], g["freq"], g["pol"], g["s0"],
                                    float(g["B_gradient"]), np.array([0.0]), g["z"], grid=True)
    assert np.array_equal(F, g["Fz_jit"])
    assert np.array_equal(pop, g["Pz_jit"])


def test_traj1d_short_bitwise(mol):
    g = golden("trajectory_golden.npz")
    beams = (g["kdir"], g["freq"], g["pol"].astype(float), g["s0"])
    n_steps = g["short_z"].shape[1]
    z0 = g["short_z"][:, 0]
    v0 = g["short_v"][:, 0]
    zf, vf, na, zt, vt = orc.traj1d(mol, beams, float(g["B_gradient"]), z0, v0, 1e-6, n_steps,
                                    save_full=True)
    assert np.array_equal(zt, g["short_z"])
    assert np.array_equal(vt, g["short_v"])


@pytest.mark.slow
def test_traj1d_reference_endpoints(mol):
    g = golden("trajectory_golden.npz")
    beams = (g["kdir"], g["freq"], g["pol"].astype(float), g["s0"])
    n_steps = int(float(g["t_max"]) / float(g["dt"]))
    zf, vf, na, _, _ = orc.traj1d(mol, beams, float(g["B_gradient"]), g["ref_z0"], g["ref_v0"],
                                  float(g["dt"]), n_steps)
    assert np.array_equal(zf, g["ref_zf_jit"])
    assert np.array_equal(vf, g["ref_vf_jit"])
    zf, vf, na, _, _ = orc.traj1d(mol, beams, float(g["B_gradient"]), g["batch_z0"],
                                  g["batch_v0"], float(g["dt"]), n_steps)
    assert np.array_equal(zf, g["batch_zf_jit"])
    assert np.array_equal(vf, g["batch_vf_jit"])
    assert np.array_equal(na, g["batch_n_actual"])
