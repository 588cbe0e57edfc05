#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the molmot reference.

Run in a container that has the reference checkout (default
/root/reference, or $MOLMOT_REFERENCE):

    python tests/golden/make_golden.py             # SrOH fixtures
    python tests/golden/make_golden.py analysis    # analysis_golden.npz
    python tests/golden/make_golden.py molecules   # molecules_golden.npz (CaF, CaOH)
    python tests/golden/make_golden.py force3d     # force3d_reference.npz (3D, synthetic molecules)

It (1) extracts the reference's own golden arrays from
validation/three_way_results.npz and validation/trajectory_cpu_vs_gpu_results.npz,
and (2) runs the reference's CPU functions on seeded inputs and saves their
outputs.  The fixtures are small .npz files; the GPU box, which has no
reference checkout, reads only these.  Library versions used are recorded
in each file under the key ``versions``.
"""
from __future__ import annotations

import os
import sys

import numpy as np

REF = os.environ.get("MOLMOT_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/molmot_numba_cache")
sys.path.insert(0, REF)


def versions():
    import numba
    import scipy
    return np.array(f"numpy {np.__version__}; scipy {scipy.__version__}; numba {numba.__version__}")


def beams_to_arrays(beams):
    return (np.array([b.kdir_z for b in beams]), np.array([b.freq_offset for b in beams]),
            np.array([b.polarization for b in beams], dtype=np.int32),
            np.array([b.s0 for b in beams]))


def hallas_beams(mol, ratios):
    """validation/sroh_redmot_three_way.py:67-103 with the given power ratios."""
    from molmot.constants import c, h
    from molmot.obe.fields import LaserBeam
    E = mol.energies
    n_g, n_e = mol.n_ground, mol.n_excited
    det = np.array([-10.3, -5.9, -9.2, -29.9]) * 1e6
    e_last = E[n_g + n_e - 1]
    freqs = [e_last - E[0] + det[0], e_last - E[0] + det[1],
             e_last - E[9] + det[2], e_last - E[9] + det[3]]
    Isat = np.pi * h * c * mol.Gamma / (3.0 * 687e-9 ** 3)
    r = np.array(ratios, dtype=float)
    r /= r.sum()
    sats = (100.0 * 1e-3 * r) * (2.0 / (np.pi * 10e-3 ** 2)) / Isat
    beams = []
    for f, q, s in zip(freqs, [2, 0, 2, 0], sats):
        for d in (+1, -1):
            qe = q if d > 0 else (2 - q if q != 1 else 1)
            beams.append(LaserBeam(direction=np.array([0.0, 0.0, float(d)]), freq_offset=f,
                                   polarization=qe, s0=s))
    return beams, np.array(freqs), sats


def main():
    from molmot.molecules.sroh import load_sroh_from_julia
    from molmot.obe.fields import make_dc_mot_beams, make_rf_mot_beams
    from molmot.obe.rate_equations import solve_rate_equations
    from molmot.obe.rate_equations_jit import solve_rate_equations_jit
    from molmot.mot.simulator import DCMOTSimulator, RFMOTSimulator
    from molmot.mot import force_scan as fs
    from molmot.propagation.trajectories_jit import simulate_trajectory_jit

    mol = load_sroh_from_julia(os.path.join(REF, "julia_sim"), verbose=False)
    ver = versions()

    # ---- (1) the reference's own golden arrays: config 1, Hallas ratios ----
    tw = np.load(os.path.join(REF, "validation", "three_way_results.npz"))
    beams, freqs, sats = hallas_beams(mol, [0.50, 0.08, 0.15, 0.27])
    kd, fr, po, s0 = beams_to_arrays(beams)
    keep = ["z_arr", "v_arr", "Fz_cpu_s", "Fv_cpu_s", "Pz_cpu_s", "k_cpu_s", "beta_cpu_s",
            "Fz_gpu", "Fv_gpu", "Pz_gpu", "k_gpu", "beta_gpu"]
    np.savez(os.path.join(HERE, "three_way_golden.npz"),
             **{k: tw[k] for k in keep}, kdir=kd, freq=fr, pol=po, s0=s0, B_gradient=0.214,
             F_unit=1.054571817e-34 * mol.k * mol.Gamma / 2.0, versions=ver,
             source=np.array("validation/three_way_results.npz + sroh_redmot_three_way.py:67-103"))

    # config 1 as BASELINE names it: equal 100 mW split
    beams_eq, freqs_eq, sats_eq = hallas_beams(mol, [0.25, 0.25, 0.25, 0.25])
    kd, fr, po, s0 = beams_to_arrays(beams_eq)
    z = np.linspace(-5e-3, 5e-3, 101)
    Fz_jit = np.array([solve_rate_equations_jit(mol, beams_eq, 0.0, zi, 0.214)[0] for zi in z])
    Pz_jit = np.array([solve_rate_equations_jit(mol, beams_eq, 0.0, zi, 0.214)[1] for zi in z])
    Fz_py = np.array([solve_rate_equations(mol, beams_eq, 0.0, zi, 0.214)[0] for zi in z])
    sim_like = type("S", (), {})()
    sim_like.force = lambda v, zz: solve_rate_equations_jit(mol, beams_eq, v, zz, 0.214)
    k_jit = fs.spring_constant(sim_like)
    a_jit = fs.damping_coefficient(sim_like)
    np.savez(os.path.join(HERE, "config1_equal_split.npz"), z=z, Fz_jit=Fz_jit, Pz_jit=Pz_jit,
             Fz_py=Fz_py, k_jit=k_jit, alpha_jit=a_jit, kdir=kd, freq=fr, pol=po, s0=s0,
             B_gradient=0.214, sats=sats_eq, versions=ver)

    # ---- (2) seeded random points through the JIT core and the Python path ----
    rng = np.random.default_rng(20261203)
    n_sets, n_pts = 24, 16
    rows = {k: [] for k in ["kdir", "freq", "pol", "s0", "B", "v", "z", "F_jit", "p_jit", "R_jit",
                            "F_py", "p_py", "R_py"]}
    for s in range(n_sets):
        b = make_dc_mot_beams(mol, delta_Gamma=rng.uniform(-3, 0), split_Gamma=rng.uniform(0, 2),
                              s0=10 ** rng.uniform(-1, 1))
        kd, fr, po, s0 = beams_to_arrays(b)
        # per-frequency random detuning/s0 as in the batched-map workload
        fr = fr + np.repeat(rng.uniform(-40e6, 0, 4), 2)
        s0 = np.repeat(10 ** rng.uniform(-1, 1, 4), 2)
        from molmot.obe.fields import LaserBeam
        b = [LaserBeam(np.array([0.0, 0.0, kd[i]]), fr[i], int(po[i]), s0[i]) for i in range(8)]
        B = rng.uniform(0.05, 0.4)
        for _ in range(n_pts):
            v, zz = rng.uniform(-10, 10), rng.uniform(-1e-2, 1e-2)
            Fj, pj, Rj = solve_rate_equations_jit(mol, b, v, zz, B)
            Fp, pp, Rp = solve_rate_equations(mol, b, v, zz, B)
            for k, val in zip(rows, [kd, fr, po, s0, B, v, zz, Fj, pj, Rj, Fp, pp, Rp]):
                rows[k].append(val)
    out = {k: np.array(v) for k, v in rows.items()}
    np.savez(os.path.join(HERE, "random_points.npz"), n_sets=n_sets, n_pts=n_pts, versions=ver, **out)

    # ---- RF MOT, force_scan API values (DC and RF simulators) ----
    dc = DCMOTSimulator(mol, delta_Gamma=-0.30, split_Gamma=0.40, s0=1.0, B_gradient=0.16)
    rf = RFMOTSimulator(mol, delta_Gamma=-1.0, s0=1.0, B_gradient=0.16)
    zs = np.linspace(-3e-3, 3e-3, 7)
    vs = np.linspace(-5, 5, 7)
    F_dc, P_dc, R_dc = fs.force_vs_z(dc, zs)
    F_rf, P_rf, R_rf = fs.force_vs_z(rf, zs)
    np.savez(os.path.join(HERE, "force_scan_api.npz"), zs=zs, vs=vs,
             F_dc_z=F_dc, P_dc_z=P_dc, R_dc_z=R_dc, F_dc_v=fs.force_vs_v(dc, vs),
             F_rf_z=F_rf, P_rf_z=P_rf, R_rf_z=R_rf, F_rf_v=fs.force_vs_v(rf, vs),
             k_dc=fs.spring_constant(dc), a_dc=fs.damping_coefficient(dc),
             k_rf=fs.spring_constant(rf), a_rf=fs.damping_coefficient(rf),
             vcap_dc=fs.capture_velocity(dc, v_max=6.0, dv=0.5, n_steps=3000),
             versions=ver)
    opt = fs.optimize_parameters(mol, {"delta": np.array([-1.0, -0.5, -0.2]),
                                       "split": np.array([0.2, 0.7])}, 0.16, verbose=False)
    np.savez(os.path.join(HERE, "optimize_parameters.npz"), delta=opt["delta_scan"],
             split=opt["split_scan"], K_map=opt["K_map"], beta_map=opt["beta_map"],
             delta_best=opt["delta_best"], split_best=opt["split_best"], versions=ver)

    # ---- 1D trajectories: the reference's golden endpoints + short JIT runs ----
    tj = np.load(os.path.join(REF, "validation", "trajectory_cpu_vs_gpu_results.npz"))
    keep = ["ref_z0", "ref_v0", "ref_zf_py", "ref_vf_py", "ref_zf_jit", "ref_vf_jit",
            "ref_zf_gpu", "ref_vf_gpu", "batch_z0", "batch_v0", "batch_zf_jit", "batch_vf_jit",
            "batch_zf_gpu", "batch_vf_gpu", "batch_n_actual", "t_max", "dt"]
    sim = DCMOTSimulator(mol, delta_Gamma=-0.20, split_Gamma=0.70, s0=1.0, B_gradient=0.16)
    kd, fr, po, s0 = beams_to_arrays(sim._beams)
    short = []
    for z0, v0 in [(3e-3, 0.0), (0.0, -2.0), (2e-3, -1.0), (0.0, -5.0)]:
        _, za, va = simulate_trajectory_jit(sim, z0, v0, t_max=2e-3, dt=1e-6)
        short.append((za, va))
    np.savez(os.path.join(HERE, "trajectory_golden.npz"), **{k: tj[k] for k in keep},
             kdir=kd, freq=fr, pol=po, s0=s0, B_gradient=0.16,
             short_z=np.array([s[0] for s in short]), short_v=np.array([s[1] for s in short]),
             short_t_max=2e-3, versions=ver,
             source=np.array("validation/trajectory_cpu_vs_gpu_results.npz; short runs: "
                             "molmot/propagation/trajectories_jit.py simulate_trajectory_jit"))
    # ---- per-axis 3D trajectories, RF trajectory, Monte-Carlo temperature ----
    from molmot.propagation.trajectories import (simulate_trajectories_3d, simulate_trajectory,
                                                 monte_carlo_temperature)
    dc2 = DCMOTSimulator(mol, delta_Gamma=-0.20, split_Gamma=0.70, s0=1.0, B_gradient=0.16)
    r0s = [np.array([1e-3, -0.5e-3, 2e-3]), np.array([0.0, 2e-3, -1e-3])]
    v0s = [np.array([0.5, -0.3, 1.0]), np.array([-1.0, 0.2, 0.0])]
    tr3 = simulate_trajectories_3d(dc2, r0s, v0s, t_max=6e-4, dt=1e-6)
    rf2 = RFMOTSimulator(mol, delta_Gamma=-1.0, s0=1.0, B_gradient=0.16)
    _, zrf, vrf = simulate_trajectory(rf2, 2e-3, -1.0, t_max=8e-4, dt=1e-6)
    T_mc = monte_carlo_temperature(dc2, n_particles=6, t_max=1.5e-3, dt=1e-6,
                                   t_equilibrium=0.5e-3)
    np.savez(os.path.join(HERE, "trajectory_api_golden.npz"),
             r0=np.array(r0s), v0=np.array(v0s), r3=np.array([t[1] for t in tr3]),
             v3=np.array([t[2] for t in tr3]), t_max3=6e-4, z_rf=zrf, v_rf=vrf, t_max_rf=8e-4,
             T_mc=T_mc, mc_n=6, mc_t_max=1.5e-3, mc_t_eq=0.5e-3, versions=ver)
    # ---- 3D rate-equation force (molmot/mot/simulator_3d.py:168-365) ----
    from molmot.mot.simulator_3d import MOTSimulator3D, rate_eq_force_3d
    from molmot.obe.obe_subdoppler import make_beam_pairs_dc4
    rng3 = np.random.default_rng(3)
    cases = []
    for d, sp, s0_, Bg in [(-0.30, 0.40, 1.0, 0.16), (-1.0, 0.7, 3.0, 0.214), (-0.5, 1.2, 0.5, 0.3)]:
        sim3 = MOTSimulator3D(mol, make_beam_pairs_dc4(mol, d, sp, s0_), B_gradient=Bg)
        kh = np.array([b.k_hat for b in sim3.beams])
        fq = np.array([b.freq for b in sim3.beams])
        ql = np.array([b.q_lab for b in sim3.beams], dtype=np.int32)
        sb = np.array([b.s0 for b in sim3.beams])
        rad = np.array([b.beam_radius for b in sim3.beams])
        r = np.concatenate([np.zeros((1, 3)), rng3.normal(0, 2e-3, (14, 3)),
                            np.array([[0, 0, 1e-3], [1e-3, 0, 0], [0, 0, -2e-3]])])
        v = np.concatenate([np.zeros((1, 3)), rng3.normal(0, 1.0, (14, 3)), np.zeros((3, 3))])
        F = np.zeros((len(r), 3)); R = np.zeros(len(r)); P = np.zeros((len(r), 12))
        for i in range(len(r)):
            F[i], R[i], P[i] = rate_eq_force_3d(mol, sim3.beams, r[i], v[i], Bg)
        cases.append(dict(khat=kh, freq=fq, q=ql, s0=sb, radius=rad, B=Bg, r=r, v=v, F=F, R=R, P=P))
    np.savez(os.path.join(HERE, "force3d_golden.npz"), versions=ver, n_cases=len(cases),
             **{f"c{i}_{k}": val for i, c in enumerate(cases) for k, val in c.items()})
    # short leapfrog trajectories (MOTSimulator3D.simulate_trajectory_3d, :443-504)
    sim3 = MOTSimulator3D(mol, make_beam_pairs_dc4(mol, -0.30, 0.40, 1.0), B_gradient=0.16)
    r0s = np.array([[1e-3, -1e-3, 0.5e-3], [0.0, 0.5e-3, -2e-3]])
    v0s = np.array([[0.3, 0.2, -0.5], [-0.4, 0.0, 0.6]])
    trs = [sim3.simulate_trajectory_3d(r0s[i], v0s[i], t_max=1.2e-4, dt=1e-6) for i in range(2)]
    np.savez(os.path.join(HERE, "traj3d_golden.npz"), r0=r0s, v0=v0s, t_max=1.2e-4, dt=1e-6,
             r=np.array([t[1] for t in trs]), v=np.array([t[2] for t in trs]), versions=ver)
    print("golden fixtures written to", HERE)


def analysis_golden():
    """molmot/mot/analysis.py on seeded synthetic ensembles (oracle/analysis.py
    synthetic_ensemble), in the reference's list-of-tuples form."""
    from molmot.mot import analysis as an
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.analysis import synthetic_ensemble
    out = {"versions": versions()}
    mass = 104.0 * 1.66053906660e-27
    for k, (seed, n, S) in enumerate([(7, 150, 600), (11, 60, 300)]):
        t, Z, V = synthetic_ensemble(seed, n, S)
        res = [(t, Z[i], V[i]) for i in range(n)]
        c, sz, sv, na = an.sigma_vs_time(res, time_bins=40)
        _, T = an.temperature_vs_time(res, mass, time_bins=40)
        _, n0 = an.density_vs_time(res, N_total=2000, time_bins=40)
        out.update({f"e{k}_seed": seed, f"e{k}_n": n, f"e{k}_steps": S, f"e{k}_t": c, f"e{k}_sz": sz,
                    f"e{k}_sv": sv, f"e{k}_na": na, f"e{k}_T": T, f"e{k}_n0": n0,
                    f"e{k}_capture": an.capture_fraction(res, r_max=3e-3, t_min=1e-3),
                    f"e{k}_capture_t0": an.capture_fraction(res, r_max=5e-3, t_min=0.0),
                    f"e{k}_survived": np.array([an.survived(r) for r in res]),
                    f"e{k}_gfit": an.gaussian_fit(Z[:, S // 2]),
                    f"e{k}_gfit_final": an.gaussian_fit(Z[:, -1], bins=80, range_mm=(-5, 5)),
                    f"e{k}_mbfit": an.maxwell_boltzmann_fit_1d(V[:, -1], mass)})
    out["mass"] = mass
    np.savez(os.path.join(HERE, "analysis_golden.npz"), **out)
    print("analysis golden written")


def molecules_golden():
    """CaF and CaOH (molmot/molecules/caf.py:90, caoh.py:89, built by the
    reference's own Hamiltonian code): the MolecularData arrays, the derived
    fields, the reference's DC MOT beams, and _rate_eq_core forces at seeded
    random points (the 1D path; their ground Zeeman spectra are 6 + 6
    degenerate like SrOH's, so the 3D model is ill-posed for them too)."""
    from molmot.molecules.caf import build_caf_hamiltonian
    from molmot.molecules.caoh import build_caoh_hamiltonian
    from molmot.obe.fields import LaserBeam, make_dc_mot_beams
    from molmot.obe.rate_equations_jit import solve_rate_equations_jit
    out = {"versions": versions()}
    rng = np.random.default_rng(20261204)
    for name, build in (("caf", build_caf_hamiltonian), ("caoh", build_caoh_hamiltonian)):
        m = build(verbose=False)
        for key in ("energies", "tdm", "zeeman_x", "zeeman_y", "zeeman_z", "d_squared", "zeeman_z_diag"):
            out[f"{name}_{key}"] = np.asarray(getattr(m, key))
        for key in ("Gamma", "k", "mass", "wavelength", "n_ground", "n_excited", "omega_J12",
                    "omega_J32", "omega_mean"):
            out[f"{name}_{key}"] = np.asarray(getattr(m, key))
        kd, fr, po, s0 = beams_to_arrays(make_dc_mot_beams(m, delta_Gamma=-0.25, split_Gamma=0.6, s0=1.5))
        out.update({f"{name}_dc_kdir": kd, f"{name}_dc_freq": fr, f"{name}_dc_pol": po, f"{name}_dc_s0": s0})
        n_sets, n_pts = 8, 16
        rows = {k: [] for k in ["kdir", "freq", "pol", "s0", "B", "v", "z", "F", "p", "R"]}
        for _ in range(n_sets):
            b = make_dc_mot_beams(m, delta_Gamma=rng.uniform(-3, 0), split_Gamma=rng.uniform(0, 2),
                                  s0=10 ** rng.uniform(-1, 1))
            kd, fr, po, s0 = beams_to_arrays(b)
            fr = fr + np.repeat(rng.uniform(-40e6, 0, 4), 2)
            s0 = np.repeat(10 ** rng.uniform(-1, 1, 4), 2)
            b = [LaserBeam(np.array([0.0, 0.0, kd[i]]), fr[i], int(po[i]), s0[i]) for i in range(8)]
            B = rng.uniform(0.05, 0.4)
            for _ in range(n_pts):
                v, zz = rng.uniform(-10, 10), rng.uniform(-1e-2, 1e-2)
                F, p, R = solve_rate_equations_jit(m, b, v, zz, B)
                for k, val in zip(rows, [kd, fr, po, s0, B, v, zz, F, p, R]):
                    rows[k].append(val)
        out.update({f"{name}_pts_{k}": np.array(v) for k, v in rows.items()})
        out[f"{name}_n_sets"], out[f"{name}_n_pts"] = n_sets, n_pts
    np.savez(os.path.join(HERE, "molecules_golden.npz"), **out)
    print("molecules golden written")


def force3d_reference_golden():
    """The reference's 3D model (molmot/mot/simulator_3d.py:168-365
    rate_eq_force_3d, :443-504 MOTSimulator3D.simulate_trajectory_3d) run on
    synthetic molecules (12 + 4, 8 + 3 and 16 + 8 levels) whose ground Zeeman
    Hamiltonian has a non-degenerate spectrum (molmot_b200.molecules.synthetic;
    the eigenbasis, and so the force, is a well-posed function of the
    inputs): 72 (r, v) points and 3 leapfrog trajectories of 200 steps per
    molecule.  Also the reference's
    own spread on the SrOH cases of force3d_golden.npz: the largest change of
    its force under 1e-15 relative Hermitian perturbations of the Zeeman
    Hamiltonian passed to numpy.linalg.eigh (6 draws per case), relative to
    max |F| of the case.  Writes force3d_reference.npz."""
    import importlib
    from molmot.mot.simulator_3d import MOTSimulator3D, rate_eq_force_3d
    from molmot.obe.obe_subdoppler import make_beam_pairs_dc4
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from molmot_b200.molecules.synthetic import synthetic_molecule
    out = {"versions": versions()}
    mols = [(12, 4, 5, -0.5, 0.5, 1.0, 0.2), (8, 3, 21, -0.8, 0.3, 2.0, 0.25),
            (16, 8, 41, -0.6, 0.4, 1.5, 0.22)]
    out["n_mol"] = len(mols)
    for i, (ng, ne, seed, d, sp, s0_, Bg) in enumerate(mols):
        m = synthetic_molecule(ng, ne, seed)
        sim = MOTSimulator3D(m, make_beam_pairs_dc4(m, d, sp, s0_), B_gradient=Bg)
        rng = np.random.default_rng(100 + i)
        r = np.concatenate([rng.normal(0, 3e-3, (64, 3)), np.zeros((1, 3)),
                            [[0, 0, 2e-3], [1e-3, 0, 0], [0, -1e-3, 0], [0, 0, -4e-3],
                             [2e-3, 2e-3, 1e-3], [-1e-3, 0.5e-3, 3e-3], [5e-3, -4e-3, 2e-3]]])
        v = np.concatenate([rng.normal(0, 2.0, (64, 3)), np.zeros((8, 3))])
        F = np.zeros((len(r), 3)); R = np.zeros(len(r)); P = np.zeros((len(r), ng))
        for j in range(len(r)):
            F[j], R[j], P[j] = rate_eq_force_3d(m, sim.beams, r[j], v[j], Bg)
        r0 = np.array([[1e-3, -1e-3, 0.5e-3], [0.0, 0.5e-3, -2e-3], [2e-3, 1e-3, 0.0]])
        v0 = np.array([[0.3, 0.2, -0.5], [-0.4, 0.0, 0.6], [0.0, 0.1, 0.1]])
        trs = [sim.simulate_trajectory_3d(r0[j], v0[j], t_max=2e-4, dt=1e-6) for j in range(3)]
        out.update({f"m{i}_ng": ng, f"m{i}_ne": ne, f"m{i}_seed": seed, f"m{i}_B": Bg,
                    f"m{i}_pairs": np.array([d, sp, s0_]),
                    f"m{i}_khat": np.array([b.k_hat for b in sim.beams]),
                    f"m{i}_freq": np.array([b.freq for b in sim.beams]),
                    f"m{i}_q": np.array([b.q_lab for b in sim.beams], dtype=np.int32),
                    f"m{i}_s0": np.array([b.s0 for b in sim.beams]),
                    f"m{i}_radius": np.array([b.beam_radius for b in sim.beams]),
                    f"m{i}_r": r, f"m{i}_v": v, f"m{i}_F": F, f"m{i}_R": R, f"m{i}_P": P,
                    f"m{i}_r0": r0, f"m{i}_v0": v0, f"m{i}_t_max": 2e-4, f"m{i}_dt": 1e-6,
                    f"m{i}_traj_r": np.array([t[1] for t in trs]),
                    f"m{i}_traj_v": np.array([t[2] for t in trs])})
    # the reference's own spread on the SrOH cases
    from molmot.molecules.sroh import load_sroh_from_julia
    from molmot.mot.simulator_3d import Beam3D
    mol = load_sroh_from_julia(os.path.join(REF, "julia_sim"), verbose=False)
    g = np.load(os.path.join(HERE, "force3d_golden.npz"))
    orig = np.linalg.eigh
    prng = np.random.default_rng(0)

    def perturbed(H):
        E = prng.normal(size=H.shape) + 1j * prng.normal(size=H.shape)
        return orig(H + 1e-15 * np.abs(H).max() * (E + E.conj().T) / 2)

    spreads = []
    for c in range(int(g["n_cases"])):
        K = lambda k: g[f"c{c}_{k}"]
        beams = [Beam3D(k_hat=K("khat")[b], freq=K("freq")[b], q_lab=int(K("q")[b]), s0=K("s0")[b],
                        beam_radius=K("radius")[b]) for b in range(len(K("freq")))]
        scale = np.abs(K("F")).max()
        spread = 0.0
        np.linalg.eigh = perturbed
        try:
            for _ in range(6):
                Fp = np.array([rate_eq_force_3d(mol, beams, K("r")[j], K("v")[j], float(K("B")))[0]
                               for j in range(len(K("r")))])
                spread = max(spread, float(np.abs(Fp - K("F")).max() / scale))
        finally:
            np.linalg.eigh = orig
        spreads.append(spread)
    out["sroh_spread"] = np.array(spreads)
    np.savez(os.path.join(HERE, "force3d_reference.npz"), **out)
    print("force3d_reference.npz written; SrOH spreads", spreads)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "analysis":
        analysis_golden()
    elif len(sys.argv) > 1 and sys.argv[1] == "force3d":
        force3d_reference_golden()
    elif len(sys.argv) > 1 and sys.argv[1] == "molecules":
        molecules_golden()
    else:
        main()
        analysis_golden()
