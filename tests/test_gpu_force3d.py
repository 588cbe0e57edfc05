"""GPU 3D force and leapfrog ensembles against the reference's own outputs
and the numpy oracle (a restatement of molmot/mot/simulator_3d.py with numpy
eigh, itself pinned to the reference in test_force3d_oracle.py).

Two regimes:
* Synthetic molecules whose ground Zeeman Hamiltonian B.Z has a
  non-degenerate spectrum: the eigenbasis is unique, the 3D force is a
  well-posed function of the inputs, and the GPU must match the reference's
  rate_eq_force_3d and simulate_trajectory_3d outputs
  (force3d_reference.npz) to 1e-10 of max|F|; recoil kicks (this build's
  model, absent from the reference) are checked against the oracle.
* SrOH: its ground Zeeman block is pure electron-spin Zeeman, so B.Z has
  two exactly 6-fold degenerate eigenvalues and the reference pairs
  hyperfine energies with whatever basis LAPACK returns inside those
  subspaces.  A 1e-15 relative perturbation of H moves the reference's own
  force by percents of max|F| (its spread, computed by running the
  reference and stored in force3d_reference.npz); no independent eigensolver
  can reproduce it more closely.  The GPU's deviation from the reference's
  golden forces must stay within that recorded spread.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
TOL3D = 1e-10


def _case(g, c):
    return lambda k: g[f"c{c}_{k}"]


@pytest.fixture(scope="module")
def synth(gpu):
    from molmot_b200.molecules.synthetic import synthetic_molecule
    from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
    m = synthetic_molecule(12, 4, 5)
    sim = MOTSimulator3D(m, make_beam_pairs_dc4(m, -0.5, 0.5, 1.0), B_gradient=0.2)
    beams3 = (np.array([b.k_hat for b in sim.beams]), np.array([b.freq for b in sim.beams]),
              np.array([b.q_lab for b in sim.beams]), np.array([b.s0 for b in sim.beams]),
              np.array([b.beam_radius for b in sim.beams]))
    return m, sim, beams3


@pytest.mark.parametrize("i", [0, 1, 2])
def test_force3d_synthetic_vs_reference(gpu, i):
    from molmot_b200.engine import beam_sets_3d, force3d_batch, pack_for
    from molmot_b200.molecules.synthetic import synthetic_molecule
    g = golden("force3d_reference.npz")
    K = lambda k: g[f"m{i}_{k}"]
    m = synthetic_molecule(int(K("ng")), int(K("ne")), int(K("seed")))
    bs = beam_sets_3d(K("khat"), K("freq"), K("q"), K("s0"), K("radius"), float(K("B")))
    o = force3d_batch(pack_for(m), bs, K("r"), K("v"))
    F, R, P = (o[k].cpu().numpy() for k in ("F", "R", "pop"))
    assert np.abs(F - K("F")).max() <= TOL3D * np.abs(K("F")).max()
    assert np.abs(R - K("R")).max() <= TOL3D * np.abs(K("R")).max()
    assert np.abs(P - K("P")).max() <= TOL3D


@pytest.mark.parametrize("i", [0, 1, 2])
def test_leapfrog_synthetic_vs_reference(gpu, i):
    from molmot_b200.molecules.synthetic import synthetic_molecule
    from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
    g = golden("force3d_reference.npz")
    K = lambda k: g[f"m{i}_{k}"]
    m = synthetic_molecule(int(K("ng")), int(K("ne")), int(K("seed")))
    d, sp, s0 = K("pairs")
    sim = MOTSimulator3D(m, make_beam_pairs_dc4(m, d, sp, s0), B_gradient=float(K("B")))
    assert np.array_equal(np.array([b.freq for b in sim.beams]), K("freq"))
    t, R, V = sim.simulate_ensemble_arrays(K("r0"), K("v0"), float(K("t_max")), float(K("dt")))
    Rg, Vg = K("traj_r"), K("traj_v")
    assert R.shape == Rg.shape
    assert np.abs(R - Rg).max() <= TOL3D * np.abs(Rg).max()
    assert np.abs(V - Vg).max() <= TOL3D * np.abs(Vg).max()


def test_leapfrog_kicks_synthetic_vs_oracle(synth):
    from oracle import force3d as o3
    m, sim, beams3 = synth
    r0 = np.array([[1e-3, -1e-3, 0.5e-3], [0.0, 0.5e-3, -2e-3], [2e-3, 1e-3, 0.0]])
    v0 = np.array([[0.3, 0.2, -0.5], [-0.4, 0.0, 0.6], [0.0, 0.1, 0.1]])
    n = 80
    for kicks in (False, True):
        t, R, V = sim.simulate_ensemble_arrays(r0, v0, n * 1e-6, 1e-6, kicks=kicks, seed=1234)
        for i in range(3):
            _, Ro, Vo = o3.leapfrog3d(m, beams3, 0.2, r0[i], v0[i], n * 1e-6, kicks=kicks,
                                      seed=1234, particle=i)
            assert np.abs(R[i] - Ro).max() < 1e-13, (kicks, i)
            assert np.abs(V[i] - Vo).max() < 1e-9, (kicks, i)


def test_checkpoint_resume_bitwise(synth):
    m, sim, _ = synth
    r0 = np.array([[1e-3, -1e-3, 0.5e-3], [0.0, 0.5e-3, -2e-3]])
    v0 = np.array([[0.3, 0.2, -0.5], [-0.4, 0.0, 0.6]])
    full = sim.run_ensemble(r0, v0, 60e-6, kicks=True, seed=99)
    a = sim.run_ensemble(r0, v0, 25e-6, kicks=True, seed=99)
    b = sim.run_ensemble(a["r"], a["vh"], 60 - 25, kicks=True, seed=99, step0=25)
    assert np.array_equal(full["r"].cpu().numpy(), b["r"].cpu().numpy())
    assert np.array_equal(full["vh"].cpu().numpy(), b["vh"].cpu().numpy())
    assert int(full["n_events"].sum()) == int(a["n_events"].sum() + b["n_events"].sum())


def test_kick_statistics(synth):
    """Zero-mean isotropic kicks, Poisson event counts with mean R dt:
    one step, kicked minus unkicked velocities of identical particles."""
    m, sim, _ = synth
    N = 8192
    r0 = np.tile([[1e-3, -0.5e-3, 0.8e-3]], (N, 1))
    v0 = np.zeros((N, 3))
    on = sim.run_ensemble(r0, v0, 2e-6, kicks=True, seed=7)
    off = sim.run_ensemble(r0, v0, 2e-6, kicks=False)
    dv = (on["vh"] - off["vh"]).cpu().numpy()
    nev = on["n_events"].cpu().numpy()
    v_rec = 1.054571817e-34 * m.k / m.mass
    # the kicked step evaluates the force at r_1 = r_0 + dt v_1/2 with v_1/2 = v_0 + dt F_0 / 2m
    F0, _, _ = sim.force_3d(r0[0], v0[0])
    vh0 = v0[0] + 0.5 * 1e-6 * F0 / m.mass
    _, R1, _ = sim.force_3d(off["r"][0].cpu().numpy(), vh0)
    lam = R1 * 1e-6
    assert abs(nev.mean() / lam - 1) < 4 * np.sqrt(lam / N) / lam + 0.02
    assert abs((dv ** 2).sum(1).mean() / (2 * nev.mean() * v_rec ** 2) - 1) < 0.05
    assert np.abs(dv.mean(0)).max() < 5 * v_rec * np.sqrt(2 * nev.mean() / 3 / N)


def test_sroh_force3d_within_reference_spread(mol, gpu):
    from molmot_b200.engine import pack_for, beam_sets_3d, force3d_batch
    g = golden("force3d_golden.npz")
    spread = golden("force3d_reference.npz")["sroh_spread"]
    for c in range(int(g["n_cases"])):
        K = _case(g, c)
        bs = beam_sets_3d(K("khat"), K("freq"), K("q"), K("s0"), K("radius"), float(K("B")))
        F = force3d_batch(pack_for(mol), bs, K("r"), K("v"))["F"].cpu().numpy()
        scale = np.abs(K("F")).max()
        dev = np.abs(F - K("F")).max() / scale
        assert dev <= spread[c], (c, dev, spread[c])
        # the point at the origin (B = 0) is well posed: bare basis
        assert abs(F[0] - K("F")[0]).max() < 1e-10 * scale


def test_simulator3d_api(mol, gpu):
    """The reference's own 3D checks (tests/test_all_functions.py:522-559)."""
    from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4, compute_3d_force_map
    sim = MOTSimulator3D(mol, make_beam_pairs_dc4(mol, -0.30, 0.40, 1.0), B_gradient=0.16)
    assert len(sim.beams) == 24
    F, R, p = sim.force_3d(np.zeros(3), np.zeros(3))
    assert F.shape == (3,) and np.linalg.norm(F) < 1e-20
    F, _, _ = sim.force_3d(np.array([0.0, 0.0, 1e-3]), np.zeros(3))
    assert F[2] < 0
    c1, c2, Fx, Fz, Rm = compute_3d_force_map(sim, "xz", n_points=9)
    assert Fx.shape == (9, 9) and np.all(Rm > 0)


def test_sroh_leapfrog_close_to_reference(mol, gpu):
    """SrOH leapfrog vs the reference's trajectories: the per-step forces agree
    to the reference's own ~1e-3 ill-posedness, which over 120 steps of 1 us
    moves positions by ~1e-9 m at most."""
    from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
    t = golden("traj3d_golden.npz")
    sim = MOTSimulator3D(mol, make_beam_pairs_dc4(mol, -0.30, 0.40, 1.0), B_gradient=0.16)
    out = sim.simulate_ensemble_3d(list(t["r0"]), list(t["v0"]), float(t["t_max"]), float(t["dt"]))
    for i, (tt, R, V) in enumerate(out):
        assert np.abs(R - t["r"][i]).max() < 1e-9
        assert np.abs(V - t["v"][i]).max() < 1e-4
