"""Molecules beyond the register-resident kernel classes (n_ground > 12 or
n_excited > 4, up to 48 + 16) through the drop-in 1D entry points:
mm_force_batch (force_vs_z and force maps), mm_traj_run (1D and per-axis
trajectories) and mm_force_adjoint, as the reference's kernel compiles for
any molecule size (molmot_cuda/rate_equations_cuda.py:287-320).

Checks against the CPU oracle: forces, rates and populations at 1e-10 of
max |F| (every precision runs the FP64 shared-memory kernels for these
molecules); 1D trajectories to 1e-12 m after 300 steps; the per-axis model
against the oracle's point solve step by step; adjoint gradients against
FP64 torch autograd of the dense restatement at 1e-8 of the largest
component per set."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SIZES = [(16, 8, 31), (48, 16, 33), (24, 6, 32), (13, 4, 34), (8, 6, 35)]
TOL = 1e-10


def _mol(n_g, n_e, seed):
    from molmot_b200.molecules.synthetic import synthetic_molecule
    return synthetic_molecule(n_g, n_e, seed)


def _sets(m, n_sets, seed):
    """n_sets parameter sets around dc_beams_for(m): detunings moved by up to
    -10 MHz, s0 scaled by 0.3..3, B' in [0.1, 0.4] T/m."""
    from molmot_b200.molecules.synthetic import dc_beams_for
    kd, fr, po, s0 = dc_beams_for(m)
    rng = np.random.default_rng(seed)
    kdir = np.tile(kd, (n_sets, 1))
    freq = fr[None, :] + np.repeat(rng.uniform(-10e6, 0.0, (n_sets, 4)), 2, axis=1)
    pol = np.tile(po, (n_sets, 1))
    s0s = s0[None, :] * np.repeat(10 ** rng.uniform(-0.5, 0.5, (n_sets, 4)), 2, axis=1)
    B = rng.uniform(0.1, 0.4, n_sets)
    return kdir, freq, pol, s0s, B


@pytest.mark.parametrize("n_g,n_e,seed", SIZES)
@pytest.mark.parametrize("precision", ["fp64", "fp64_reduced", "fp32"])
def test_large_force_maps_vs_oracle(gpu, n_g, n_e, seed, precision):
    from molmot_b200.engine import BeamSets, MoleculePack, force_batch
    from oracle import rate_eq as orc
    m = _mol(n_g, n_e, seed)
    kdir, freq, pol, s0, B = _sets(m, 3, seed)
    v = np.linspace(-8, 8, 9)
    z = np.linspace(-8e-3, 8e-3, 11)
    out = force_batch(MoleculePack(m), BeamSets(kdir, freq, pol, s0, B), v, z, grid=True,
                      precision=precision)
    F, P, R, st = orc.force_batch(m, kdir, freq, pol, s0, B, v, z, grid=True)
    Fg = out["F"].cpu().numpy().reshape(3, -1)
    for s in range(3):
        sl = slice(s * 99, (s + 1) * 99)
        assert np.abs(Fg[s] - F[sl]).max() <= TOL * np.abs(F[sl]).max(), (s, precision)
    assert np.abs(out["R"].cpu().numpy().ravel() - R).max() <= TOL * np.abs(R).max()
    assert np.abs(out["pop"].cpu().numpy().reshape(-1, n_g) - P).max() <= TOL
    assert np.array_equal(out["status"].cpu().numpy().ravel(), st)


@pytest.mark.parametrize("n_g,n_e,seed", SIZES[:3])
def test_large_force_vs_z_api(gpu, n_g, n_e, seed):
    """force_vs_z / force_vs_v / spring_constant of the reference's API on a
    simulator with the molecule's own beams."""
    from molmot_b200 import force_scan as fs
    from molmot_b200.fields import LaserBeam
    from molmot_b200.simulator import BeamListSimulator
    from oracle import rate_eq as orc
    m = _mol(n_g, n_e, seed)
    kdir, freq, pol, s0, B = _sets(m, 1, seed + 1)
    beams = [LaserBeam(np.array([0.0, 0.0, kdir[0, b]]), freq[0, b], int(pol[0, b]), s0[0, b])
             for b in range(kdir.shape[1])]
    sim = BeamListSimulator(m, beams, float(B[0]))
    z = np.linspace(-5e-3, 5e-3, 101)
    F, P, R = fs.force_vs_z(sim, z, v=0.3)
    Fo, Po, Ro, _ = orc.force_batch(m, kdir, freq, pol, s0, B, np.full(101, 0.3), z, points_per_set=101)
    assert np.abs(F - Fo).max() <= TOL * np.abs(Fo).max()
    assert np.abs(P - Po).max() <= TOL
    vv = np.linspace(-5, 5, 41)
    Fv = fs.force_vs_v(sim, vv, z=1e-3)
    Fvo = orc.force_batch(m, kdir, freq, pol, s0, B, vv, np.full(41, 1e-3), points_per_set=41)[0]
    assert np.abs(Fv - Fvo).max() <= TOL * np.abs(Fvo).max()
    k = fs.spring_constant(sim)
    Fk = orc.force_batch(m, kdir, freq, pol, s0, B, np.zeros(2), np.array([0.3e-3, -0.3e-3]),
                         points_per_set=2)[0]
    assert k == pytest.approx(-(Fk[0] - Fk[1]) / 0.6e-3, rel=1e-9, abs=1e-30)


@pytest.mark.parametrize("n_g,n_e,seed", SIZES[:3])
def test_large_traj1d_vs_oracle(gpu, n_g, n_e, seed):
    from molmot_b200.engine import BeamSets, MoleculePack, traj
    from oracle import rate_eq as orc
    m = _mol(n_g, n_e, seed)
    kdir, freq, pol, s0, B = _sets(m, 1, seed + 2)
    rng = np.random.default_rng(seed)
    z0 = rng.normal(0, 2e-3, 40)
    v0 = rng.normal(0, 1.0, 40)
    o = traj(MoleculePack(m), BeamSets(kdir, freq, pol, s0, B), z0, v0, 1e-6, 300)
    zf, vf, na, _, _ = orc.traj1d(m, (kdir[0], freq[0], pol[0].astype(float), s0[0]), float(B[0]), z0, v0,
                                  1e-6, 300)
    assert np.abs(o["r_final"].cpu().numpy().ravel() - zf).max() <= 1e-12
    assert np.abs(o["v_final"].cpu().numpy().ravel() - vf).max() <= 1e-9
    assert np.array_equal(o["n_actual"].cpu().numpy(), na)


def test_large_per_axis_and_rf_average(gpu):
    """The per-axis model (ndim 3) and the two-set average (n_avg 2) against
    the oracle's point solve, step by step (symplectic Euler per axis, x and y
    at -B'/2)."""
    from molmot_b200.engine import BeamSets, MoleculePack, traj
    from oracle import rate_eq as orc
    m = _mol(16, 8, 31)
    kdir, freq, pol, s0, B = _sets(m, 2, 77)
    B[1] = -B[0]
    r0 = np.array([[1e-3, -0.5e-3, 0.8e-3], [-2e-3, 1e-3, 0.0]])
    v0 = np.array([[0.4, -0.2, 0.1], [0.0, 0.3, -0.5]])
    n = 40
    o = traj(MoleculePack(m), BeamSets(kdir, freq, pol, s0, B), r0, v0, 1e-6, n, ndim=3, n_avg=2)
    mult = [-0.5, -0.5, 1.0]
    for p in range(2):
        x, u = r0[p].copy(), v0[p].copy()
        for _ in range(1, n):
            for d in range(3):
                Fs = [orc.point(m, (kdir[a], freq[a], pol[a].astype(float), s0[a]), u[d], x[d],
                                B[a] * mult[d])[0] for a in range(2)]
                F = 0.5 * (Fs[0] + Fs[1])
                u[d] = u[d] + F / m.mass * 1e-6
                x[d] = x[d] + u[d] * 1e-6
        assert np.abs(o["r_final"].cpu().numpy()[p] - x).max() <= 1e-13
        assert np.abs(o["v_final"].cpu().numpy()[p] - u).max() <= 1e-10


@pytest.mark.parametrize("n_g,n_e,seed", [(16, 8, 31), (48, 16, 33)])
@pytest.mark.parametrize("precision", ["fp64", "fp64_reduced"])
def test_large_adjoint_vs_torch_autograd(gpu, n_g, n_e, seed, precision):
    from molmot_b200.autograd import steady_state_force
    from oracle import torch_dense as td
    m = _mol(n_g, n_e, seed)
    kdir, freq, pol, s0, B = _sets(m, 3, seed + 3)
    pps = 12
    rng = np.random.default_rng(seed)
    v = rng.uniform(-8, 8, 3 * pps)
    z = rng.uniform(-8e-3, 8e-3, 3 * pps)
    w = torch.as_tensor(rng.normal(size=3 * pps), dtype=torch.float64)

    def leaves(dev):
        return [torch.tensor(a, dtype=torch.float64, device=dev, requires_grad=True) for a in (freq, s0, B)]

    f1, p1, b1 = leaves(gpu)
    F1 = steady_state_force(m, kdir, pol, f1, p1, b1, v, z, pps, precision=precision)
    (F1.cpu() * w).sum().backward()
    f2, p2, b2 = leaves("cpu")
    F2 = td.force(m, kdir, pol, f2, p2, b2, v, z, pps)
    assert np.abs(F1.detach().cpu().numpy() - F2.detach().numpy()).max() <= TOL * F2.abs().max().item()
    (F2 * w).sum().backward()
    for a, b in [(f1, f2), (p1, p2), (b1, b2)]:
        ga, gb = a.grad.cpu().numpy(), b.grad.numpy()
        scale = np.abs(gb).max(axis=-1, keepdims=True) if gb.ndim > 1 else np.abs(gb).max()
        assert np.all(np.abs(ga - gb) <= 1e-8 * scale + 1e-300), float(np.max(np.abs(ga - gb) / scale))


def test_large_nonfinite_and_empty(gpu):
    from molmot_b200.engine import BeamSets, MoleculePack, force_batch
    m = _mol(16, 8, 31)
    kdir, freq, pol, s0, B = _sets(m, 1, 5)
    v = np.array([0.5, np.nan, 1.0, np.inf])
    z = np.array([1e-3, 0.0, np.nan, 2e-3])
    out = force_batch(MoleculePack(m), BeamSets(kdir, freq, pol, s0, B), v, z, points_per_set=4)
    F = out["F"].cpu().numpy()
    st = out["status"].cpu().numpy()
    assert np.isfinite(F[0]) and np.all(np.isnan(F[1:]))
    assert np.all(st[1:] & 2) and st[0] == 0
    e = force_batch(MoleculePack(m), BeamSets(kdir, freq, pol, s0, B), np.zeros(0), np.zeros(0))
    assert e["F"].numel() == 0
