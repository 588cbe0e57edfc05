"""GPU parity of the 1D steady-state force kernels against the oracle and the
reference's golden arrays.

Tolerances (max |dF| / max |F| over each parameter set):
  plain FP64 form:            1e-10  (the reference's JIT constant hbar)
  plain FP64, CODATA hbar:    1e-10  against the reference's pure-Python path
  FP32 bulk + FP64 LU/refine: 1e-6
"""
import numpy as np
import pytest

from conftest import golden
from oracle import rate_eq as orc

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-6


def rel_to_max(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(a)), np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def pack(mol, gpu):
    from molmot_b200.engine import MoleculePack
    return MoleculePack(mol)


def _beams(g, B):
    from molmot_b200.engine import BeamSets
    return BeamSets(g["kdir"], g["freq"], g["pol"], g["s0"], B)


@pytest.mark.parametrize("precision,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_config1_hallas_vs_reference_gpu_golden(pack, precision, tol):
    from molmot_b200.engine import force_batch
    g = golden("three_way_golden.npz")
    bs = _beams(g, float(g["B_gradient"]))
    out = force_batch(pack, bs, np.array([0.0]), g["z_arr"], grid=True, precision=precision)
    Fz = out["F"].cpu().numpy().ravel() / g["F_unit"]
    assert rel_to_max(Fz, g["Fz_gpu"]) < tol
    assert np.max(np.abs(out["pop"].cpu().numpy().reshape(-1, 12) - g["Pz_gpu"])) < tol * 10
    out = force_batch(pack, bs, g["v_arr"], np.array([0.0]), grid=True, precision=precision)
    assert rel_to_max(out["F"].cpu().numpy().ravel() / g["F_unit"], g["Fv_gpu"]) < tol


def test_config1_hallas_vs_reference_python_golden(pack):
    from molmot_b200.engine import force_batch
    from molmot_b200.constants import hbar
    g = golden("three_way_golden.npz")
    bs = _beams(g, float(g["B_gradient"]))
    out = force_batch(pack, bs, np.array([0.0]), g["z_arr"], grid=True, hbar=hbar,
                      uniform_fallback=True)
    assert rel_to_max(out["F"].cpu().numpy().ravel() / g["F_unit"], g["Fz_cpu_s"]) < TOL64


def test_config1_equal_split(pack):
    from molmot_b200.engine import force_batch
    g = golden("config1_equal_split.npz")
    bs = _beams(g, float(g["B_gradient"]))
    out = force_batch(pack, bs, np.array([0.0]), g["z"], grid=True)
    assert rel_to_max(out["F"].cpu().numpy().ravel(), g["Fz_jit"]) < TOL64
    assert np.max(np.abs(out["pop"].cpu().numpy().reshape(-1, 12) - g["Pz_jit"])) < 1e-12


@pytest.mark.parametrize("precision,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_random_parameter_sets_points_layout(pack, precision, tol):
    from molmot_b200.engine import BeamSets, force_batch
    g = golden("random_points.npz")
    ns, npts = int(g["n_sets"]), int(g["n_pts"])
    sel = lambda a: a.reshape(ns, npts, *a.shape[1:])[:, 0]
    bs = BeamSets(sel(g["kdir"]), sel(g["freq"]), sel(g["pol"]), sel(g["s0"]), sel(g["B"]))
    out = force_batch(pack, bs, g["v"], g["z"], points_per_set=npts, precision=precision)
    F = out["F"].cpu().numpy().reshape(ns, npts)
    Fj = g["F_jit"].reshape(ns, npts)
    # normalise by max|F| of each set's force map (v in +-10 m/s, z in +-10 mm),
    # which is how the tolerance is defined; 16 random points alone under-sample it
    vg, zg = np.linspace(-10, 10, 64), np.linspace(-1e-2, 1e-2, 64)
    for s in range(ns):
        Fmap = orc.force_batch(pack.mol, sel(g["kdir"])[s], sel(g["freq"])[s], sel(g["pol"])[s],
                               sel(g["s0"])[s], sel(g["B"])[s], vg, zg, grid=True,
                               want_pop=False)[0]
        scale = max(np.max(np.abs(Fmap)), np.max(np.abs(Fj[s])))
        assert np.max(np.abs(F[s] - Fj[s])) / scale < tol, s
    R = out["R"].cpu().numpy().reshape(ns, npts)
    assert rel_to_max(R, g["R_jit"].reshape(ns, npts)) < tol * 10
    assert np.all(out["status"].cpu().numpy() == 0)


def _random_sets(mol, rng, n_sets):
    """Parameter sets shaped like the batched-map workload: 4 detunings in
    [-40, 0] MHz, per-frequency s0 log-uniform in [0.1, 10], B' in [5, 40] G/cm."""
    E = mol.energies
    ref = np.array([E[15] - E[0], E[15] - E[0], E[15] - E[9], E[15] - E[9]])
    det = rng.uniform(-40e6, 0.0, (n_sets, 4))
    s0 = 10 ** rng.uniform(-1, 1, (n_sets, 4))
    B = rng.uniform(5, 40, n_sets) * 1e-2
    pols = np.array([2, 0, 2, 0])
    kdir = np.tile([1.0, -1.0], (n_sets, 4))
    freq = np.repeat(ref[None, :] + det, 2, axis=1)
    pol = np.tile(np.stack([pols, 2 - pols], 1).ravel(), (n_sets, 1))
    s0b = np.repeat(s0, 2, axis=1)
    return kdir, freq, pol, s0b, B


@pytest.mark.parametrize("precision,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_grid_layout_many_sets_vs_oracle(mol, pack, precision, tol):
    from molmot_b200.engine import BeamSets, force_batch
    rng = np.random.default_rng(7)
    n_sets = 12
    kdir, freq, pol, s0, B = _random_sets(mol, rng, n_sets)
    v = np.linspace(-10, 10, 48)
    z = np.linspace(-1e-2, 1e-2, 40)
    bs = BeamSets(kdir, freq, pol, s0, B)
    out = force_batch(pack, bs, v, z, grid=True, precision=precision)
    Fo, popo, Ro, sto = orc.force_batch(mol, kdir, freq, pol, s0, B, v, z, grid=True)
    F = out["F"].cpu().numpy().reshape(n_sets, -1)
    Fo = Fo.reshape(n_sets, -1)
    errs = [rel_to_max(F[s], Fo[s]) for s in range(n_sets)]
    assert max(errs) < tol, errs
    pop = out["pop"].cpu().numpy().reshape(-1, 12)
    assert np.max(np.abs(pop - popo)) < tol * 100
    assert np.allclose(pop.sum(1), 1.0, atol=1e-12)


def test_ragged_and_single_points(mol, pack):
    """Point counts that do not fill a CTA, a single point, and a tail set."""
    from molmot_b200.engine import BeamSets, force_batch
    rng = np.random.default_rng(3)
    kdir, freq, pol, s0, B = _random_sets(mol, rng, 3)
    bs = BeamSets(kdir, freq, pol, s0, B)
    for n, pps in [(1, 1), (7, 5), (37, 13), (1000, 400)]:
        v = rng.uniform(-10, 10, n)
        z = rng.uniform(-1e-2, 1e-2, n)
        out = force_batch(pack, bs, v, z, points_per_set=pps)
        Fo = orc.force_batch(mol, kdir, freq, pol, s0, B, v, z, points_per_set=pps)[0]
        assert rel_to_max(out["F"].cpu().numpy(), Fo) < TOL64, (n, pps)


def test_hbar_parameter_scales_force(pack, mol):
    from molmot_b200.engine import force_batch
    g = golden("config1_equal_split.npz")
    bs = _beams(g, float(g["B_gradient"]))
    a = force_batch(pack, bs, np.array([0.0]), g["z"], grid=True, hbar=1.0545718e-34)["F"]
    b = force_batch(pack, bs, np.array([0.0]), g["z"], grid=True, hbar=2 * 1.0545718e-34)["F"]
    assert rel_to_max(2 * a.cpu().numpy(), b.cpu().numpy()) < 1e-15


def test_argument_errors_raise(pack):
    from molmot_b200.engine import BeamSets, force_batch
    g = golden("config1_equal_split.npz")
    bs = _beams(g, 0.2)
    with pytest.raises(RuntimeError):
        force_batch(pack, bs, np.zeros(10), np.zeros(10), points_per_set=3)  # needs 4 sets
    with pytest.raises(RuntimeError):
        BeamSets(g["kdir"], g["freq"], np.full(8, 3), g["s0"], 0.2)


def test_traj1d_short_vs_reference(mol, pack):
    from molmot_b200.engine import BeamSets, traj1d
    g = golden("trajectory_golden.npz")
    bs = _beams(g, float(g["B_gradient"]))
    n_steps = g["short_z"].shape[1]
    zf, vf, na, zt, vt = traj1d(pack, bs, g["short_z"][:, 0], g["short_v"][:, 0], 1e-6, n_steps,
                                save_full=True)
    assert np.max(np.abs(zt.cpu().numpy() - g["short_z"])) < 1e-12
    assert np.max(np.abs(vt.cpu().numpy() - g["short_v"])) < 1e-9


def test_traj1d_reference_endpoints(mol, pack):
    """The reference's 4 trajectories and 100-particle batch (30,000 steps)."""
    from molmot_b200.engine import traj1d
    g = golden("trajectory_golden.npz")
    bs = _beams(g, float(g["B_gradient"]))
    n_steps = int(float(g["t_max"]) / float(g["dt"]))
    zf, vf, na, _, _ = traj1d(pack, bs, g["ref_z0"], g["ref_v0"], float(g["dt"]), n_steps)
    assert np.max(np.abs(zf.cpu().numpy() - g["ref_zf_jit"])) < 1e-10
    assert np.max(np.abs(vf.cpu().numpy() - g["ref_vf_jit"])) < 1e-8
    zf, vf, na, _, _ = traj1d(pack, bs, g["batch_z0"], g["batch_v0"], float(g["dt"]), n_steps)
    assert np.array_equal(na.cpu().numpy(), g["batch_n_actual"])
    assert np.max(np.abs(zf.cpu().numpy() - g["batch_zf_jit"])) < 1e-10
    assert np.max(np.abs(vf.cpu().numpy() - g["batch_vf_jit"])) < 1e-8
