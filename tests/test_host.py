"""Host-side logic that needs no GPU: inputs, samplers, simulator adapters."""
import numpy as np
import pytest

from conftest import golden


def test_sroh_loader_matches_golden_beams(mol):
    from molmot_b200.fields import make_dc_mot_beams
    g = golden("trajectory_golden.npz")
    b = make_dc_mot_beams(mol, delta_Gamma=-0.20, split_Gamma=0.70, s0=1.0)
    assert np.array_equal([x.freq_offset for x in b], g["freq"])
    assert np.array_equal([x.polarization for x in b], g["pol"])
    assert np.array_equal([x.kdir_z for x in b], g["kdir"])


def test_molecule_derived_fields(mol):
    assert mol.d_squared.shape == (12, 4, 3)
    assert int((mol.d_squared > 1e-15).sum()) == 39
    assert mol.omega_J32 > mol.omega_J12  # J=1/2 lies ~55 MHz above J=3/2
    from molmot_b200.flops import active_triples, flops_per_point
    from molmot_b200.fields import make_dc_mot_beams
    pols = [b.polarization for b in make_dc_mot_beams(mol)]
    A = active_triples(mol.d_squared, pols)
    assert A == 96
    assert abs(flops_per_point(12, 4, 8, A)[0] - 4822) < 1


def test_constants():
    from molmot_b200 import constants as C
    from molmot_b200.molecules import K_WAVE, MASS_KG
    assert abs(C.v_recoil(K_WAVE, MASS_KG) - 5.53e-3) < 0.02e-3
    assert C.HBAR_JIT != C.hbar


def test_samplers_moments():
    from molmot_b200 import trajectories as tr
    rng = np.random.default_rng(42)
    v = tr.sample_maxwell_boltzmann(5e-3, 1.74356601993e-25, 10000, rng)
    sigma = np.sqrt(1.380649e-23 * 5e-3 / 1.74356601993e-25)
    assert abs(v.std() / sigma - 1) < 0.1 and abs(sigma - 0.629) < 0.01
    r = tr.sample_gaussian_position(1e-3, 10000, rng)
    assert abs(r.std() / 1e-3 - 1) < 0.1
    d = np.array([tr.sample_direction(rng) for _ in range(2000)])
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0)
    assert np.all(np.abs(d.mean(0)) < 0.1)
    u = tr.sample_uniform_sphere(2e-3, 500, rng)
    assert np.all(np.linalg.norm(u, axis=1) <= 2e-3)
    vs = tr.make_velocity_sampler(5e-3, 1.74356601993e-25)
    vv = np.array([vs() for _ in range(4000)])
    assert vv.shape == (4000, 3) and abs(vv.std() / sigma - 1) < 0.1
    assert np.array_equal(tr.make_velocity_sampler(5e-3, 1.0, "fixed")(), np.zeros(3))
    ps = tr.make_position_sampler(1e-3, "uniform_sphere")
    assert np.linalg.norm(ps()) <= 1e-3
    with pytest.raises(ValueError):
        tr.make_velocity_sampler(5e-3, 1.0, "thermal")


def test_as_gpu_simulator_rejects_unknown():
    from molmot_b200.simulator import as_gpu_simulator
    with pytest.raises(TypeError):
        as_gpu_simulator(object())


def test_reference_simulator_objects_adapt(mol):
    """The reference's DC/RF simulator classes map onto GPU simulators
    (attribute-compatible), checked without launching anything."""
    from molmot_b200.simulator import as_gpu_simulator, BeamListSimulator, RFMOTSimulator

    class RefDC:
        pass
    s = RefDC()
    s.mol_data, s._beams, s.B_gradient, s.Gamma_eff_factor = mol, [], 0.16, 1.0
    assert isinstance(as_gpu_simulator(s), BeamListSimulator)

    class RefRF:
        pass
    r = RefRF()
    r.mol_data, r.delta_Gamma, r.s0, r.B_gradient, r.Gamma_eff_factor = mol, -1.0, 1.0, 0.16, 1.0
    g = as_gpu_simulator(r)
    assert isinstance(g, RFMOTSimulator)
    (b0, B0), (b1, B1) = g.param_sets()
    assert B0 == -B1 and [x.polarization for x in b0] != [x.polarization for x in b1]


def test_trajectory_gradient_parameter_maps():
    """Host-side checks of mm_traj_grad_run's parameter maps (no GPU)."""
    from molmot_b200 import _lib
    from molmot_b200.trajgrad import _param_map
    m = _param_map([0, 0, 1, 1, -1, -1, 2, 2], 8, 3, "freq_par")
    assert list(m)[:8] == [0, 0, 1, 1, -1, -1, 2, 2] and all(x == -1 for x in list(m)[8:])
    assert len(m) == _lib.MM_MAX_BEAMS
    assert all(x == -1 for x in _param_map(None, 8, 3, "s0_par"))
    with pytest.raises(ValueError):
        _param_map([0, 3], 2, 3, "freq_par")       # index beyond n_par
    with pytest.raises(ValueError):
        _param_map([0, 1, 2], 2, 3, "freq_par")    # one entry per beam
    import ctypes
    assert ctypes.sizeof(_lib.TgradOpts) == 8 * 7 + 4 * 2 + 4 * 2 * _lib.MM_MAX_BEAMS + 4 * 2


def test_static_uneven_output_checks():
    """UnevenBatch.force_static hands the caller's buffers to the kernels as
    they are, so each must be rejected on the host when its dtype, device,
    layout or length is wrong (no GPU needed: the checks run first)."""
    import torch
    from molmot_b200.uneven import check_static_out
    dev = torch.device("cuda", 0)
    n = 10
    ok = torch.empty(n, dtype=torch.float64)  # right dtype and length, but on the host
    with pytest.raises(ValueError, match="must be on cuda:0"):
        check_static_out({"F": ok}, n, dev)
    cpu = torch.device("cpu")  # the same rules, checked against the host device
    check_static_out({"F": ok, "R": ok.clone(), "status": torch.zeros(n, dtype=torch.int32)}, n, cpu)
    with pytest.raises(ValueError, match="'F'"):
        check_static_out({}, n, cpu)
    with pytest.raises(ValueError, match="float64"):
        check_static_out({"F": torch.empty(n, dtype=torch.float32)}, n, cpu)
    with pytest.raises(ValueError, match="int32"):
        check_static_out({"F": ok, "status": torch.zeros(n, dtype=torch.int64)}, n, cpu)
    with pytest.raises(ValueError, match="contiguous"):
        check_static_out({"F": torch.empty(2 * n, dtype=torch.float64)[::2]}, n, cpu)
    with pytest.raises(ValueError, match="hold 10"):
        check_static_out({"F": torch.empty(n - 1, dtype=torch.float64)}, n, cpu)
    with pytest.raises(ValueError, match="unknown output"):
        check_static_out({"F": ok, "pop": ok}, n, cpu)
