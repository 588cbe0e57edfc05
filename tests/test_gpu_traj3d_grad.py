"""Tangents of the 3D leapfrog ensemble through the 24-beam force
(mm_traj3d_grad_run, trajgrad.traj3d_grad): d(r, v)/d theta for the four
frequency components, a saturation parameter shared by all beams and B',
on synthetic molecules whose ground Zeeman spectrum is non-degenerate
(12 + 4 and 16 + 8 levels, the molecules of force3d_reference.npz).

Checks:
  * the trajectory equals mm_traj3d_run's (MOTSimulator3D.run_ensemble) bit
    for bit, recoil kicks included;
  * tangents equal FP64 torch autograd through the unrolled dense leapfrog
    (oracle/torch_dense3d.py, torch.linalg.eigh) to 1e-8 of each parameter's
    largest tangent, with kicks held fixed;
  * tangents agree with central differences of the GPU trajectory to 1e-3
    (the difference quotients carry ~1e-4 of rounding noise: transition
    frequencies round to 1/16 Hz at 4.3e14 Hz);
  * a run resumed from a checkpoint gives the unbroken run's bits;
  * SrOH, whose spectrum has exactly degenerate 6 + 6 clusters, is refused.
"""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

N_STEPS = 40
R0 = np.array([[1e-3, -1e-3, 0.5e-3], [0.0, 0.5e-3, -2e-3], [2e-3, 1e-3, 0.4e-3]])
V0 = np.array([[0.3, 0.2, -0.5], [-0.4, 0.0, 0.6], [0.0, 0.1, 0.1]])


def _setup(i):
    from molmot_b200.engine import beam_sets_3d, pack_for
    from molmot_b200.molecules.synthetic import synthetic_molecule
    g = golden("force3d_reference.npz")
    K = lambda k: g[f"m{i}_{k}"]
    m = synthetic_molecule(int(K("ng")), int(K("ne")), int(K("seed")))
    beams = tuple(np.array(K(k)) for k in ("khat", "freq", "q", "s0", "radius"))
    B = float(K("B"))
    # parameters: the four frequency components (beams 6 c .. 6 c + 5 share
    # component c), one s0 shift for every beam, B'
    n_b = len(beams[1])
    comp = np.array([b // (n_b // 4) for b in range(n_b)])
    freq_par = list(comp)
    s0_par = [4] * n_b
    return m, pack_for(m), beams, B, freq_par, s0_par, 5


def _run(m, pack, beams, B, freq_par, s0_par, bp, theta=None, **kw):
    from molmot_b200.engine import beam_sets_3d
    from molmot_b200.trajgrad import traj3d_grad
    kh, fq, q, s0, rad = beams
    fq = fq.copy()
    s0 = s0.copy()
    if theta is not None:
        fq = fq + np.array([theta[k] for k in freq_par])
        s0 = s0 + theta[4]
        B = B + theta[5]
    bs = beam_sets_3d(kh, fq, q, s0, rad, B)
    return traj3d_grad(pack, bs, R0, V0, 1e-6, N_STEPS, n_par=6, freq_par=freq_par, s0_par=s0_par,
                       bprime_par=bp, **kw)


@pytest.mark.parametrize("i", [0, 2])
def test_trajectory_equals_traj3d_run(gpu, i):
    from molmot_b200.constants import hbar as HBAR_CODATA
    from molmot_b200.engine import beam_sets_3d, traj3d
    m, pack, beams, B, fp, sp, bp = _setup(i)
    out = _run(m, pack, beams, B, fp, sp, bp, kicks=True, seed=77)
    ref = traj3d(pack, beam_sets_3d(*beams, B), R0, V0, 1e-6, N_STEPS, kicks=True, seed=77, hbar=HBAR_CODATA)
    assert torch.equal(out["r"], ref["r"]) and torch.equal(out["vh"], ref["vh"])
    assert torch.equal(out["v"], ref["v"])
    assert torch.equal(out["n_events"], ref["n_events"]) and int(out["n_events"].sum()) > 0
    assert int(out["status"].abs().sum()) == 0


def _torch_tangents(m, beams, B, fp, sp, bp, kicks=None):
    """d v_sync / d theta and d r / d theta (N, 3, 6) by torch autograd
    through the unrolled dense leapfrog; kicks [n_steps, N, 3] held fixed."""
    from oracle import torch_dense3d as td3
    kh, fq, q, s0, rad = beams
    theta = torch.zeros(6, dtype=torch.float64, requires_grad=True)
    M = torch.zeros((len(fq), 6), dtype=torch.float64)
    for b, k in enumerate(fp):
        M[b, k] = 1.0
    freq = torch.as_tensor(fq) + M @ theta
    s0t = torch.as_tensor(s0) + theta[4]
    Bt = torch.as_tensor(B, dtype=torch.float64) + theta[5]
    r0 = torch.as_tensor(R0)
    v0 = torch.as_tensor(V0)
    vs, r = td3.leapfrog(m, (kh, freq, q, s0t, rad), Bt, r0, v0, N_STEPS, kicks=kicks)
    out = np.zeros((2, R0.shape[0], 3, 6))
    for w, y in enumerate((vs, r)):
        for p in range(R0.shape[0]):
            for c in range(3):
                out[w, p, c] = torch.autograd.grad(y[p, c], theta, retain_graph=True)[0].numpy()
    return out[0], out[1], vs.detach().numpy(), r.detach().numpy()


def _check(a, b, tol):
    scale = np.abs(b).max(axis=(0, 1), keepdims=True)  # per parameter
    assert np.all(np.abs(a - b) <= tol * scale), float((np.abs(a - b) / scale).max())


@pytest.mark.parametrize("i", [0, 2])
def test_tangents_vs_torch_autograd(gpu, i):
    m, pack, beams, B, fp, sp, bp = _setup(i)
    out = _run(m, pack, beams, B, fp, sp, bp)
    dv_t, dr_t, vs_t, r_t = _torch_tangents(m, beams, B, fp, sp, bp)
    assert np.abs(out["v"].cpu().numpy() - vs_t).max() <= 1e-10 * np.abs(vs_t).max()
    assert np.abs(out["r"].cpu().numpy() - r_t).max() <= 1e-12
    _check(out["dv"].cpu().numpy(), dv_t, 1e-8)
    _check(out["dr"].cpu().numpy(), dr_t, 1e-8)


def test_tangents_with_fixed_kicks_vs_torch_autograd(gpu):
    """Kicks on: the torch model adds the same kick vectors (the oracle's
    Philox draws at the GPU trajectory's rates), held fixed."""
    from oracle import force3d as o3
    from oracle import torch_dense3d as td3
    m, pack, beams, B, fp, sp, bp = _setup(0)
    out = _run(m, pack, beams, B, fp, sp, bp, kicks=True, seed=5)
    kh, fq, q, s0, rad = beams
    # the kicks of each update from the dense model's own rates (its trajectory
    # agrees with the GPU's to rounding, so the Poisson counts are the same)
    v_rec = 1.054571817e-34 * m.k / m.mass
    kicks = np.zeros((N_STEPS, R0.shape[0], 3))
    with torch.no_grad():
        r = torch.as_tensor(R0)
        F0 = td3.force3d(m, kh, fq, q, s0, rad, r, torch.as_tensor(V0), B)[0]
        vh = torch.as_tensor(V0) + 0.5e-6 * F0 / m.mass
        for j in range(1, N_STEPS):
            r = r + 1e-6 * vh
            F, Rs, _ = td3.force3d(m, kh, fq, q, s0, rad, r, vh, B)
            for p in range(R0.shape[0]):
                kicks[j, p] = o3.recoil_kick(5, p, j, float(Rs[p]), 1e-6, v_rec)[0]
            vh = vh + 1e-6 * F / m.mass + torch.as_tensor(kicks[j])
    dv_t, dr_t, vs_t, _ = _torch_tangents(m, beams, B, fp, sp, bp, kicks=torch.as_tensor(kicks))
    assert np.abs(out["v"].cpu().numpy() - vs_t).max() <= 1e-10 * np.abs(vs_t).max()
    _check(out["dv"].cpu().numpy(), dv_t, 1e-8)
    _check(out["dr"].cpu().numpy(), dr_t, 1e-8)


def test_tangents_vs_central_differences(gpu):
    m, pack, beams, B, fp, sp, bp = _setup(0)
    out = _run(m, pack, beams, B, fp, sp, bp)
    dv = out["dv"].cpu().numpy()
    base_s0 = beams[3][0]
    for k, h in [(0, 2e4), (3, 2e4), (4, 1e-4 * base_s0), (5, 1e-4 * B)]:
        th = np.zeros(6)
        th[k] = h
        vp = _run(m, pack, beams, B, fp, sp, bp, theta=th)["v"].cpu().numpy()
        th[k] = -h
        vm = _run(m, pack, beams, B, fp, sp, bp, theta=th)["v"].cpu().numpy()
        fd = (vp - vm) / (2 * h)
        scale = np.abs(dv[:, :, k]).max()
        assert np.abs(fd - dv[:, :, k]).max() <= 1e-3 * scale, k


def test_checkpoint_resume_bitwise(gpu):
    m, pack, beams, B, fp, sp, bp = _setup(0)
    full = _run(m, pack, beams, B, fp, sp, bp, kicks=True, seed=3, ckpt_every=10)
    assert full["ckpt"].shape[0] == 3  # updates 10, 20, 30 of 1..39
    from molmot_b200.engine import beam_sets_3d
    from molmot_b200.trajgrad import traj3d_grad
    res = traj3d_grad(pack, beam_sets_3d(*beams, B), None, None, 1e-6, N_STEPS - 21, n_par=6,
                      freq_par=fp, s0_par=sp, bprime_par=bp, kicks=True, seed=3, step0=21,
                      state=full["ckpt"][1], n_actual=torch.zeros(3, dtype=torch.int32))
    assert torch.equal(res["state"], full["state"])
    assert torch.equal(res["v"], full["v"]) and torch.equal(res["dv"], full["dv"])


def test_sroh_is_refused(mol, gpu):
    from molmot_b200.engine import pack_for
    from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
    from molmot_b200.trajgrad import DegenerateSpectrum, traj3d_grad
    sim = MOTSimulator3D(mol, make_beam_pairs_dc4(mol, -0.30, 0.40, 1.0), B_gradient=0.16)
    with pytest.raises(DegenerateSpectrum):
        traj3d_grad(pack_for(mol), sim._bs(), R0, V0, 1e-6, 5, n_par=1, freq_par=[0] * 24)
