"""Trajectory tangents of the per-axis 3D MOT model (mm_traj_grad_run).

Checks, SrOH 4-frequency DC MOT (8 beams), parameters: the 4 detunings,
the s0 of the first frequency component and B':
  * the trajectories equal the per-axis model of mm_traj_run (FP64) to 1e-9
    of the state's scale, stop steps included;
  * tangents against FP64 torch autograd through the same model unrolled with
    the dense restatement of oracle/torch_dense.py -- 1e-8 of the largest
    tangent component of each parameter;
  * tangents against central differences of the kernel's own trajectories
    (relative steps 1e-3) -- 1e-5 of the largest component;
  * with recoil kicks (fixed noise): the same central differences on the
    particles whose Poisson counts the steps leave unmoved (at least 14 of
    16; a particle whose count moves shows a jump of a whole recoil kick);
  * a run resumed from a checkpoint gives the unbroken run's bits.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DT = 1e-6
FREQ_PAR = [0, 0, 1, 1, 2, 2, 3, 3]
S0_PAR = [4, 4, -1, -1, -1, -1, -1, -1]
BP_PAR = 5
N_PAR = 6


@pytest.fixture(scope="module")
def setup(mol, gpu):
    from molmot_b200.engine import MoleculePack
    from molmot_b200.fields import beam_arrays, make_dc_mot_beams
    kdir, freq, pol, s0 = beam_arrays(make_dc_mot_beams(mol, delta_Gamma=-0.20, split_Gamma=0.70,
                                                       s0=2.0))
    s0 = s0 * np.array([1.0, 1.0, 0.7, 0.7, 1.3, 1.3, 0.9, 0.9])
    return MoleculePack(mol), kdir, freq, pol, s0, 0.16


def _bs(kdir, freq, pol, s0, bg):
    from molmot_b200.engine import BeamSets
    return BeamSets(kdir[None], freq[None], pol[None], s0[None], [bg])


def _shift(freq, s0, bg, k, h):
    f, s, b = freq.copy(), s0.copy(), bg
    if k < 4:
        f[np.array(FREQ_PAR) == k] += h
    elif k == 4:
        s[np.array(S0_PAR) == 4] += h
    else:
        b += h
    return f, s, b


def _ens(n, seed, v_sigma=0.63):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 1e-3, (n, 3)), rng.normal(0, v_sigma, (n, 3))


def _run(pack, kdir, freq, pol, s0, bg, r0, v0, n_steps, **kw):
    from molmot_b200.trajgrad import traj_grad
    out = traj_grad(pack, _bs(kdir, freq, pol, s0, bg), r0, v0, DT, n_steps, n_par=N_PAR,
                    freq_par=FREQ_PAR, s0_par=S0_PAR, bprime_par=BP_PAR, **kw)
    torch.cuda.synchronize()
    return out


def test_trajectories_equal_per_axis_model(setup):
    from molmot_b200.engine import traj
    pack, kdir, freq, pol, s0, bg = setup
    r0, v0 = _ens(64, 1)
    v0[:4] *= 80.0  # a few fast particles leave the 15 mm sphere within the run
    S = 400
    g = _run(pack, kdir, freq, pol, s0, bg, r0, v0, S)
    t = traj(pack, _bs(kdir, freq, pol, s0, bg), r0, v0, DT, S + 1, ndim=3)
    # mm_traj_run counts samples (S + 1 for a particle that stayed), the
    # gradient run the absolute step a particle stopped at
    assert torch.equal(g["n_actual"], torch.where(t["n_actual"] == S + 1, S, t["n_actual"]))
    assert int((g["n_actual"] < S).sum()) >= 1
    assert float((g["r"] - t["r_final"]).abs().max()) < 1e-9 * 1e-2
    assert float((g["v"] - t["v_final"]).abs().max()) < 1e-9 * float(t["v_final"].abs().max())


def test_tangents_vs_torch_autograd(setup, mol):
    from oracle import torch_dense as td
    pack, kdir, freq, pol, s0, bg = setup
    n, S = 4, 40
    r0, v0 = _ens(n, 2)
    g = _run(pack, kdir, freq, pol, s0, bg, r0, v0, S)
    r_gpu = g["r"].cpu().numpy().ravel()
    dr = g["dr"].cpu().numpy().reshape(3 * n, N_PAR)
    dv = g["dv"].cpu().numpy().reshape(3 * n, N_PAR)
    theta = torch.zeros(N_PAR, dtype=torch.float64, requires_grad=True)
    fq = torch.as_tensor(freq) + torch.stack([theta[k] for k in FREQ_PAR])
    sv = torch.as_tensor(s0) + torch.stack([theta[k] if k >= 0 else torch.zeros((), dtype=torch.float64)
                                            for k in S0_PAR])
    Bp = bg + theta[BP_PAR]
    mult = torch.tensor([-0.5, -0.5, 1.0], dtype=torch.float64)
    npts = 3 * n
    Fq = fq[None].expand(npts, -1)
    Sv = sv[None].expand(npts, -1)
    Bg = (Bp * mult).repeat(n)
    Kd = np.ascontiguousarray(np.broadcast_to(kdir, (npts, len(kdir))))
    Po = np.ascontiguousarray(np.broadcast_to(pol, (npts, len(pol))))
    x = torch.as_tensor(r0.ravel())
    u = torch.as_tensor(v0.ravel())
    for _ in range(S):
        F = td.force(mol, Kd, Po, Fq, Sv, Bg, u, x, 1)
        u = u + F / mol.mass * DT
        x = x + u * DT
    rng = np.random.default_rng(3)
    wx = torch.as_tensor(rng.normal(size=npts)) * 1e3
    wv = torch.as_tensor(rng.normal(size=npts))
    ((wx * x).sum() + (wv * u).sum()).backward()
    ref = theta.grad.numpy()
    got = wx.numpy() @ dr + wv.numpy() @ dv
    assert np.allclose(r_gpu, x.detach().numpy(), rtol=0, atol=1e-13)
    scale = np.abs(wx.numpy())[:, None] * np.abs(dr) + np.abs(wv.numpy())[:, None] * np.abs(dv)
    assert np.all(np.abs(got - ref) <= 1e-8 * scale.sum(0)), (got, ref)


def test_tangents_vs_central_fd(setup):
    pack, kdir, freq, pol, s0, bg = setup
    r0, v0 = _ens(32, 4)
    S = 250
    g = _run(pack, kdir, freq, pol, s0, bg, r0, v0, S)
    steps = [1e4, 1e4, 1e4, 1e4, 1e-3 * s0[0], 1e-3 * bg]
    for k in range(N_PAR):
        fp, sp, bp = _shift(freq, s0, bg, k, steps[k])
        fm, sm, bm = _shift(freq, s0, bg, k, -steps[k])
        # the step the parameter actually took (frequencies near 4.3e14 Hz round to 1/16 Hz)
        h2 = (fp - fm).max() if k < 4 else (sp - sm).max() if k == 4 else bp - bm
        a = _run(pack, kdir, fp, pol, sp, bp, r0, v0, S)
        b = _run(pack, kdir, fm, pol, sm, bm, r0, v0, S)
        for key, dkey in (("r", "dr"), ("v", "dv")):
            fd = ((a[key] - b[key]) / h2).cpu().numpy()
            tg = g[dkey][:, :, k].cpu().numpy()
            assert np.max(np.abs(fd - tg)) <= 1e-5 * np.max(np.abs(tg)), (k, key)


def test_kicks_at_fixed_noise(setup):
    pack, kdir, freq, pol, s0, bg = setup
    r0, v0 = _ens(16, 5)
    S = 60
    kw = dict(kicks=True, seed=1234)
    g = _run(pack, kdir, freq, pol, s0, bg, r0, v0, S, **kw)
    quiet = _run(pack, kdir, freq, pol, s0, bg, r0, v0, S)
    assert float((g["v"] - quiet["v"]).abs().max()) > 1e-3  # kicks of ~5.5 mm/s happened
    ok = np.ones(16, bool)
    # steps well above the model's own resolution: the Doppler-shifted beam
    # frequency (~4.3e14 Hz) rounds to 1/16 Hz, so smaller steps see a staircase
    for k in (0, 3, 5):
        h = 1e4 if k < 4 else 1e-3 * bg
        fp, sp, bp = _shift(freq, s0, bg, k, h)
        fm, sm, bm = _shift(freq, s0, bg, k, -h)
        h2 = (fp - fm).max() if k < 4 else bp - bm
        a = _run(pack, kdir, fp, pol, sp, bp, r0, v0, S, **kw)
        b = _run(pack, kdir, fm, pol, sm, bm, r0, v0, S, **kw)
        fd = ((a["v"] - b["v"]) / h2).cpu().numpy()
        tg = g["dv"][:, :, k].cpu().numpy()
        err = np.abs(fd - tg).max(axis=1)
        ok &= err <= 1e-5 * np.abs(tg).max()
    assert ok.sum() >= 14, ok


def test_checkpoint_resume_bitwise(setup):
    pack, kdir, freq, pol, s0, bg = setup
    r0, v0 = _ens(48, 6)
    v0[:3] *= 60.0
    kw = dict(kicks=True, seed=99)
    full = _run(pack, kdir, freq, pol, s0, bg, r0, v0, 300, ckpt_every=50, **kw)
    ck = full["ckpt"]
    assert ck.shape[0] == 6
    assert torch.equal(ck[-1], full["state"])
    half = _run(pack, kdir, freq, pol, s0, bg, r0, v0, 100, **kw)
    assert torch.equal(half["state"], ck[1])
    rest = _run(pack, kdir, freq, pol, s0, bg, None, None, 200, state=ck[1], step0=100,
                n_actual=half["n_actual"], **kw)
    assert torch.equal(rest["state"], full["state"])
    assert torch.equal(rest["n_actual"], full["n_actual"])


def test_small_and_large_ensemble_paths_agree(setup):
    """An ensemble of at most one CTA per SM keeps the rate sums in shared
    memory and runs the gradient pass beam by beam; a larger one recomputes
    the rates and runs it ground state by ground state.  The same particles
    give the same trajectories bit for bit and the same tangents to
    rounding in both."""
    pack, kdir, freq, pol, s0, bg = setup
    r_small, v_small = _ens(64, 21)
    r_big, v_big = _ens(16384, 22)  # 4 lanes per particle: 512 CTAs of 128 threads
    r_big[:64], v_big[:64] = r_small, v_small
    kw = dict(kicks=True, seed=5)
    a = _run(pack, kdir, freq, pol, s0, bg, r_small, v_small, 120, **kw)
    b = _run(pack, kdir, freq, pol, s0, bg, r_big, v_big, 120, **kw)
    sa, sb = a["state"], b["state"][:64]
    assert torch.equal(sa[:, :6], sb[:, :6])
    assert torch.equal(a["n_actual"], b["n_actual"][:64])
    tan_a, tan_b = sa[:, 6:], sb[:, 6:]
    scale = tan_a.abs().amax(dim=0).clamp_min(1e-300)
    assert float(((tan_a - tan_b).abs() / scale).max()) < 1e-12


def test_mean_kinetic_energy_autograd(setup):
    from molmot_b200.trajgrad import mean_kinetic_energy
    pack, kdir, freq, pol, s0, bg = setup
    r0, v0 = _ens(32, 7)
    theta = torch.zeros(N_PAR, dtype=torch.float64, requires_grad=True)
    E = mean_kinetic_energy(theta, pack, kdir, freq, pol, s0, bg, r0, v0, DT, 200, freq_par=FREQ_PAR,
                            s0_par=S0_PAR, bprime_par=BP_PAR)
    E.backward()
    g = _run(pack, kdir, freq, pol, s0, bg, r0, v0, 200)
    m = pack.mass
    assert abs(E.item() - 0.5 * m * float((g["v"] ** 2).sum(1).mean())) <= 1e-15 * E.item()
    ref = (m * (g["v"][:, :, None] * g["dv"]).sum(1).mean(0)).cpu()
    assert torch.allclose(theta.grad, ref, rtol=1e-14, atol=0)


def test_rejects_bad_parameter_maps(setup):
    from molmot_b200.trajgrad import traj_grad
    pack, kdir, freq, pol, s0, bg = setup
    r0, v0 = _ens(4, 8)
    with pytest.raises(ValueError):
        traj_grad(pack, _bs(kdir, freq, pol, s0, bg), r0, v0, DT, 10, n_par=2, freq_par=FREQ_PAR)
    with pytest.raises(RuntimeError):
        traj_grad(pack, _bs(kdir, freq, pol, s0, bg), r0, v0, DT, 10, n_par=2, bprime_par=5)
