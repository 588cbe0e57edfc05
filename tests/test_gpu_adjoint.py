"""Adjoint gradients of the steady-state force (mm_force_adjoint) and of the
MOT coefficients k, beta (33-point stencils) with respect to the 4
detunings, 4 powers (s0) and B'.

Both adjoint forms (precision "fp64": the elimination's transposed solve;
"fp64_reduced": the excited-chain solve's transposed system) are checked:
  * against FP64 torch autograd of a dense restatement (oracle/torch_dense.py)
    -- tolerance 1e-8 of the largest gradient component per parameter set;
  * against central finite differences of the GPU forward with
    h = 1e-4 relative (1e-3 for B') -- tolerance 1e-5 relative;
  * against each other on smaller molecules (1e-9 of the largest component);
  * the reduced form's forward equals mm_force_batch's FP64-reduced force bit
    for bit, and a batch with a structurally invalid set runs the elimination
    adjoint (bit-identical to precision "fp64").
"""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _sets(mol, n_sets, seed):
    """Parameter sets as in the batched-map workload: 4 detunings in [-40, 0] MHz,
    per-frequency s0 log-uniform in [0.1, 10], B' in [5, 40] G/cm."""
    rng = np.random.default_rng(seed)
    E = mol.energies
    ref = np.array([E[15] - E[0], E[15] - E[0], E[15] - E[9], E[15] - E[9]])
    det = rng.uniform(-40e6, 0.0, (n_sets, 4))
    s0 = 10 ** rng.uniform(-1, 1, (n_sets, 4))
    B = rng.uniform(5, 40, n_sets) * 1e-2
    pols = np.array([2, 0, 2, 0])
    kdir = np.tile([1.0, -1.0], (n_sets, 4))
    pol = np.tile(np.stack([pols, 2 - pols], 1).ravel(), (n_sets, 1))
    return ref, det, s0, B, kdir, pol


def _params(ref, det, s0, B, dev):
    f = torch.tensor(det, dtype=torch.float64, device=dev, requires_grad=True)
    p = torch.tensor(s0, dtype=torch.float64, device=dev, requires_grad=True)
    b = torch.tensor(B, dtype=torch.float64, device=dev, requires_grad=True)
    freq = (torch.as_tensor(ref, dtype=torch.float64, device=dev)[None, :] + f).repeat_interleave(2, 1)
    s0b = p.repeat_interleave(2, 1)
    return f, p, b, freq, s0b


@pytest.mark.parametrize("precision", ["fp64", "fp64_reduced"])
def test_adjoint_vs_torch_autograd(mol, gpu, precision):
    from molmot_b200.autograd import steady_state_force
    from oracle import torch_dense as td
    ref, det, s0, B, kdir, pol = _sets(mol, 6, 1)
    rng = np.random.default_rng(2)
    pps = 40
    v = rng.uniform(-10, 10, 6 * pps)
    z = rng.uniform(-1e-2, 1e-2, 6 * pps)
    w = torch.as_tensor(rng.normal(size=6 * pps), dtype=torch.float64)
    f1, p1, b1, freq1, s01 = _params(ref, det, s0, B, gpu)
    F1 = steady_state_force(mol, kdir, pol, freq1, s01, b1, v, z, pps, precision=precision)
    (F1.cpu() * w).sum().backward()
    f2, p2, b2, freq2, s02 = _params(ref, det, s0, B, "cpu")
    F2 = td.force(mol, kdir, pol, freq2, s02, b2, v, z, pps)
    assert np.abs(F1.detach().cpu().numpy() - F2.detach().numpy()).max() < 1e-10 * F2.abs().max().item()
    (F2 * w).sum().backward()
    for a, b in [(f1, f2), (p1, p2), (b1, b2)]:
        ga, gb = a.grad.cpu().numpy(), b.grad.numpy()
        scale = np.abs(gb).max(axis=-1, keepdims=True) if gb.ndim > 1 else np.abs(gb).max()
        assert np.all(np.abs(ga - gb) <= 1e-8 * scale + 1e-300), (ga, gb)


@pytest.mark.parametrize("precision", ["fp64", "fp64_reduced"])
def test_mot_coefficient_gradients_vs_central_fd(mol, gpu, precision):
    from molmot_b200.autograd import mot_coefficients
    ref, det, s0, B, kdir, pol = _sets(mol, 4, 3)
    f, p, b, freq, s0b = _params(ref, det, s0, B, gpu)
    k, beta = mot_coefficients(mol, kdir, pol, freq, s0b, b, precision=precision)
    gk = torch.autograd.grad(k.sum(), [f, p, b], retain_graph=True)
    gbeta = torch.autograd.grad(beta.sum(), [f, p, b])

    def kb(det_, s0_, B_):
        with torch.no_grad():
            _, _, _, fr, s0bb = _params(ref, det_, s0_, B_, gpu)
            bb = torch.tensor(B_, dtype=torch.float64, device=gpu)
            kk, be = mot_coefficients(mol, kdir, pol, fr, s0bb, bb, precision=precision)
        return kk.cpu().numpy(), be.cpu().numpy()

    for which, base in [(0, det), (1, s0), (2, B)]:
        for idx in np.ndindex(base.shape[1:] if base.ndim > 1 else ()):
            # h = 1e-4 relative; for B' 1e-3: a 1e-4 step of B' moves the transition
            # frequencies by ~100 Hz, where the FP64 model itself resolves omega = Es_e - Es_g
            # only to its 0.0625 Hz ulp, so that difference quotient carries ~3e-5 of
            # rounding noise (the dense torch model shows the same)
            h = (1e-3 if which == 2 else 1e-4) * np.abs(base[(slice(None),) + idx])
            args_p = [det.copy(), s0.copy(), B.copy()]
            args_m = [det.copy(), s0.copy(), B.copy()]
            args_p[which][(slice(None),) + idx] += h
            args_m[which][(slice(None),) + idx] -= h
            kp, bp = kb(*args_p)
            km, bm = kb(*args_m)
            if which == 0:
                # a detuning enters as the absolute frequency ref + det (~4.3e14 Hz, ulp
                # 0.0625 Hz): divide by the step the frequencies actually took
                i0 = idx[0]
                h = ((ref[i0] + args_p[0][:, i0]) - (ref[i0] + args_m[0][:, i0])) / 2
            fd_k = (kp - km) / (2 * h)
            fd_b = (bp - bm) / (2 * h)
            ad_k = gk[which].cpu().numpy()[(slice(None),) + idx]
            ad_b = gbeta[which].cpu().numpy()[(slice(None),) + idx]
            # relative to the largest sensitivity of each coefficient in the set
            sk = np.max(np.abs(gk[which].cpu().numpy().reshape(4, -1) * base.reshape(4, -1)), axis=1)
            sb = np.max(np.abs(gbeta[which].cpu().numpy().reshape(4, -1) * base.reshape(4, -1)), axis=1)
            scale = np.abs(base[(slice(None),) + idx])
            assert np.all(np.abs(fd_k - ad_k) * scale <= 1e-5 * sk), (which, idx)
            assert np.all(np.abs(fd_b - ad_b) * scale <= 1e-5 * sb), (which, idx)


def test_adjoint_forward_equals_force_batch(mol, gpu):
    from molmot_b200.engine import BeamSets, force_batch, force_adjoint, pack_for
    g = golden("random_points.npz")
    ns, npts = int(g["n_sets"]), int(g["n_pts"])
    sel = lambda a: a.reshape(ns, npts, *a.shape[1:])[:, 0]
    bs = BeamSets(sel(g["kdir"]), sel(g["freq"]), sel(g["pol"]), sel(g["s0"]), sel(g["B"]))
    F, G = force_adjoint(pack_for(mol), bs, g["v"], g["z"], points_per_set=npts)
    F2 = force_batch(pack_for(mol), bs, g["v"], g["z"], points_per_set=npts)["F"]
    # same rates, matrix and elimination; the force maps split a point over 2
    # lanes and the adjoint over 4, so the back-substitution and normalisation
    # sums associate differently: equal to rounding
    assert float((F - F2).abs().max()) <= 1e-14 * float(F2.abs().max())
    assert G.shape == (ns * npts, 17)


def test_reduced_adjoint_forward_equals_reduced_force(mol, gpu):
    import bench
    from molmot_b200.engine import BeamSets, force_batch, force_adjoint, pack_for
    bs = BeamSets(*bench.make_params(mol, 16, 7))
    v = np.linspace(-10, 10, 24)
    z = np.linspace(-1e-2, 1e-2, 20)
    F, G = force_adjoint(pack_for(mol), bs, v, z, grid=True, precision="fp64_reduced")
    F2 = force_batch(pack_for(mol), bs, v, z, grid=True, precision="fp64_reduced")["F"]
    assert torch.equal(F, F2.reshape(-1))
    Fp, Gp = force_adjoint(pack_for(mol), bs, v, z, grid=True, precision="fp64")
    scale = Gp.view(16, -1, 17).abs().amax(dim=1, keepdim=True)
    err = ((G - Gp).view(16, -1, 17).abs() / scale).nan_to_num(0.0)
    assert float(err.max()) < 1e-9


@pytest.mark.parametrize("n_g,n_e", [(4, 2), (7, 3), (9, 4)])
def test_reduced_adjoint_smaller_molecules(gpu, n_g, n_e):
    from molmot_b200.engine import BeamSets, MoleculePack, force_adjoint
    from molmot_b200.molecules.synthetic import dc_beams_for, synthetic_molecule
    m = synthetic_molecule(n_g, n_e, 100 + n_g)
    kd, fr, po, s0 = dc_beams_for(m)
    pk = MoleculePack(m)
    bs = BeamSets(kd[None], fr[None], po[None], s0[None], [0.2])
    v = np.linspace(-10, 10, 33)
    z = np.linspace(-1e-2, 1e-2, 29)
    Fr, Gr = force_adjoint(pk, bs, v, z, grid=True, precision="fp64_reduced")
    Fp, Gp = force_adjoint(pk, bs, v, z, grid=True, precision="fp64")
    assert float((Fr - Fp).abs().max()) <= 1e-12 * float(Fp.abs().max())
    scale = Gp.abs().amax(dim=0)
    assert float(((Gr - Gp).abs() / scale).nan_to_num(0.0).max()) < 1e-9


def test_reduced_adjoint_invalid_set_runs_elimination(mol, gpu):
    """A set whose beams are all pi leaves ground state 11 unpumped: the
    batch runs the elimination adjoint, bit for bit."""
    import bench
    from molmot_b200.engine import BeamSets, force_adjoint, pack_for
    kdir, freq, pol, s0, B = bench.make_params(mol, 3, 11)
    pol = pol.copy()
    pol[1] = 1
    bs = BeamSets(kdir, freq, pol, s0, B)
    v = np.linspace(-5, 5, 9)
    z = np.linspace(-5e-3, 5e-3, 7)
    Fr, Gr = force_adjoint(pack_for(mol), bs, v, z, grid=True, precision="fp64_reduced")
    Fp, Gp = force_adjoint(pack_for(mol), bs, v, z, grid=True, precision="fp64")
    assert torch.equal(Fr, Fp) and torch.equal(Gr.nan_to_num(7.0), Gp.nan_to_num(7.0))


def test_adjoint_rejects_fp32(mol, gpu):
    from molmot_b200.engine import BeamSets, force_adjoint, pack_for
    g = golden("random_points.npz")
    bs = BeamSets(g["kdir"][:1], g["freq"][:1], g["pol"][:1], g["s0"][:1], g["B"][:1])
    with pytest.raises(ValueError):
        force_adjoint(pack_for(mol), bs, g["v"][:4], g["z"][:4], precision="fp32")


@pytest.mark.parametrize("precision", ["fp64", "fp64_reduced"])
def test_mot_coefficient_gradients_at_config_scale(mol, gpu, precision):
    """Gradients of k and beta (33-point stencils) for 32 of the 1024
    parameter sets of the differentiation workload (bench.py: every 32nd set
    of make_params(mol, 1024, SEED + 7)), against FP64 torch autograd of the
    same coefficients through the dense restatement: 1e-8 of each set's
    largest gradient component, per coefficient and parameter group."""
    import bench
    from molmot_b200.autograd import mot_coefficients, stencil_weights
    from oracle import torch_dense as td
    kdir, freq, pol, s0, B = bench.make_params(mol, 1024, bench.SEED + 7)
    idx = np.arange(0, 1024, 32)
    kdir, freq, pol, s0, B = kdir[idx], freq[idx], pol[idx], s0[idx], B[idx]
    ref = freq[:, ::2].copy()  # 4 frequencies (each shared by a +z/-z pair)
    det0 = np.zeros_like(ref)
    s00 = s0[:, ::2].copy()

    def leaves(dev):
        f = torch.tensor(det0, dtype=torch.float64, device=dev, requires_grad=True)
        p = torch.tensor(s00, dtype=torch.float64, device=dev, requires_grad=True)
        b = torch.tensor(B, dtype=torch.float64, device=dev, requires_grad=True)
        fr = (torch.as_tensor(ref, dtype=torch.float64, device=dev) + f).repeat_interleave(2, 1)
        return f, p, b, fr, p.repeat_interleave(2, 1)

    f1, p1, b1, fr1, s01 = leaves(gpu)
    k1, be1 = mot_coefficients(mol, kdir, pol, fr1, s01, b1, precision=precision)
    g1 = [torch.autograd.grad(c.sum(), [f1, p1, b1], retain_graph=True) for c in (k1, be1)]
    # the dense restatement on the same stencils
    n, n_sets = 33, len(idx)
    zs = np.linspace(-0.3e-3, 0.3e-3, n)
    vs = np.linspace(-0.1, 0.1, n)
    v = np.tile(np.concatenate([np.zeros(n), vs]), n_sets)
    z = np.tile(np.concatenate([zs, np.zeros(n)]), n_sets)
    f2, p2, b2, fr2, s02 = leaves("cpu")
    F2 = td.force(mol, kdir, pol, fr2, s02, b2, v, z, 2 * n).view(n_sets, 2 * n)
    k2 = -(F2[:, :n] * torch.as_tensor(stencil_weights(zs))).sum(1)
    be2 = -(F2[:, n:] * torch.as_tensor(stencil_weights(vs))).sum(1) / mol.mass
    assert np.allclose(k1.detach().cpu().numpy(), k2.detach().numpy(), rtol=1e-9, atol=0)
    assert np.allclose(be1.detach().cpu().numpy(), be2.detach().numpy(), rtol=1e-9, atol=0)
    g2 = [torch.autograd.grad(c.sum(), [f2, p2, b2], retain_graph=True) for c in (k2, be2)]
    for ga_all, gb_all in zip(g1, g2):
        for ga, gb in zip(ga_all, gb_all):
            ga, gb = ga.cpu().numpy().reshape(n_sets, -1), gb.numpy().reshape(n_sets, -1)
            scale = np.abs(gb).max(axis=1, keepdims=True)
            assert np.all(np.abs(ga - gb) <= 1e-8 * scale), float((np.abs(ga - gb) / scale).max())
