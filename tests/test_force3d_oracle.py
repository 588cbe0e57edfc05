"""The 3D oracle (oracle/force3d.py, a numpy restatement of the reference's
rate_eq_force_3d and leapfrog) against the reference's own outputs on
synthetic molecules with a non-degenerate ground Zeeman spectrum
(tests/golden/force3d_reference.npz, written by make_golden.py force3d by
running molmot/mot/simulator_3d.py:168-365 and :443-504).  There the 3D force
is a well-posed function of the inputs, so the restatement must reproduce the
reference to rounding: 1e-12 of max |F| (forces, rates, populations) and of
the trajectory's extent."""
import numpy as np
import pytest

from conftest import golden

TOL = 1e-12


def _mol(g, i):
    from molmot_b200.molecules.synthetic import synthetic_molecule
    return synthetic_molecule(int(g[f"m{i}_ng"]), int(g[f"m{i}_ne"]), int(g[f"m{i}_seed"]))


def _beams(g, i):
    return tuple(g[f"m{i}_{k}"] for k in ("khat", "freq", "q", "s0", "radius"))


@pytest.mark.parametrize("i", [0, 1, 2])
def test_oracle_force3d_matches_reference(i):
    from oracle import force3d as o3
    g = golden("force3d_reference.npz")
    m = _mol(g, i)
    kh, fq, q, s0, rad = _beams(g, i)
    B = float(g[f"m{i}_B"])
    r, v = g[f"m{i}_r"], g[f"m{i}_v"]
    out = [o3.force3d(m, kh, fq, q, s0, rad, r[j], v[j], B) for j in range(len(r))]
    F = np.array([o[0] for o in out])
    R = np.array([o[1] for o in out])
    P = np.array([o[2] for o in out])
    assert np.abs(F - g[f"m{i}_F"]).max() <= TOL * np.abs(g[f"m{i}_F"]).max()
    assert np.abs(R - g[f"m{i}_R"]).max() <= TOL * np.abs(g[f"m{i}_R"]).max()
    assert np.abs(P - g[f"m{i}_P"]).max() <= TOL


@pytest.mark.parametrize("i", [0, 1, 2])
def test_oracle_leapfrog_matches_reference(i):
    from oracle import force3d as o3
    g = golden("force3d_reference.npz")
    m = _mol(g, i)
    B = float(g[f"m{i}_B"])
    R0, V0 = g[f"m{i}_r0"], g[f"m{i}_v0"]
    for j in range(len(R0)):
        _, R, V = o3.leapfrog3d(m, _beams(g, i), B, R0[j], V0[j], float(g[f"m{i}_t_max"]),
                                float(g[f"m{i}_dt"]))
        Rg, Vg = g[f"m{i}_traj_r"][j], g[f"m{i}_traj_v"][j]
        assert R.shape == Rg.shape
        assert np.abs(R - Rg).max() <= TOL * np.abs(Rg).max()
        assert np.abs(V - Vg).max() <= 1e-10 * np.abs(Vg).max()


def test_reference_sroh_spread_is_recorded():
    """The SrOH 3D model is ill-posed (6 + 6 degenerate ground Zeeman
    clusters): the reference's own force moves by percents under 1e-15
    perturbations of the matrix it diagonalises; the GPU tolerance for SrOH
    is that recorded spread."""
    g = golden("force3d_reference.npz")
    s = g["sroh_spread"]
    assert s.shape == (int(golden("force3d_golden.npz")["n_cases"]),)
    assert np.all(s > 1e-3)


@pytest.mark.parametrize("i", [0, 2])
def test_torch_restatement_matches_reference_and_fd(i):
    """oracle/torch_dense3d.py (the autograd checker of the 3D tangents)
    reproduces the reference's 3D force on the non-degenerate molecules, and
    its autograd derivatives agree with central differences of the numpy
    oracle (with respect to position, velocity, a beam frequency, a
    saturation parameter and B')."""
    import torch
    from oracle import force3d as o3
    from oracle import torch_dense3d as td3
    g = golden("force3d_reference.npz")
    m = _mol(g, i)
    kh, fq, q, s0, rad = _beams(g, i)
    B = float(g[f"m{i}_B"])
    r = torch.tensor(g[f"m{i}_r"][:16], dtype=torch.float64)
    v = torch.tensor(g[f"m{i}_v"][:16], dtype=torch.float64)
    F, R, P = td3.force3d(m, kh, fq, q, s0, rad, r, v, B)
    Fg = g[f"m{i}_F"][:16]
    assert np.abs(F.numpy() - Fg).max() <= 1e-12 * np.abs(Fg).max()
    # derivatives at one point
    j = 3
    rr = r[j:j + 1].clone().requires_grad_(True)
    vv = v[j:j + 1].clone().requires_grad_(True)
    fqt = torch.tensor(fq, requires_grad=True)
    s0t = torch.tensor(s0, requires_grad=True)
    Bt = torch.tensor(B, dtype=torch.float64, requires_grad=True)
    Fz = td3.force3d(m, kh, fqt, q, s0t, rad, rr, vv, Bt)[0][0, 2]
    gr, gv, gf, gs, gB = torch.autograd.grad(Fz, [rr, vv, fqt, s0t, Bt])
    base = lambda **kw: o3.force3d(m, kw.get("kh", kh), kw.get("fq", fq), q, kw.get("s0", s0), rad,
                                   kw.get("r", r[j].numpy()), kw.get("v", v[j].numpy()),
                                   kw.get("B", B))[0][2]

    def cd(key, x0, h, idx=None):
        xp, xm = np.array(x0, dtype=float), np.array(x0, dtype=float)
        if idx is None:
            xp, xm = x0 + h, x0 - h
        else:
            xp[idx] += h
            xm[idx] -= h
        return (base(**{key: xp}) - base(**{key: xm})) / (2 * h)

    # central differences carry ~1e-4 of truncation and rounding noise here (the
    # transition frequencies round to 1/16 Hz at 4.3e14 Hz): 2e-3 relative
    close = lambda fd, ad: abs(fd - ad) <= 2e-3 * abs(ad)
    for c in range(3):
        assert close(cd("r", r[j].numpy(), 1e-6, c), gr[0, c].item()), ("r", c)
        assert close(cd("v", v[j].numpy(), 1e-3, c), gv[0, c].item()), ("v", c)
    b = 2
    assert close(cd("fq", fq, 2.0e4, b), gf[b].item())
    assert close(cd("s0", s0, 1e-4 * s0[b], b), gs[b].item())
    assert close(cd("B", B, 1e-4 * B), gB.item())
