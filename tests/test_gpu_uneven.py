"""Uneven batches of synthetic molecules (n_ground 4..48, n_excited 4..16)
against the CPU oracle, persistent vs one-CTA-per-item launches, graph replay
and the autotuner."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch(gpu):
    from molmot_b200.uneven import MoleculeBank, UnevenBatch, make_uneven_workload
    from molmot_b200.engine import BeamSets
    mols, counts, (kdir, freq, pol, s0), B, v, z = make_uneven_workload(
        n_mol=30, seed=5, min_pts=5, max_pts=70)
    bank = MoleculeBank(mols)
    bs = BeamSets(kdir, freq, pol, s0, B)
    ub = UnevenBatch(bank, counts, bs)
    return mols, counts, (kdir, freq, pol, s0), B, v, z, ub


def test_uneven_vs_oracle(batch):
    from oracle import rate_eq as orc
    mols, counts, (kdir, freq, pol, s0), B, v, z, ub = batch
    out = ub.force(v, z)
    F = out["F"].cpu().numpy()
    off = np.concatenate([[0], np.cumsum(counts)])
    sizes = set()
    for m, mol in enumerate(mols):
        a, b = off[m], off[m + 1]
        Fo = orc.force_batch(mol, kdir[m:m + 1], freq[m:m + 1], pol[m:m + 1], s0[m:m + 1], B[m:m + 1],
                             v[a:b], z[a:b], want_pop=False)[0]
        scale = np.abs(Fo).max()
        assert np.abs(F[a:b] - Fo).max() <= 1e-10 * scale, (m, mol.n_ground, mol.n_excited)
        sizes.add((mol.n_ground > 16) + (mol.n_ground > 32))
    assert sizes == {0, 1, 2}  # every size class exercised
    assert np.all(out["status"].cpu().numpy() == 0)


def test_persistent_equals_per_item_and_graph(batch):
    mols, counts, beams, B, v, z, ub = batch
    a = ub.force(v, z, persistent=True)["F"].clone()
    b = ub.force(v, z, persistent=False)["F"].clone()
    assert torch.equal(a, b)
    g, out, vg, zg = ub.graph(v, z)
    out["F"].zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out["F"], a)


def test_autotune_keeps_results(batch):
    mols, counts, beams, B, v, z, ub = batch
    ref = ub.force(v, z)["F"].clone()
    w = ub.autotune(v, z, candidates=(2, 4), reps=1)
    assert len(w) == 3
    assert torch.equal(ub.force(v, z)["F"], ref)


def test_uneven_config_scale_sample_vs_oracle(gpu):
    """The full uneven workload of bench.py (2048 molecules, 64..4096 points
    each, seed 20261203) in one persistent call; per size class the molecules
    with the most points, ground states and excited states plus a random one
    against the CPU oracle at 1e-10 of each molecule's max |F|."""
    import bench
    from molmot_b200.engine import BeamSets
    from molmot_b200.uneven import MoleculeBank, UnevenBatch, make_uneven_workload, sample_molecules
    from oracle import rate_eq as orc
    mols, counts, (kdir, freq, pol, s0), B, v, z = make_uneven_workload(n_mol=2048, seed=bench.SEED)
    ub = UnevenBatch(MoleculeBank(mols), counts, BeamSets(kdir, freq, pol, s0, B))
    F = ub.force(torch.as_tensor(v, device=gpu), torch.as_tensor(z, device=gpu))["F"].cpu().numpy()
    ng = np.array([m.n_ground for m in mols])
    ne = np.array([m.n_excited for m in mols])
    pick = sample_molecules(ng, ne, counts)
    assert len(pick) == 12 and 48 in ng[pick] and int(counts.max()) in counts[pick]
    off = np.concatenate([[0], np.cumsum(counts)])
    for m in pick:
        a, b = off[m], off[m + 1]
        Fo = orc.force_batch(mols[m], kdir[m:m + 1], freq[m:m + 1], pol[m:m + 1], s0[m:m + 1],
                             B[m:m + 1], v[a:b], z[a:b], want_pop=False)[0]
        assert np.abs(F[a:b] - Fo).max() <= 1e-10 * np.abs(Fo).max(), (m, ng[m], ne[m])
