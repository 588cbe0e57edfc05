"""mm_uneven_force_static (no plan, no allocation; work list and counters in
the library's fixed device array) against mm_uneven_force on the same batch,
on consecutive calls: the counters must be zeroed and the work list rewritten
by every call.  Collected last so it also runs after every other GPU test has
used the library; it passes alone in a fresh process as well."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative to the largest |F| of the batch, as the uneven-batch oracle test


def _batch(n_mol, seed, min_pts, max_pts, chunk_groups=8):
    from molmot_b200.engine import BeamSets
    from molmot_b200.uneven import MoleculeBank, UnevenBatch, make_uneven_workload
    mols, counts, (kdir, freq, pol, s0), B, v, z = make_uneven_workload(
        n_mol=n_mol, seed=seed, min_pts=min_pts, max_pts=max_pts)
    ub = UnevenBatch(MoleculeBank(mols), counts, BeamSets(kdir, freq, pol, s0, B),
                     chunk_groups=chunk_groups)
    dev = torch.device("cuda", 0)
    return ub, torch.as_tensor(v, device=dev), torch.as_tensor(z, device=dev)


def _nan_out(n, dev):
    return {"F": torch.full((n,), float("nan"), dtype=torch.float64, device=dev),
            "R": torch.full((n,), float("nan"), dtype=torch.float64, device=dev),
            "status": torch.full((n,), -1, dtype=torch.int32, device=dev)}


def test_static_matches_plan_on_consecutive_calls(gpu):
    a, va, za = _batch(30, 5, 5, 70)
    b, vb, zb = _batch(17, 9, 40, 400)
    ref_a = {k: t.clone() for k, t in a.force(va, za).items()}
    ref_b = {k: t.clone() for k, t in b.force(vb, zb).items()}
    torch.cuda.synchronize()
    outs_a = [_nan_out(a.n_points, va.device) for _ in range(2)]
    out_b = _nan_out(b.n_points, vb.device)
    # allocated up front; the calls themselves allocate nothing
    a.force_static(va, za, outs_a[0])
    a.force_static(va, za, outs_a[1])
    b.force_static(vb, zb, out_b)
    torch.cuda.synchronize()
    for out, ref in [(outs_a[0], ref_a), (outs_a[1], ref_a), (out_b, ref_b)]:
        scale = ref["F"].abs().max().item()
        assert torch.isfinite(out["F"]).all()
        assert (out["F"] - ref["F"]).abs().max().item() <= TOL * scale
        assert (out["R"] - ref["R"]).abs().max().item() <= TOL * ref["R"].abs().max().item()
        assert torch.equal(out["status"], ref["status"])


def test_static_refuses_oversize_batch(gpu):
    from molmot_b200.engine import BeamSets
    from molmot_b200.molecules.synthetic import dc_beams_for, synthetic_molecule
    from molmot_b200.uneven import MoleculeBank, UnevenBatch
    mol = synthetic_molecule(8, 4, 3)
    kdir, freq, pol, s0 = (x[None] for x in dc_beams_for(mol))
    # one molecule of the n_g <= 16 class, chunk_groups 1: 8 points per work item,
    # so 43,681 items (one above the fixed array's capacity) need 349,448 points
    n = 43681 * 8
    ub = UnevenBatch(MoleculeBank([mol]), [n], BeamSets(kdir, freq, pol, s0, np.array([0.2])),
                     chunk_groups=1)
    g = torch.Generator(device="cpu").manual_seed(4)
    v = (torch.rand(n, generator=g, dtype=torch.float64) * 20 - 10).to("cuda:0")
    z = (torch.rand(n, generator=g, dtype=torch.float64) * 2e-2 - 1e-2).to("cuda:0")
    out = {"F": torch.zeros(n, dtype=torch.float64, device="cuda:0")}
    with pytest.raises(RuntimeError, match="43680"):
        ub.force_static(v, z, out)
    # one item fewer fits
    ub2 = UnevenBatch(MoleculeBank([mol]), [43680 * 8], BeamSets(kdir, freq, pol, s0, np.array([0.2])),
                      chunk_groups=1)
    m = 43680 * 8
    ub2.force_static(v[:m], z[:m], {"F": out["F"][:m]})
    ref = ub2.force(v[:m], z[:m])["F"]
    torch.cuda.synchronize()
    assert (out["F"][:m] - ref).abs().max().item() <= TOL * ref.abs().max().item()
