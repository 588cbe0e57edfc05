"""Size-independent properties on the full batched-map workload (4096
seeded parameter sets x 256 x 256 grid = 2.68e8 points), where the oracle is
too slow to compare point by point:

* the force is linear in hbar and the scattering rate independent of it,
  bit for bit (doubling hbar is exact in binary);
* permuting the parameter sets permutes the maps, bit for bit;
* two runs give the same bits;
* the chunked host path (force_maps_to_host) equals the device path;
* the FP64-reduced form agrees with the plain elimination to 1e-12 of max|F|
  on every set, and the FP32 form to 1e-6.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N_SETS, NV, NZ = 4096, 256, 256


@pytest.fixture(scope="module")
def workload(mol, gpu):
    import bench
    from molmot_b200.engine import BeamSets, MoleculePack
    params = bench.make_params(mol, N_SETS, bench.SEED)
    v = torch.as_tensor(np.linspace(-10, 10, NV), device=gpu)
    z = torch.as_tensor(np.linspace(-1e-2, 1e-2, NZ), device=gpu)
    return MoleculePack(mol), params, BeamSets(*params), v, z


def _maps(pack, bs, v, z, precision, hbar=None, want_R=False):
    from molmot_b200.engine import force_batch
    return force_batch(pack, bs, v, z, grid=True, precision=precision, hbar=hbar, want_pop=False,
                       want_R=want_R, want_status=False)


def test_hbar_linearity_and_determinism(workload):
    pack, _, bs, v, z = workload
    a = _maps(pack, bs, v, z, "fp32", hbar=1.0545718e-34, want_R=True)
    b = _maps(pack, bs, v, z, "fp32", hbar=2 * 1.0545718e-34, want_R=True)
    assert torch.equal(2 * a["F"], b["F"])
    assert torch.equal(a["R"], b["R"])
    c = _maps(pack, bs, v, z, "fp32", hbar=1.0545718e-34, want_R=True)
    assert torch.equal(a["F"], c["F"])
    assert torch.isfinite(a["F"]).all()


def test_set_permutation(workload):
    from molmot_b200.engine import BeamSets
    pack, params, bs, v, z = workload
    perm = np.random.default_rng(1).permutation(N_SETS)
    bs_p = BeamSets(*(p[perm] for p in params))
    a = _maps(pack, bs, v, z, "fp32")["F"]
    b = _maps(pack, bs_p, v, z, "fp32")["F"]
    assert torch.equal(a[torch.as_tensor(perm, device=a.device)], b)


def test_host_path_equals_device_path(workload):
    from molmot_b200.engine import force_maps_to_host
    pack, _, bs, v, z = workload
    dev = _maps(pack, bs, v, z, "fp32")["F"].cpu()
    host = force_maps_to_host(pack, bs, v, z, precision="fp32", chunk_sets=256)
    assert torch.equal(dev, host)


def test_forms_agree_on_every_set(workload):
    pack, _, bs, v, z = workload
    plain = _maps(pack, bs, v, z, "fp64")["F"]
    scale = plain.abs().amax(dim=(1, 2))
    red = _maps(pack, bs, v, z, "fp64_reduced")["F"]
    assert float(((red - plain).abs().amax(dim=(1, 2)) / scale).max()) < 1e-12
    del red
    f32 = _maps(pack, bs, v, z, "fp32")["F"]
    assert float(((f32 - plain).abs().amax(dim=(1, 2)) / scale).max()) < 1e-6
