"""The CPU leg of bench.py (its reference arm and cpu_baseline): the
reference's own numba core, imported unchanged from the reference installed
in baseline/_ref, must give the C oracle's forces on a small grid.  Skipped
where that install is absent (the leg then runs the C oracle itself)."""
import os

import numpy as np
import pytest

from conftest import ROOT


@pytest.mark.skipif(not os.path.isdir(os.path.join(ROOT, "baseline", "_ref", "molmot")),
                    reason="the reference is not installed in baseline/_ref")
def test_reference_leg_matches_oracle(mol):
    import bench
    from oracle import rate_eq as orc
    cpu = bench.CpuForceMaps(mol)
    assert cpu.kind == "reference"
    kdir, freq, pol, s0, B = bench.make_params(mol, 3, bench.SEED)
    v = np.linspace(-10, 10, 7)
    z = np.linspace(-1e-2, 1e-2, 9)
    F = cpu(kdir, freq, pol, s0, B, v, z)
    Fo = orc.force_batch(mol, kdir, freq, pol, s0, B, v, z, grid=True, want_pop=False)[0]
    assert F.shape == Fo.shape
    assert np.array_equal(F, Fo)  # the oracle restates _rate_eq_core in its operation order
