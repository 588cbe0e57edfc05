"""CaF and CaOH molecules from tests/golden/molecules_golden.npz (built there
by the reference's own Hamiltonian code, tests/golden/make_golden.py)."""
import numpy as np

from conftest import golden

NAMES = ("caf", "caoh")


def load(name):
    from molmot_b200.molecules import MolecularData
    g = golden("molecules_golden.npz")
    mol = MolecularData(energies=g[f"{name}_energies"], tdm=g[f"{name}_tdm"],
                        zeeman_x=g[f"{name}_zeeman_x"], zeeman_y=g[f"{name}_zeeman_y"],
                        zeeman_z=g[f"{name}_zeeman_z"], Gamma=float(g[f"{name}_Gamma"]),
                        k=float(g[f"{name}_k"]), mass=float(g[f"{name}_mass"]),
                        wavelength=float(g[f"{name}_wavelength"]), n_ground=int(g[f"{name}_n_ground"]),
                        n_excited=int(g[f"{name}_n_excited"]),
                        n_states=int(g[f"{name}_n_ground"]) + int(g[f"{name}_n_excited"]))
    return mol, g


def points(g, name):
    """Per-point rows of the seeded random points, and the per-set beam arrays."""
    ns, npt = int(g[f"{name}_n_sets"]), int(g[f"{name}_n_pts"])
    row = lambda k: g[f"{name}_pts_{k}"]
    per_set = lambda a: a.reshape(ns, npt, *a.shape[1:])[:, 0]
    sets = tuple(per_set(row(k)) for k in ("kdir", "freq", "pol", "s0", "B"))
    return ns, npt, sets, row("v"), row("z"), row("F"), row("p"), row("R")


def set_err(F, Fref, ns):
    F = np.asarray(F).reshape(ns, -1)
    Fref = np.asarray(Fref).reshape(ns, -1)
    return np.max(np.abs(F - Fref), axis=1) / np.max(np.abs(Fref), axis=1)
