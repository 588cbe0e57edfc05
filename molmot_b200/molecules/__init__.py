"""Molecule containers and loaders (the hot path's input format)."""
from .sroh import (MolecularData, load_sroh_from_julia, SROH_DATA_DIR, GAMMA_RAD,
                   GAMMA_HZ, K_WAVE, LAMBDA_M, MASS_KG)

__all__ = ["MolecularData", "load_sroh_from_julia", "SROH_DATA_DIR", "GAMMA_RAD",
           "GAMMA_HZ", "K_WAVE", "LAMBDA_M", "MASS_KG"]
