"""molmot_b200 -- B200-native batched rate-equation steady-state force.

A drop-in for the hot path of molmot (the multi-level rate-equation MOT
force, its force scans and the trajectory ensembles it drives), computed by
hand-written sm_100a CUDA kernels behind a C ABI (include/molmot_b200.h,
built into molmot_b200/lib/libmolmot_b200.so).  PyTorch provides device
memory, streams and autograd.
"""
__version__ = "0.1.0"

from .constants import hbar, HBAR_JIT  # noqa: F401
from .molecules import MolecularData, load_sroh_from_julia  # noqa: F401
from .fields import LaserBeam, make_dc_mot_beams, make_rf_mot_beams  # noqa: F401


def has_cuda() -> bool:
    """True when a CUDA device is visible and the native library is built."""
    try:
        import torch
        from . import _lib
        if not torch.cuda.is_available():
            return False
        _lib.load()
        return True
    except Exception:
        return False
