"""ctypes binding of libmolmot_b200.so (the C ABI declared in include/molmot_b200.h).

The shared library is built in-tree by ``molmot_b200/csrc/Makefile`` into
``molmot_b200/lib/``.  There is no fallback: if the library is missing or a
call fails, a RuntimeError is raised.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmolmot_b200.so")

MM_MAX_GROUND = 48
MM_MAX_EXCITED = 16
MM_MAX_BEAMS = 32
MM_PREC_FP64 = 0
MM_PREC_FP32_REFINE = 1
MM_PREC_FP64_REDUCED = 2
MM_LAYOUT_POINTS = 0
MM_LAYOUT_GRID = 1
MM_ST_PIVOT = 1
MM_ST_NONFINITE = 2
MM_ST_ZERO_POP = 4
MM_ST_DEGENERATE = 8

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p


class MolDesc(ctypes.Structure):
    _fields_ = [("n_ground", ctypes.c_int32), ("n_excited", ctypes.c_int32),
                ("energies", _vp), ("d_squared", _vp), ("zeeman_z_diag", _vp),
                ("Gamma", ctypes.c_double), ("k", ctypes.c_double), ("mass", ctypes.c_double),
                ("zeeman_ground_re", _vp), ("zeeman_ground_im", _vp),
                ("zeeman_excited_z", _vp), ("tdm_abs", _vp)]


class BeamDesc(ctypes.Structure):
    _fields_ = [("n_beams", ctypes.c_int32), ("kdir", _vp), ("freq", _vp), ("pol", _vp),
                ("s0", _vp), ("b_gradient", _vp), ("gamma_eff", ctypes.c_double),
                ("khat", _vp), ("radius", _vp)]


class BatchOpts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("layout", ctypes.c_int32),
                ("points_per_set", ctypes.c_int64), ("nv", ctypes.c_int64),
                ("nz", ctypes.c_int64), ("hbar", ctypes.c_double),
                ("uniform_fallback", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class TrajOpts(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int32), ("n_avg", ctypes.c_int32), ("n_steps", ctypes.c_int64),
                ("dt", ctypes.c_double), ("r_escape", ctypes.c_double), ("i_eq", ctypes.c_int64),
                ("precision", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("hbar", ctypes.c_double)]


MM_TGRAD_MAX_PAR = 8


class TgradOpts(ctypes.Structure):
    _fields_ = [("n_steps", ctypes.c_int64), ("step0", ctypes.c_int64),
                ("ckpt_every", ctypes.c_int64), ("dt", ctypes.c_double),
                ("r_escape", ctypes.c_double), ("hbar", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("kicks", ctypes.c_int32), ("n_par", ctypes.c_int32),
                ("freq_par", ctypes.c_int32 * MM_MAX_BEAMS), ("s0_par", ctypes.c_int32 * MM_MAX_BEAMS),
                ("bprime_par", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class T3gradOpts(ctypes.Structure):
    _fields_ = [("n_steps", ctypes.c_int64), ("step0", ctypes.c_int64),
                ("ckpt_every", ctypes.c_int64), ("dt", ctypes.c_double),
                ("r_escape", ctypes.c_double), ("hbar", ctypes.c_double), ("gap_tol", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("kicks", ctypes.c_int32), ("n_par", ctypes.c_int32),
                ("freq_par", ctypes.c_int32 * MM_MAX_BEAMS), ("s0_par", ctypes.c_int32 * MM_MAX_BEAMS),
                ("bprime_par", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class UnevenOpts(ctypes.Structure):
    _fields_ = [("warps_per_cta", ctypes.c_int32 * 3), ("chunk_groups", ctypes.c_int32)]


#: every symbol include/molmot_b200.h declares, with (restype, argtypes)
SIGNATURES = {
    "mm_last_error": (ctypes.c_char_p, []),
    "mm_version": (ctypes.c_char_p, []),
    "mm_pack_create": (ctypes.c_int, [ctypes.POINTER(MolDesc), ctypes.POINTER(_vp)]),
    "mm_pack_destroy": (ctypes.c_int, [_vp]),
    "mm_beams_create": (ctypes.c_int, [ctypes.POINTER(BeamDesc), ctypes.c_int32, ctypes.POINTER(_vp)]),
    "mm_beams_destroy": (ctypes.c_int, [_vp]),
    "mm_force_batch": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int64,
                                      ctypes.POINTER(BatchOpts), _vp, _vp, _vp, _vp, _vp]),
    "mm_traj1d_run": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_double,
                                     ctypes.c_int64, ctypes.c_double, ctypes.POINTER(BatchOpts),
                                     _vp, _vp, _vp, _vp, _vp, _vp]),
    "mm_traj_run": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(TrajOpts), _vp, _vp, ctypes.c_int64,
                                   _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mm_force_adjoint": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int64,
                                        ctypes.POINTER(BatchOpts), _vp, _vp, _vp]),
    "mm_force3d_batch": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int64,
                                        ctypes.c_double, _vp, _vp, _vp, _vp, _vp]),
    "mm_traj3d_run": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int64,
                                     ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int32, ctypes.c_uint64, ctypes.c_double,
                                     _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mm_beams_view": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(_vp)]),
    "mm_bank_create": (ctypes.c_int, [ctypes.POINTER(MolDesc), ctypes.c_int32, ctypes.POINTER(_vp)]),
    "mm_bank_destroy": (ctypes.c_int, [_vp]),
    "mm_uneven_plan_create": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64),
                                             ctypes.POINTER(UnevenOpts), ctypes.POINTER(_vp)]),
    "mm_uneven_plan_destroy": (ctypes.c_int, [_vp]),
    "mm_uneven_force": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int32,
                                       ctypes.c_int32, _vp, _vp, _vp, _vp]),
    "mm_uneven_force_static": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_int64),
                                              ctypes.POINTER(UnevenOpts), _vp, _vp, ctypes.c_double,
                                              ctypes.c_int32, _vp, _vp, _vp, _vp]),
    "mm_ensemble_stats": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64, _vp, ctypes.c_int32,
                                         ctypes.c_double, _vp, _vp]),
    "mm_histogram": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int32, _vp, _vp]),
    "mm_traj3d_grad_run": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(T3gradOpts), ctypes.c_int64, _vp, _vp,
                                          _vp, _vp, _vp, _vp, _vp]),
    "mm_traj3d_grad_checkpoints": (ctypes.c_int64, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]),
    "mm_traj_grad_run": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(TgradOpts), ctypes.c_int64, _vp, _vp,
                                        _vp, _vp]),
}

_lib = None


def load():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"molmot_b200: {LIB_PATH} is missing; build it with "
                "`make -C molmot_b200/csrc` (or __graft_entry__.build()).  "
                "There is no CPU fallback.")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    msg = load().mm_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed (rc={rc}): {last_error()}")
