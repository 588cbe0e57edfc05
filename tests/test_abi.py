"""The C-ABI library: it loads, exports every symbol include/molmot_b200.h
declares, and rejects bad arguments before touching the GPU (no compute
calls here, so this runs without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "molmot_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"MM_API\s+(?:const\s+)?\w+\s*\*?\s*(mm_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["mm_pack_create", "mm_beams_create", "mm_force_batch", "mm_traj1d_run",
              "mm_last_error"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    from molmot_b200 import _lib
    L = _lib.load()
    for s in declared_symbols():
        assert hasattr(L, s), s
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"


def test_version_and_error_strings():
    from molmot_b200 import _lib
    L = _lib.load()
    assert b"sm_100a" in L.mm_version()
    assert isinstance(L.mm_last_error(), bytes)


def test_pack_create_rejects_bad_sizes():
    from molmot_b200 import _lib
    L = _lib.load()
    d = _lib.MolDesc()
    E = np.zeros(2)
    d.n_ground, d.n_excited = 0, 1
    d.energies = d.d_squared = d.zeeman_z_diag = ctypes.c_void_p(E.ctypes.data)
    d.Gamma, d.k, d.mass = 1.0, 1.0, 1.0
    h = ctypes.c_void_p()
    assert L.mm_pack_create(ctypes.byref(d), ctypes.byref(h)) < 0
    assert b"out of range" in L.mm_last_error()
    assert not h.value


def test_beams_create_rejects_bad_polarisation():
    from molmot_b200 import _lib
    L = _lib.load()
    kd = np.ones(2)
    pol = np.array([0, 5], dtype=np.int32)
    d = _lib.BeamDesc()
    d.n_beams = 2
    d.kdir = d.freq = d.s0 = d.b_gradient = ctypes.c_void_p(kd.ctypes.data)
    d.pol = ctypes.c_void_p(pol.ctypes.data)
    h = ctypes.c_void_p()
    assert L.mm_beams_create(ctypes.byref(d), 1, ctypes.byref(h)) < 0
    assert b"polarization" in L.mm_last_error()


def test_force_batch_rejects_null_handles():
    from molmot_b200 import _lib
    L = _lib.load()
    o = _lib.BatchOpts()
    rc = L.mm_force_batch(None, None, None, None, 1, ctypes.byref(o), None, None, None, None, None)
    assert rc < 0
    assert b"null" in L.mm_last_error()


def test_option_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror of a header struct has the C compiler's size and
    field offsets (gcc on a probe that includes the header)."""
    import shutil
    import subprocess
    from molmot_b200 import _lib
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    pairs = [("mm_mol_desc", _lib.MolDesc), ("mm_beam_desc", _lib.BeamDesc),
             ("mm_batch_opts", _lib.BatchOpts), ("mm_traj_opts", _lib.TrajOpts),
             ("mm_uneven_opts", _lib.UnevenOpts), ("mm_tgrad_opts", _lib.TgradOpts),
             ("mm_t3grad_opts", _lib.T3gradOpts)]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "molmot_b200.h"', "int main(void) {"]
    for cname, cls in pairs:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        a, b, c = ln.split()
        got[(a, b)] = int(c)
    for cname, cls in pairs:
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
