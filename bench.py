#!/usr/bin/env python3
"""Benchmark: batched SrOH steady-state force maps (the batched-map workload).

Workload (per GPU, weak scaling): 4096 seeded parameter sets (4 detunings
U[-40, 0] MHz added to the SrOH transition references, per-frequency s0
log-uniform in [0.1, 10], B' U[5, 40] G/cm), each a 256 x 256 grid of
v in [-10, 10] m/s and z in [-10, 10] mm: 2.68e8 steady-state force
evaluations per step.  Synthetic inputs of exactly that shape (seed 20261203
+ rank).

value      : force evaluations/s of the FP32-bulk form (FP32 Lorentzians, FP64
             sums, populations from the FP64 solve of the excited-state chain),
             inputs resident, device-timed (CUDA events), max over ranks.
plain_fp64 : the same for the plain FP64 form on the same grid.
e2e        : the same metric through the public API with host arrays: per step
             the parameter sets and grid axes go host->device and the force
             maps come back device->host into page-locked memory, chunk by
             chunk, overlapped with the computation (inside the timed region).
roofline   : the force kernel against the measured FP64/FP32 FMA peaks of
             this GPU (the FMA probe of libmolmot_probe.so); algorithmic FLOPs
             per point of the form that runs (molmot_b200/flops.py).
cpu_baseline: the reference's own numba core (_rate_eq_core, from the reference
             installed in baseline/_ref) on all host cores, on a bounded sample
             of the same workload, plus a one-thread figure.

Output: three JSON lines -- every measurement (long), then the compact
evidence line (the other forms, accuracy, trajectories, adjoints, uneven
batch), then the headline.

`--impl reference` prints the CPU reference arm instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "16-level steady-state force evals/s and particle-steps/s: plain FP64 vs FP32+refine @1e-6"
N_SETS, NV, NZ = 4096, 256, 256
# dram__bytes_read.sum + dram__bytes_write.sum per point of force_reduced_kernel
# (FP32 form, grid layout, F only), from an ncu capture of a 512-set launch
TRAFFIC_PER_POINT = (416000 + 266039552) / (512 * 256 * 256)
SEED = 20261203


def make_params(mol, n_sets, seed):
    rng = np.random.default_rng(seed)
    E = mol.energies
    ref = np.array([E[15] - E[0], E[15] - E[0], E[15] - E[9], E[15] - E[9]])
    det = rng.uniform(-40e6, 0.0, (n_sets, 4))
    s0 = 10 ** rng.uniform(-1, 1, (n_sets, 4))
    B = rng.uniform(5, 40, n_sets) * 1e-2
    pols = np.array([2, 0, 2, 0])
    kdir = np.tile([1.0, -1.0], (n_sets, 4))
    freq = np.repeat(ref[None, :] + det, 2, axis=1)
    pol = np.tile(np.stack([pols, 2 - pols], 1).ravel(), (n_sets, 1)).astype(np.int32)
    s0b = np.repeat(s0, 2, axis=1)
    return kdir, freq, pol, s0b, B


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_figure(nbytes, ms):
    """Secondary HBM figure of the force kernel: algorithmic bytes per launch
    over its time, against the measured copy bandwidth of MEASURED_PEAKS.json
    (6.65 TB/s, an earlier measurement on this GPU type, if that file is absent)."""
    peak, src = 6650.0, "fallback"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, src = float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        pass
    gbs = nbytes / (ms * 1e-3) / 1e9
    return {"achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak, "peak_source": src}


def peak_probe(torch):
    """Measured FP64 and FP32 FMA throughput (TFLOP/s) of this GPU, from the
    FMA-chain probe in molmot_b200/lib/libmolmot_probe.so (a measurement aid
    built beside the product library, not part of its ABI)."""
    import ctypes
    path = os.path.join(ROOT, "molmot_b200", "lib", "libmolmot_probe.so")
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing; build it with make -C molmot_b200/csrc")
    L = ctypes.CDLL(path)
    L.fma_peak_probe.restype = ctypes.c_int
    L.fma_peak_probe.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    out = {}
    for which, name, iters in [(0, "fp64", 4096), (1, "fp32", 16384)]:
        best = 0.0
        for _ in range(3):
            ms, fl = ctypes.c_double(), ctypes.c_double()
            rc = L.fma_peak_probe(which, iters, ctypes.byref(ms), ctypes.byref(fl),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            if rc != 0:
                raise RuntimeError(f"fma_peak_probe failed (rc={rc})")
            best = max(best, fl.value / (ms.value * 1e-3) / 1e12)
        out[name] = best
    return out


REF_DIR = os.path.join(ROOT, "baseline", "_ref")


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


class CpuForceMaps:
    """CPU force maps of the batched-map workload for the CPU legs.

    kind "reference": the reference's numba core, molmot/obe/rate_equations_jit.py
    :18-145 (_rate_eq_core), imported unchanged from the reference installed in
    baseline/_ref, driven by a numba prange harness over the points of each
    set's (v, z) grid on every host core (numba's default thread count).
    kind "port": when baseline/_ref is absent, the C restatement of the same
    core (oracle/rate_eq_oracle.c) with one pthread per host core."""

    def __init__(self, mol):
        self.mol = mol
        self.E = np.ascontiguousarray(mol.energies, dtype=np.float64)
        self.d2 = np.ascontiguousarray(mol.d_squared, dtype=np.float64)
        self.zd = np.ascontiguousarray(mol.zeeman_z_diag, dtype=np.float64)
        if os.path.isdir(os.path.join(REF_DIR, "molmot")):
            os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(REF_DIR, ".numba_cache"))
            if REF_DIR not in sys.path:
                sys.path.insert(0, REF_DIR)
            import numba
            from numba import njit, prange
            from molmot.obe.rate_equations_jit import _rate_eq_core

            @njit(parallel=True)
            def grid(E, d2, zd, kdir, freq, pol, s0, B, v, z, Gamma, k, geff, n_g, n_e, out):
                nv, nz = v.shape[0], z.shape[0]
                per = nv * nz
                for i in prange(kdir.shape[0] * per):
                    s = i // per
                    r = i - s * per
                    iv = r // nz
                    out[i] = _rate_eq_core(E, d2, zd, kdir[s], freq[s], pol[s], s0[s], v[iv],
                                           z[r - iv * nz], B[s], Gamma, k, geff, n_g, n_e)[0]

            self.numba, self.grid, self.kind = numba, grid, "reference"
            self.what = ("the reference's _rate_eq_core (molmot/obe/rate_equations_jit.py:18-145), "
                         "unchanged from baseline/_ref, numba prange harness over points")
        else:
            from oracle import rate_eq as orc
            self.orc, self.kind = orc, "port"
            self.what = ("C restatement of _rate_eq_core (oracle/rate_eq_oracle.c), pthreads over "
                         "points (the reference install baseline/_ref is absent)")

    def threads(self):
        return self.numba.get_num_threads() if self.kind == "reference" else self.orc.max_threads()

    def set_threads(self, n):
        if self.kind == "reference":
            self.numba.set_num_threads(n)
        self._n = n

    def __call__(self, kdir, freq, pol, s0, B, v, z):
        """F [n_sets * nv * nz] of the grids; the reference wrapper's layout:
        polarisations as float64 (rate_equations_jit.py:155-159)."""
        m = self.mol
        if self.kind == "reference":
            out = np.empty(kdir.shape[0] * v.size * z.size)
            self.grid(self.E, self.d2, self.zd, np.ascontiguousarray(kdir, dtype=np.float64),
                      np.ascontiguousarray(freq, dtype=np.float64),
                      np.ascontiguousarray(pol, dtype=np.float64),
                      np.ascontiguousarray(s0, dtype=np.float64), np.ascontiguousarray(B, dtype=np.float64),
                      np.ascontiguousarray(v, dtype=np.float64), np.ascontiguousarray(z, dtype=np.float64),
                      float(m.Gamma), float(m.k), 1.0, int(m.n_ground), int(m.n_excited), out)
            return out
        return self.orc.force_batch(m, kdir, freq, pol, s0, B, v, z, grid=True, want_pop=False,
                                    n_threads=getattr(self, "_n", 0))[0]


def cpu_baseline(mol, n_sets_sample=1024):
    """The CPU leg of the force maps on the bench host: all cores on 1024 of the
    4096 parameter sets (6.7e7 points, about 10-20 s), and one thread on 8 sets."""
    cpu = CpuForceMaps(mol)
    kdir, freq, pol, s0, B = make_params(mol, n_sets_sample, SEED)
    v = np.linspace(-10, 10, NV)
    z = np.linspace(-1e-2, 1e-2, NZ)
    cpu(kdir[:1], freq[:1], pol[:1], s0[:1], B[:1], v[:4], z[:4])  # compile
    threads = cpu.threads()
    t0 = time.perf_counter()
    cpu(kdir, freq, pol, s0, B, v, z)
    dt = time.perf_counter() - t0
    n = n_sets_sample * NV * NZ
    one = 8
    cpu.set_threads(1)
    t1 = time.perf_counter()
    cpu(kdir[:one], freq[:one], pol[:one], s0[:one], B[:one], v, z)
    dt1 = time.perf_counter() - t1
    cpu.set_threads(threads)
    return {"value": n / dt, "unit": "force evals/s", "cores": threads, "kind": cpu.kind,
            "sample": f"{n_sets_sample} of the {N_SETS} parameter sets x full {NV}x{NZ} grid "
                      f"({n} points, {dt:.2f} s): {cpu.what}",
            "one_thread": {"value": one * NV * NZ / dt1, "sample": f"{one} sets x {NV}x{NZ} grid"},
            "cpu_model": cpu_model(), "os_cpu_count": os.cpu_count()}


def _ev_time(torch, fn, reps=3):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _graph_time(torch, fn, reps=20):
    """Device time of fn (ms) with the host's launch overhead taken out: fn is
    captured once in a CUDA graph (outputs from the graph's own pool) and the
    graph is replayed reps times between two events."""
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        fn()  # warm-up outside capture (kernel attributes, module load)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    g.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del g
    return ms


def secondary_measurements(torch, mol, pack, dev, peaks):
    """Particle-steps/s of the trajectory ensembles and the adjoint's cost."""
    from molmot_b200.engine import BeamSets, force_batch, force_adjoint, traj
    from molmot_b200.fields import make_dc_mot_beams
    from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
    out = {}
    rng = np.random.default_rng(SEED)
    # 3D quadrupole MOT, 24 beams, 65,536 particles: r ~ N(0, 1 mm), v ~ MB(5 mK), kicks on
    N3, S3 = 65536, 24
    sim3 = MOTSimulator3D(mol, make_beam_pairs_dc4(mol, -0.30, 0.40, 1.0), B_gradient=0.16)
    sig_v = float(np.sqrt(1.380649e-23 * 5e-3 / mol.mass))
    r0 = torch.as_tensor(rng.normal(0, 1e-3, (N3, 3)), device=dev)
    v0 = torch.as_tensor(rng.normal(0, sig_v, (N3, 3)), device=dev)
    ms = _ev_time(torch, lambda: sim3.run_ensemble(r0, v0, S3 * 1e-6, kicks=True, seed=SEED), 2)
    ps = N3 * S3 / (ms * 1e-3)
    out["traj3d"] = {"metric": "particle-steps/s", "value": ps, "particles": N3, "steps": S3,
                     "ms": ms, "workload": "SrOH 3D quadrupole MOT, 24 beams, leapfrog dt=1us, "
                     "Philox recoil kicks, FP64 state"}
    # a 1000-step chunk of the same ensemble (one launch, timed once)
    from molmot_b200.constants import hbar as HBAR_CODATA
    from molmot_b200.engine import pack_for, traj3d
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    o3 = traj3d(pack_for(mol), sim3._bs(), r0, v0, 1e-6, 1000, kicks=True, seed=SEED, hbar=HBAR_CODATA)
    e1.record()
    torch.cuda.synchronize()
    ms_l = e0.elapsed_time(e1)
    out["traj3d"]["long"] = {"steps": 1000, "ms": ms_l, "value": N3 * 1000 / (ms_l * 1e-3),
                             "alive_fraction": float((o3["r"].norm(dim=1) <= 0.015).double().mean())}
    # 1D DC MOT ensemble (the reference's trajectory configuration), 65,536 particles
    bs1 = BeamSets.from_beams(make_dc_mot_beams(mol, -0.20, 0.70, 1.0), 0.16)
    z0 = torch.as_tensor(rng.normal(0, 2e-3, 65536), device=dev)
    u0 = torch.as_tensor(rng.normal(0, 1.0, 65536), device=dev)
    S1 = 1000
    ms = _ev_time(torch, lambda: traj(pack, bs1, z0, u0, 1e-6, S1), 2)
    out["traj1d"] = {"metric": "particle-steps/s", "value": 65536 * (S1 - 1) / (ms * 1e-3),
                     "particles": 65536, "steps": S1, "ms": ms,
                     "workload": "SrOH 1D DC MOT (delta -0.2, split 0.7, s0 1, B' 0.16 T/m), Euler, "
                                 "plain FP64 (the reference's operation order)"}
    ms = _ev_time(torch, lambda: traj(pack, bs1, z0, u0, 1e-6, S1, precision="fp32"), 2)
    out["traj1d_fp32"] = {"metric": "particle-steps/s", "value": 65536 * (S1 - 1) / (ms * 1e-3),
                          "particles": 65536, "steps": S1, "ms": ms,
                          "workload": "the same ensemble, FP32-bulk force (reduced solve), one "
                                      "particle per thread"}
    # trajectory gradient: d<E_kin>/d(4 detunings) of the per-axis 3D model,
    # 4096 particles x 1000 steps, kicks at fixed noise, checkpoints every 50 steps
    from molmot_b200.trajgrad import traj_grad
    NG, SG = 4096, 1000
    rg = torch.as_tensor(rng.normal(0, 1e-3, (NG, 3)), device=dev)
    vg = torch.as_tensor(rng.normal(0, sig_v, (NG, 3)), device=dev)
    fpar = [0, 0, 1, 1, 2, 2, 3, 3]
    run = lambda: traj_grad(pack, bs1, rg, vg, 1e-6, SG, n_par=4, freq_par=fpar, kicks=True,
                            seed=SEED, ckpt_every=50)
    msg = _ev_time(torch, run, 2)
    msf = _ev_time(torch, lambda: traj(pack, bs1, rg, vg, 1e-6, SG + 1, ndim=3), 2)
    g = run()
    grad = (mol.mass * (g["v"][:, :, None] * g["dv"]).sum(1).mean(0)).cpu().numpy()
    out["traj_grad"] = {"metric": "particle-steps/s", "value": NG * SG / (msg * 1e-3),
                        "particles": NG, "steps": SG, "ms": msg, "forward_fp64_ms": msf,
                        "cost_ratio_vs_fp64_forward": msg / msf,
                        "dE_ddetuning_J_per_Hz": [float(x) for x in grad],
                        "workload": "SrOH per-axis 3D quadrupole MOT (trajectories.py:78-156), DC "
                                    "4-frequency beams, r ~ N(0, 1 mm), v ~ MB(5 mK), Euler dt=1us, "
                                    "recoil kicks at fixed noise, tangents for the 4 detunings, "
                                    "state checkpointed every 50 steps"}
    # the same gradient through the 24-beam 3D force: SrOH's ground Zeeman
    # spectrum is degenerate there (the eigenbasis derivative is undefined), so
    # a non-degenerate synthetic 12 + 4 molecule with the same beam geometry;
    # 4096 particles x 1000 leapfrog steps, kicks at fixed noise, 4 detunings,
    # checkpoints every 50 steps
    out["traj3d_grad"] = traj3d_grad_measurement(torch, dev, sig_v)
    # adjoint: 1024 parameter sets x 66 stencil points (33 z + 33 v)
    kdir, freq, pol, s0, B = make_params(mol, 1024, SEED + 7)
    bsa = BeamSets(kdir, freq, pol, s0, B)
    zs = np.linspace(-0.3e-3, 0.3e-3, 33)
    vs = np.linspace(-0.1, 0.1, 33)
    v = torch.as_tensor(np.tile(np.concatenate([np.zeros(33), vs]), 1024), device=dev)
    z = torch.as_tensor(np.tile(np.concatenate([zs, np.zeros(33)]), 1024), device=dev)
    # each form's kernels timed from CUDA-graph replays (these launches take ~0.1 ms,
    # the size of the host's per-call overhead)
    tf = _graph_time(torch, lambda: force_batch(pack, bsa, v, z, points_per_set=66, want_pop=False,
                                                want_R=False, want_status=False))
    ta = _graph_time(torch, lambda: force_adjoint(pack, bsa, v, z, points_per_set=66))
    trf = _graph_time(torch, lambda: force_batch(pack, bsa, v, z, points_per_set=66, want_pop=False,
                                                 want_R=False, want_status=False,
                                                 precision="fp64_reduced"))
    tra = _graph_time(torch, lambda: force_adjoint(pack, bsa, v, z, points_per_set=66,
                                                   precision="fp64_reduced"))
    out["adjoint"] = {"workload": "1024 parameter sets x (33 z + 33 v) stencil points, gradients "
                                  "w.r.t. 8 beam frequencies, 8 s0 and B'",
                      "forward_ms": tf, "forward_plus_adjoint_ms": ta, "cost_ratio": ta / tf,
                      "reduced": {"forward_ms": trf, "forward_plus_adjoint_ms": tra,
                                  "cost_ratio": tra / trf, "vs_elimination_adjoint": ta / tra}}
    out["uneven"] = uneven_measurement(torch, dev, peaks)
    return out


def traj3d_grad_measurement(torch, dev, sig_v):
    """Particle-steps/s of the 3D trajectory tangents (mm_traj3d_grad_run) and
    the cost against the forward-only 3D run of the same ensemble."""
    from molmot_b200.constants import hbar as HBAR_CODATA
    from molmot_b200.engine import pack_for, traj3d
    from molmot_b200.molecules.synthetic import synthetic_molecule
    from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
    from molmot_b200.trajgrad import traj3d_grad
    m = synthetic_molecule(12, 4, 5)
    sim = MOTSimulator3D(m, make_beam_pairs_dc4(m, -0.5, 0.5, 1.0), B_gradient=0.2)
    rng = np.random.default_rng(SEED + 3)
    N, S = 4096, 1000
    r0 = torch.as_tensor(rng.normal(0, 1e-3, (N, 3)), device=dev)
    v0 = torch.as_tensor(rng.normal(0, sig_v, (N, 3)), device=dev)
    bs, pk = sim._bs(), pack_for(m)
    fpar = [b // 6 for b in range(24)]
    run = lambda: traj3d_grad(pk, bs, r0, v0, 1e-6, S, n_par=4, freq_par=fpar, kicks=True, seed=SEED,
                              ckpt_every=50, allow_degenerate=True)
    ms = _ev_time(torch, run, 1)
    msf = _ev_time(torch, lambda: traj3d(pk, bs, r0, v0, 1e-6, S, kicks=True, seed=SEED, hbar=HBAR_CODATA), 1)
    o = run()
    alive = (o["r"].norm(dim=1) <= 0.015)
    g = (m.mass * (o["v"][:, :, None] * o["dv"]).sum(1)[alive].mean(0)).cpu().numpy()
    return {"metric": "particle-steps/s", "value": N * S / (ms * 1e-3), "particles": N, "steps": S, "ms": ms,
            "forward_ms": msf, "cost_ratio_vs_forward": ms / msf,
            "degenerate_particles": int(((o["status"] & 8) != 0).sum()),
            "dE_ddetuning_J_per_Hz": [float(x) for x in g],
            "workload": "synthetic 12+4 molecule with a non-degenerate ground Zeeman spectrum, 24-beam "
                        "3D quadrupole MOT, leapfrog dt=1us, recoil kicks at fixed noise, tangents for "
                        "the 4 frequency components, checkpoints every 50 steps"}


def uneven_measurement(torch, dev, peaks):
    """The uneven batch: 2048 synthetic molecules (n_ground 4..48, n_excited
    4..16), 64..4096 points each, in one persistent launch per size class
    (warps per CTA from the autotuner), its CUDA-graph replay, and one launch
    per molecule on every 8th molecule, scaled to the whole batch by points.
    Roofline: the batch's algorithmic FP64 FLOP (flops.uneven_flops) over the
    persistent time, against the FP64 FMA peak."""
    from molmot_b200.engine import BeamSets
    from molmot_b200.flops import uneven_flops
    from molmot_b200.uneven import MoleculeBank, UnevenBatch, make_uneven_workload, sample_molecules
    mols, counts, (kd, fr, po, s0), Bu, vu, zu = make_uneven_workload(n_mol=2048, seed=SEED)
    ub = UnevenBatch(MoleculeBank(mols), counts, BeamSets(kd, fr, po, s0, Bu))
    vd = torch.as_tensor(vu, device=dev)
    zd = torch.as_tensor(zu, device=dev)
    wpc = ub.autotune(vd, zd)
    ms_p = _ev_time(torch, lambda: ub.force(vd, zd), 3)
    F = ub.force(vd, zd)["F"].cpu().numpy()
    g, _, _, _ = ub.graph(vd, zd)
    ms_g = _ev_time(torch, g.replay, 3)
    del g
    off = np.concatenate([[0], np.cumsum(counts)])
    sample = list(range(0, len(mols), 8))
    singles = []
    for i in sample:
        u = UnevenBatch(MoleculeBank([mols[i]]), [counts[i]],
                        BeamSets(kd[i:i + 1], fr[i:i + 1], po[i:i + 1], s0[i:i + 1], Bu[i:i + 1]),
                        warps_per_cta=wpc)
        singles.append((u, vd[off[i]:off[i + 1]], zd[off[i]:off[i + 1]]))
    ms_s = _ev_time(torch, lambda: [u.force(a, b) for u, a, b in singles], 2)
    pts_s = int(sum(counts[i] for i in sample))
    # the same sample as one launch per molecule of the plain form (mm_force_batch,
    # FP64, the reference's elimination), as the reference launches per molecule
    from molmot_b200.engine import MoleculePack, force_batch
    plain = [(MoleculePack(mols[i]),
              BeamSets(kd[i:i + 1], fr[i:i + 1], po[i:i + 1], s0[i:i + 1], Bu[i:i + 1]),
              vd[off[i]:off[i + 1]], zd[off[i]:off[i + 1]]) for i in sample]
    ms_pl = _ev_time(torch, lambda: [force_batch(pk, b, a, c, precision="fp64", want_pop=False)
                                     for pk, b, a, c in plain], 2)
    n = int(off[-1])
    fl = uneven_flops(mols, counts, po)
    achieved = fl / (ms_p * 1e-3) / 1e12
    pick = sample_molecules([m.n_ground for m in mols], [m.n_excited for m in mols], counts)
    check = [(mols[m], (kd[m:m + 1], fr[m:m + 1], po[m:m + 1], s0[m:m + 1], Bu[m:m + 1]),
              vu[off[m]:off[m + 1]], zu[off[m]:off[m + 1]], F[off[m]:off[m + 1]]) for m in pick]
    return {"metric": "force evals/s", "points": n, "molecules": len(mols),
            "persistent_ms": ms_p, "persistent_value": n / (ms_p * 1e-3),
            "graph_replay_ms": ms_g, "warps_per_cta": list(wpc),
            "per_molecule_launches_ms_estimate": ms_s * n / pts_s,
            "per_molecule_plain_fp64_ms_estimate": ms_pl * n / pts_s,
            "per_molecule_sample": f"{len(sample)} molecules ({pts_s} points), scaled by points",
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peaks["fp64"],
                         "unit": "TFLOP/s", "frac": achieved / peaks["fp64"],
                         "flops_per_point_mean": fl / n},
            "workload": "2048 synthetic molecules, n_ground 4..48, n_excited 4..16, 64..4096 "
                        "(v, z) points each; FP64 rates in the reference's order, populations "
                        "from the FP64 excited-chain solve (the reference's elimination for "
                        "molecules the reduction does not cover)",
            "_check": check}


def uneven_oracle_check(check):
    """The uneven batch's forces against the CPU oracle on the sample of
    sample_molecules (4 molecules per size class, including the most points
    and n_ground 48): max |dF| / max |F| per molecule (the checker; part of
    the cpu_baseline leg)."""
    from oracle import rate_eq as orc
    worst = 0.0
    for mol, (kd, fr, po, s0, B), v, z, F in check:
        Fo = orc.force_batch(mol, kd, fr, po, s0, B, v, z, want_pop=False)[0]
        worst = max(worst, float(np.abs(F - Fo).max() / np.abs(Fo).max()))
    return {"max": worst, "molecules": len(check),
            "points": int(sum(len(c[2]) for c in check)),
            "n_ground": sorted({int(c[0].n_ground) for c in check})}


def evidence_line(plain, red64, accuracy, secondary):
    """The measured figures beside the headline, compact (numbers only)."""
    r = lambda x, d=4: float(f"{x:.{d}g}") if x is not None else None
    ev = {"plain_fp64": {"value": r(plain["value"]), "ms": r(plain["ms_per_step"]),
                         "frac_fp64": r(plain["roofline"]["frac"], 3),
                         "fp32_form_speedup": r(plain["fp32_form_speedup"], 3)},
          "fp64_reduced": {"value": r(red64["value"]), "ms": r(red64["ms_per_step"]),
                           "diff_vs_plain": r(red64["max_rel_diff_vs_plain_fp64_per_set"], 2)},
          "acc_fp32_vs_fp64": {k: r(accuracy["fp32_vs_fp64_per_set"][k], 2) for k in ("max", "p99")}}
    if "vs_oracle" in accuracy:
        ev["acc_vs_oracle"] = {k: r(v["max"], 2) for k, v in accuracy["vs_oracle"].items()}
    if secondary:
        t3, u = secondary["traj3d"], secondary["uneven"]
        ev["traj3d"] = {"value": r(t3["value"]), "ms": r(t3["ms"]), "steps": t3["steps"]}
        if "long" in t3:
            ev["traj3d"]["long"] = {k: r(v) for k, v in t3["long"].items()}
        ev["traj1d"] = {"fp64": r(secondary["traj1d"]["value"]), "fp32": r(secondary["traj1d_fp32"]["value"])}
        ev["traj_grad"] = {"value": r(secondary["traj_grad"]["value"]),
                           "vs_forward": r(secondary["traj_grad"]["cost_ratio_vs_fp64_forward"], 3)}
        t3g = secondary["traj3d_grad"]
        ev["traj3d_grad"] = {"value": r(t3g["value"]), "ms": r(t3g["ms"]),
                             "vs_forward": r(t3g["cost_ratio_vs_forward"], 3)}
        ev["adjoint_cost"] = {"fp64": r(secondary["adjoint"]["cost_ratio"], 3),
                              "reduced": r(secondary["adjoint"]["reduced"]["cost_ratio"], 3)}
        ev["uneven"] = {"value": r(u["persistent_value"]), "ms": r(u["persistent_ms"]),
                        "frac_fp64": r(u["roofline"]["frac"], 3), "graph_ms": r(u["graph_replay_ms"]),
                        "per_molecule_ms": r(u["per_molecule_launches_ms_estimate"]),
                        "per_molecule_plain_ms": r(u["per_molecule_plain_fp64_ms_estimate"])}
        if "accuracy_vs_oracle" in u:
            ev["uneven"]["acc_vs_oracle"] = r(u["accuracy_vs_oracle"]["max"], 2)
    return ev


def oracle_check(mol, pack, bs, v_d, z_d, kdir, freq, pol, s0, B, sets=(0, 1, 2047, 4095)):
    """Both GPU forms against the CPU oracle on a few whole sets (the checker;
    part of the cpu_baseline leg, rank 0 only)."""
    import torch
    from molmot_b200.engine import force_batch
    from oracle import rate_eq as orc
    v_h = v_d.cpu().numpy()
    z_h = z_d.cpu().numpy()
    sets = [s for s in sets if s < kdir.shape[0]]
    Fo = orc.force_batch(mol, kdir[sets], freq[sets], pol[sets], s0[sets], B[sets], v_h, z_h,
                         grid=True, want_pop=False)[0].reshape(len(sets), -1)
    res = {}
    for prec in ("fp64", "fp32"):
        o = force_batch(pack, bs, v_d, z_d, grid=True, precision=prec, want_pop=False,
                        want_R=False, want_status=False)
        F = o["F"].cpu().numpy().reshape(kdir.shape[0], -1)[sets]
        errs = np.max(np.abs(F - Fo), axis=1) / np.max(np.abs(Fo), axis=1)
        res[prec] = {"max": float(errs.max()), "sets": [int(s) for s in sets]}
    torch.cuda.synchronize()
    return res


def run_reference_arm(args):
    """The reference's own CPU path of the force maps (CpuForceMaps: its
    numba core from baseline/_ref on every host core), on this workload's
    metric and unit.  Each step is a bounded sample: 32 of the 4096 parameter
    sets over the full 256 x 256 grid.  Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from molmot_b200.molecules import load_sroh_from_julia
    mol = load_sroh_from_julia()
    cpu = CpuForceMaps(mol)
    n_sample = 32
    kdir, freq, pol, s0, B = make_params(mol, n_sample, SEED)
    v = np.linspace(-10, 10, NV)
    z = np.linspace(-1e-2, 1e-2, NZ)
    cpu(kdir[:1], freq[:1], pol[:1], s0[:1], B[:1], v[:4], z[:4])  # compile
    for _ in range(args.warmup):
        cpu(kdir, freq, pol, s0, B, v, z)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cpu(kdir, freq, pol, s0, B, v, z)
        times.append(time.perf_counter() - t0)
    n = n_sample * NV * NZ
    val = n / (sum(times) / len(times))
    sample = (f"each step: {n_sample} of the {N_SETS} parameter sets x full {NV}x{NZ} grid "
              f"({n} points) on the host CPU; {cpu.what}")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "force evals/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"SrOH batched force maps, {N_SETS} sets x {NV}x{NZ} (v,z) grid, "
                                   "8-beam DC MOT (bounded CPU sample per step)",
                       "sets_per_step_sample": n_sample},
            "cpu_baseline": {"value": val, "unit": "force evals/s", "cores": cpu.threads(),
                             "kind": cpu.kind, "sample": sample, "cpu_model": cpu_model(),
                             "os_cpu_count": os.cpu_count()},
            "e2e": {"value": val, "unit": "force evals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def traj3d_full_run(total_steps, chunk=1000):
    """The 3D ensemble at its full size: 65,536 SrOH particles, r ~ N(0, 1 mm),
    v ~ MB(5 mK), 24-beam quadrupole MOT, leapfrog dt = 1 us, Philox kicks,
    FP64 state, run as resumed chunks of `chunk` steps (each chunk one launch,
    bit-identical to one long launch).  Device time is the sum of the chunks'
    CUDA-event times; the line also gives the surviving fraction, the
    temperature of the survivors and the scattering events."""
    import torch
    from molmot_b200.constants import hbar as HBAR_CODATA
    from molmot_b200.engine import pack_for, traj3d
    from molmot_b200.molecules import load_sroh_from_julia
    from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
    dev = torch.device("cuda", 0)
    mol = load_sroh_from_julia()
    N = 65536
    sim3 = MOTSimulator3D(mol, make_beam_pairs_dc4(mol, -0.30, 0.40, 1.0), B_gradient=0.16)
    rng = np.random.default_rng(SEED)
    sig_v = float(np.sqrt(1.380649e-23 * 5e-3 / mol.mass))
    r = torch.as_tensor(rng.normal(0, 1e-3, (N, 3)), device=dev)
    vh = torch.as_tensor(rng.normal(0, sig_v, (N, 3)), device=dev)
    pack, bs = pack_for(mol), sim3._bs()
    events = torch.zeros(N, dtype=torch.int64, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = 0.0
    clocks = ClockSampler(0)
    clocks.start()
    done = 0
    o = None
    while done < total_steps:
        n = min(chunk, total_steps - done)
        e0.record()
        o = traj3d(pack, bs, r, vh, 1e-6, n, step0=done, kicks=True, seed=SEED, hbar=HBAR_CODATA)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        r, vh = o["r"], o["vh"]
        events += o["n_events"].to(torch.int64)
        done += n
    ck = clocks.stop()
    alive = r.norm(dim=1) <= 0.015
    v = o["v"][alive]
    T = float(mol.mass * (v ** 2).sum(1).mean() / (3 * 1.380649e-23)) if bool(alive.any()) else None
    line = {"metric": "particle-steps/s", "value": N * total_steps / (ms * 1e-3), "unit": "particle-steps/s",
            "n_gpus": 1, "steps": total_steps, "particles": N, "seconds": ms * 1e-3, "chunks": -(-total_steps // chunk),
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "SrOH 3D quadrupole MOT, 24 beams (4 frequency pairs x 6 directions), "
                                   "B' 0.16 T/m, leapfrog dt 1 us, Philox recoil kicks, FP64 state; "
                                   "r ~ N(0, 1 mm), v ~ Maxwell-Boltzmann at 5 mK"},
            "final": {"surviving_fraction": float(alive.double().mean()), "temperature_K": T,
                      "scattering_events": int(events.sum())},
            "clocks": ck}
    print(json.dumps(line))


def profile_case(name):
    """One small workload of a kernel family, run twice (the second launch is
    the one to capture), for ncu captures that must stay small:
      large       -- force maps of a 24 + 6 synthetic molecule (large_force_kernel),
                     64 sets x 64 x 64 points, plain FP64 and excited-chain forms;
      traj3d      -- the SrOH 3D ensemble (traj3d_kernel), 8192 particles x 24 steps;
      traj3d_grad -- 3D tangents, synthetic 12 + 4 molecule, 256 particles x 20 steps;
      traj_grad   -- per-axis tangents, SrOH, 4096 particles x 50 steps;
      uneven      -- the 2048-molecule uneven batch, one persistent call;
      adjoint     -- the FP64 elimination adjoint, 1024 SrOH sets x 66 stencil points."""
    import torch
    from molmot_b200.engine import BeamSets, MoleculePack, force_batch, pack_for
    from molmot_b200.molecules import load_sroh_from_julia
    from molmot_b200.molecules.synthetic import dc_beams_for, synthetic_molecule
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(SEED)
    t0 = time.perf_counter()
    for _ in range(2):
        if name == "large":
            m = synthetic_molecule(24, 6, 32)
            kd, fr, po, s0 = dc_beams_for(m)
            n = 64
            bs = BeamSets(np.tile(kd, (n, 1)), fr[None] + rng.uniform(-1e7, 0, (n, 1)), np.tile(po, (n, 1)),
                          np.tile(s0, (n, 1)), rng.uniform(0.1, 0.4, n))
            v = torch.as_tensor(np.linspace(-8, 8, 64), device=dev)
            z = torch.as_tensor(np.linspace(-8e-3, 8e-3, 64), device=dev)
            for prec in ("fp64", "fp64_reduced"):
                force_batch(MoleculePack(m), bs, v, z, grid=True, precision=prec, want_pop=False)
        elif name == "traj3d_grad":
            from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
            from molmot_b200.trajgrad import traj3d_grad
            m = synthetic_molecule(12, 4, 5)
            sim = MOTSimulator3D(m, make_beam_pairs_dc4(m, -0.5, 0.5, 1.0), B_gradient=0.2)
            r0 = rng.normal(0, 1e-3, (256, 3))
            v0 = rng.normal(0, 0.6, (256, 3))
            traj3d_grad(pack_for(m), sim._bs(), r0, v0, 1e-6, 20, n_par=4, freq_par=[b // 6 for b in range(24)],
                        kicks=True, seed=SEED)
        elif name == "traj3d":
            from molmot_b200.constants import hbar as HBAR_CODATA
            from molmot_b200.engine import traj3d
            from molmot_b200.simulator_3d import MOTSimulator3D, make_beam_pairs_dc4
            mol = load_sroh_from_julia()
            sim = MOTSimulator3D(mol, make_beam_pairs_dc4(mol, -0.30, 0.40, 1.0), B_gradient=0.16)
            r0 = rng.normal(0, 1e-3, (8192, 3))
            v0 = rng.normal(0, 0.6, (8192, 3))
            traj3d(pack_for(mol), sim._bs(), r0, v0, 1e-6, 24, kicks=True, seed=SEED, hbar=HBAR_CODATA)
        elif name == "traj_grad":
            from molmot_b200.fields import make_dc_mot_beams
            from molmot_b200.trajgrad import traj_grad
            mol = load_sroh_from_julia()
            bs = BeamSets.from_beams(make_dc_mot_beams(mol, -0.20, 0.70, 1.0), 0.16)
            r0 = rng.normal(0, 1e-3, (4096, 3))
            v0 = rng.normal(0, 0.6, (4096, 3))
            traj_grad(pack_for(mol), bs, r0, v0, 1e-6, 50, n_par=4, freq_par=[0, 0, 1, 1, 2, 2, 3, 3],
                      kicks=True, seed=SEED)
        elif name == "adjoint":
            from molmot_b200.engine import force_adjoint
            mol = load_sroh_from_julia()
            bsa = BeamSets(*make_params(mol, 1024, SEED + 7))
            v = np.tile(np.concatenate([np.zeros(33), np.linspace(-0.1, 0.1, 33)]), 1024)
            z = np.tile(np.concatenate([np.linspace(-0.3e-3, 0.3e-3, 33), np.zeros(33)]), 1024)
            force_adjoint(pack_for(mol), bsa, v, z, points_per_set=66)
        elif name == "uneven":
            from molmot_b200.uneven import MoleculeBank, UnevenBatch, make_uneven_workload
            mols, counts, (kd, fr, po, s0), Bu, vu, zu = make_uneven_workload(n_mol=2048, seed=SEED)
            ub = UnevenBatch(MoleculeBank(mols), counts, BeamSets(kd, fr, po, s0, Bu))
            ub.force(vu, zu)
        torch.cuda.synchronize()
    print(json.dumps({"case": name, "seconds": time.perf_counter() - t0}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--sets", type=int, default=N_SETS, help="parameter sets per GPU")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the trajectory / adjoint measurements (small profiling runs)")
    ap.add_argument("--case", default="", choices=["", "large", "traj3d", "traj3d_grad", "traj_grad", "uneven",
                                                   "adjoint"],
                    help="run one small workload of the named kernel twice and exit (profiling runs)")
    ap.add_argument("--traj3d-full", type=int, default=0, metavar="STEPS",
                    help="instead of the force maps: run the whole 3D ensemble (65,536 particles, "
                         "STEPS leapfrog steps, e.g. 30000) in 1000-step resumed chunks and print "
                         "its own JSON line (about 160 s at 30000 steps)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.traj3d_full:
        return traj3d_full_run(args.traj3d_full)
    if args.case:
        return profile_case(args.case)

    import torch
    import torch.distributed as dist
    from molmot_b200.molecules import load_sroh_from_julia
    from molmot_b200.engine import MoleculePack, BeamSets, force_batch, force_maps_to_host
    from molmot_b200.flops import active_triples, flops_per_point, flops_reduced

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    mol = load_sroh_from_julia()
    pack = MoleculePack(mol)
    n_sets = args.sets
    kdir, freq, pol, s0, B = make_params(mol, n_sets, SEED + rank)
    v_h = np.linspace(-10, 10, NV)
    z_h = np.linspace(-1e-2, 1e-2, NZ)
    bs = BeamSets(kdir, freq, pol, s0, B)
    v_d = torch.as_tensor(v_h, device=dev)
    z_d = torch.as_tensor(z_h, device=dev)
    n_pts = n_sets * NV * NZ
    out = {"F": torch.empty((n_sets, NV, NZ), dtype=torch.float64, device=dev)}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)

    def timed(precision, steps, warmup):
        for _ in range(warmup):
            force_batch(pack, bs, v_d, z_d, grid=True, precision=precision, out=out)
        barrier()
        evs = []
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            force_batch(pack, bs, v_d, z_d, grid=True, precision=precision, out=out)
            e1.record()
            evs.append((e0, e1))
        barrier()
        ms = sum(a.elapsed_time(b) for a, b in evs) / steps
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    peaks = peak_probe(torch)
    clocks = ClockSampler(local)
    clocks.start()
    ms32 = timed("fp32", args.steps, args.warmup)
    F32 = out["F"].clone()
    ms64 = timed("fp64", args.steps, args.warmup)
    F64 = out["F"].clone()
    ms64r = timed("fp64_reduced", args.steps, args.warmup)
    clk = clocks.stop()
    err64r = float((((out["F"] - F64).abs().amax(dim=(1, 2))) / F64.abs().amax(dim=(1, 2))).max())
    out["F"].copy_(F64)
    del F64
    # per-set accuracy of the FP32 form against the plain FP64 form (every set)
    scale = out["F"].abs().amax(dim=(1, 2))
    err_sets = ((F32 - out["F"]).abs().amax(dim=(1, 2)) / scale).cpu().numpy()
    del F32
    accuracy = {"fp32_vs_fp64_per_set": {"max": float(err_sets.max()),
                                         "median": float(np.median(err_sets)),
                                         "p99": float(np.quantile(err_sets, 0.99)),
                                         "sets": int(err_sets.size)}}

    # end to end through the public API with host buffers
    pinned_F = torch.empty((n_sets, NV, NZ), dtype=torch.float64, pin_memory=True)
    params_h = [np.ascontiguousarray(a) for a in (kdir, freq, pol, s0, B)]
    h2d = sum(a.nbytes for a in params_h) + v_h.nbytes + z_h.nbytes
    d2h = pinned_F.numel() * 8

    def e2e_step():
        # parameters and grid axes host->device, maps device->host in 64-set
        # chunks whose copies overlap the next chunk's computation
        b2 = BeamSets(*params_h)
        vv = torch.as_tensor(v_h).to(dev)
        zz = torch.as_tensor(z_h).to(dev)
        return force_maps_to_host(pack, b2, vv, zz, out=pinned_F, precision="fp32", chunk_sets=64)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    t = torch.tensor([sum(e2e_ms) / len(e2e_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_e2e = float(t.item())

    secondary = (secondary_measurements(torch, mol, pack, dev, peaks)
                 if world == 1 and not args.no_secondary else None)

    A = active_triples(mol.d_squared, pol[0])
    f64_32, f32_32 = flops_reduced(12, 4, A)
    f64_64, _ = flops_per_point(12, 4, 8, A)
    # FP32 form: FP64 and FP32 pipes run concurrently; the bound is the slower of the two
    t_min32 = max(f64_32 * n_pts / (peaks["fp64"] * 1e12), f32_32 * n_pts / (peaks["fp32"] * 1e12))
    achieved32 = (f64_32 + f32_32) * n_pts / (ms32 * 1e-3) / 1e12
    peak32 = (f64_32 + f32_32) * n_pts / t_min32 / 1e12
    achieved64 = f64_64 * n_pts / (ms64 * 1e-3) / 1e12

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(mol)
        accuracy["vs_oracle"] = oracle_check(mol, pack, bs, v_d, z_d, kdir, freq, pol, s0, B)
        if secondary is not None:
            secondary["uneven"]["accuracy_vs_oracle"] = uneven_oracle_check(secondary["uneven"].pop("_check"))
    elif secondary is not None:
        secondary["uneven"].pop("_check", None)

    if rank == 0:
        total = n_pts * world
        plain = {"value": total / (ms64 * 1e-3), "unit": "force evals/s", "ms_per_step": ms64,
                 "fp32_form_speedup": ms64 / ms32,
                 "roofline": {"bound": "fp64", "achieved": achieved64, "peak": peaks["fp64"],
                              "unit": "TFLOP/s", "frac": achieved64 / peaks["fp64"]}}
        red64 = {"value": total / (ms64r * 1e-3), "unit": "force evals/s", "ms_per_step": ms64r,
                 "max_rel_diff_vs_plain_fp64_per_set": err64r}
        roof = {"bound": "fp64+fp32", "achieved": achieved32, "peak": peak32, "unit": "TFLOP/s",
                "frac": achieved32 / peak32,
                "traffic": TRAFFIC_PER_POINT * n_pts, "traffic_unit": "bytes per launch",
                "algorithmic_bytes": 8 * n_pts,
                "peak_source": f"FMA probe on this GPU: fp64 {peaks['fp64']:.1f}, fp32 "
                               f"{peaks['fp32']:.1f} TFLOP/s",
                "flops_per_point": {"fp64": f64_32, "fp32": f32_32}}
        e2e = {"value": total / (ms_e2e * 1e-3), "unit": "force evals/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e,
               "api": "engine.force_maps_to_host, 64-set chunks"}
        details = {"bench_details": {
            "plain_fp64": plain, "fp64_reduced": red64, "accuracy": accuracy, "secondary": secondary,
            "roofline": dict(roof, hbm=hbm_figure(8 * n_pts, ms32),
                             reference_algorithm_equivalent_tflops=f64_64 * n_pts / (ms32 * 1e-3) / 1e12,
                             traffic_source="DRAM read + write per point of an ncu capture of "
                                            "force_reduced_kernel (512 sets), times the points"),
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk}}
        # everything, first (long); then the compact evidence line and the
        # headline, which are the last lines of the output
        print(json.dumps(details), flush=True)
        print(json.dumps({"evidence": evidence_line(plain, red64, accuracy, secondary)}), flush=True)
        line = {
            "metric": METRIC, "value": total / (ms32 * 1e-3), "unit": "force evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": f"SrOH 12+4 levels, {n_sets} parameter sets x {NV}x{NZ} (v, z) "
                                   "grid per GPU, 8-beam DC MOT; FP32 Lorentzians, FP64 sums and "
                                   "excited-chain solve",
                       "points_per_step_per_gpu": n_pts, "parallelism": f"sets sharded, {world} GPU(s)",
                       "l2": "256 MB written between timed steps"},
            "roofline": {k: roof[k] for k in ("bound", "achieved", "peak", "unit", "frac", "traffic",
                                              "peak_source")},
            "e2e": e2e,
            "gpu_launches": args.steps * 3,
            "clocks": {k: clk.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": cpu["unit"], "cores": cpu["cores"],
                                    "kind": cpu["kind"],
                                    "sample": f"1024 of 4096 sets x 256x256 grid; {cpu['kind']}: "
                                              + ("the reference's _rate_eq_core unchanged, numba prange"
                                                 if cpu["kind"] == "reference" else "C restatement"),
                                    "one_thread": round(cpu["one_thread"]["value"]),
                                    "cpu_model": cpu["cpu_model"]}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
