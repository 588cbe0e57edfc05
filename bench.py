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
             this GPU (mm_peak_probe); algorithmic FLOPs per point of the form
             that runs (molmot_b200/flops.py).
cpu_baseline: the reference's numba core restated (oracle/rate_eq_numba.py)
             on all host cores, on a bounded sample of the same workload.

`--impl reference` prints the CPU reference arm instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "16-level steady-state force evals/s and particle-steps/s: plain FP64 vs FP32+refine @1e-6"
N_SETS, NV, NZ = 4096, 256, 256
# dram__bytes_read.sum + dram__bytes_write.sum of one force_reduced_kernel launch
# over the default workload (11.46 MB + 2.22 GB)
TRAFFIC_PER_LAUNCH = 2.2315e9
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
    """Measured FP64 and FP32 FMA throughput (TFLOP/s) of this GPU."""
    import ctypes
    from molmot_b200 import _lib
    L = _lib.load()
    out = {}
    for which, name, iters in [(0, "fp64", 4096), (1, "fp32", 16384)]:
        best = 0.0
        for _ in range(3):
            ms, fl = ctypes.c_double(), ctypes.c_double()
            _lib.check(L.mm_peak_probe(which, iters, ctypes.byref(ms), ctypes.byref(fl),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
                       "mm_peak_probe")
            best = max(best, fl.value / (ms.value * 1e-3) / 1e12)
        out[name] = best
    return out


def cpu_baseline(mol, n_sets_sample=2048):
    """The reference's numba core (restated) on all host cores, on a sample of
    2048 of the 4096 parameter sets (1.3e8 points, about 15 s on 16 cores)."""
    from oracle import rate_eq_numba as nb
    kdir, freq, pol, s0, B = make_params(mol, n_sets_sample, SEED)
    v = np.linspace(-10, 10, NV)
    z = np.linspace(-1e-2, 1e-2, NZ)
    nb.force_grid(mol, kdir[:1], freq[:1], pol[:1], s0[:1], B[:1], v[:4], z[:4])  # compile
    t0 = time.perf_counter()
    nb.force_grid(mol, kdir, freq, pol, s0, B, v, z)
    dt = time.perf_counter() - t0
    n = n_sets_sample * NV * NZ
    return {"value": n / dt, "unit": "force evals/s", "cores": nb.threads(), "kind": "port",
            "sample": f"{n_sets_sample} of the {N_SETS} parameter sets, full {NV}x{NZ} grid "
                      f"({n} points, {dt:.2f} s), numba restatement of _rate_eq_core, "
                      f"prange over points, os.cpu_count()={os.cpu_count()}"}


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


def secondary_measurements(torch, mol, pack, dev):
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
                     "Philox recoil kicks, FP64 state; full 65,536 x 30,000-step run "
                     f"extrapolates to {N3 * 30000 / ps:.0f} s"}
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
    # adjoint: 1024 parameter sets x 66 stencil points (33 z + 33 v)
    kdir, freq, pol, s0, B = make_params(mol, 1024, SEED + 7)
    bsa = BeamSets(kdir, freq, pol, s0, B)
    zs = np.linspace(-0.3e-3, 0.3e-3, 33)
    vs = np.linspace(-0.1, 0.1, 33)
    v = torch.as_tensor(np.tile(np.concatenate([np.zeros(33), vs]), 1024), device=dev)
    z = torch.as_tensor(np.tile(np.concatenate([zs, np.zeros(33)]), 1024), device=dev)
    tf = _ev_time(torch, lambda: force_batch(pack, bsa, v, z, points_per_set=66, want_pop=False,
                                             want_R=False, want_status=False), 5)
    ta = _ev_time(torch, lambda: force_adjoint(pack, bsa, v, z, points_per_set=66), 5)
    trf = _ev_time(torch, lambda: force_batch(pack, bsa, v, z, points_per_set=66, want_pop=False,
                                              want_R=False, want_status=False,
                                              precision="fp64_reduced"), 5)
    tra = _ev_time(torch, lambda: force_adjoint(pack, bsa, v, z, points_per_set=66,
                                                precision="fp64_reduced"), 5)
    out["adjoint"] = {"workload": "1024 parameter sets x (33 z + 33 v) stencil points, gradients "
                                  "w.r.t. 8 beam frequencies, 8 s0 and B'",
                      "forward_ms": tf, "forward_plus_adjoint_ms": ta, "cost_ratio": ta / tf,
                      "reduced": {"forward_ms": trf, "forward_plus_adjoint_ms": tra,
                                  "cost_ratio": tra / trf, "vs_elimination_adjoint": ta / tra}}
    out["uneven"] = uneven_measurement(torch, dev)
    return out


def uneven_measurement(torch, dev):
    """The uneven batch: 2048 synthetic molecules (n_ground 4..48, n_excited
    4..16), 64..4096 points each, in one persistent launch per size class
    (warps per CTA from the autotuner), its CUDA-graph replay, and one launch
    per molecule on every 8th molecule, scaled to the whole batch by points."""
    from molmot_b200.engine import BeamSets
    from molmot_b200.uneven import MoleculeBank, UnevenBatch, make_uneven_workload
    mols, counts, (kd, fr, po, s0), Bu, vu, zu = make_uneven_workload(n_mol=2048, seed=SEED)
    ub = UnevenBatch(MoleculeBank(mols), counts, BeamSets(kd, fr, po, s0, Bu))
    vd = torch.as_tensor(vu, device=dev)
    zd = torch.as_tensor(zu, device=dev)
    wpc = ub.autotune(vd, zd)
    ms_p = _ev_time(torch, lambda: ub.force(vd, zd), 3)
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
    n = int(off[-1])
    return {"metric": "force evals/s", "points": n, "molecules": len(mols),
            "persistent_ms": ms_p, "persistent_value": n / (ms_p * 1e-3),
            "graph_replay_ms": ms_g, "warps_per_cta": list(wpc),
            "per_molecule_launches_ms_estimate": ms_s * n / pts_s,
            "per_molecule_sample": f"{len(sample)} molecules ({pts_s} points), scaled by points",
            "workload": "2048 synthetic molecules, n_ground 4..48, n_excited 4..16, 64..4096 "
                        "(v, z) points each; FP64 rates in the reference's order, populations "
                        "from the FP64 excited-chain solve (the reference's elimination for "
                        "molecules the reduction does not cover)"}


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
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from molmot_b200.molecules import load_sroh_from_julia
    from oracle import rate_eq_numba as nb
    mol = load_sroh_from_julia()
    n_sample = 64  # 4.2e6 points per step, under a second on 16 cores
    kdir, freq, pol, s0, B = make_params(mol, n_sample, SEED)
    v = np.linspace(-10, 10, NV)
    z = np.linspace(-1e-2, 1e-2, NZ)
    nb.force_grid(mol, kdir[:1], freq[:1], pol[:1], s0[:1], B[:1], v[:4], z[:4])
    for _ in range(args.warmup):
        nb.force_grid(mol, kdir, freq, pol, s0, B, v, z)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        nb.force_grid(mol, kdir, freq, pol, s0, B, v, z)
        times.append(time.perf_counter() - t0)
    n = n_sample * NV * NZ
    val = n / (sum(times) / len(times))
    sample = (f"each step: {n_sample} of the {N_SETS} parameter sets x full {NV}x{NZ} grid "
              f"({n} points) on the host CPU")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "force evals/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"SrOH batched force maps, {N_SETS} sets x {NV}x{NZ} (v,z) grid, "
                                   "8-beam DC MOT (bounded CPU sample per step)",
                       "sets_per_step_sample": n_sample},
            "cpu_baseline": {"value": val, "unit": "force evals/s", "cores": nb.threads(),
                             "kind": "port", "sample": sample},
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
    ap.add_argument("--traj3d-full", type=int, default=0, metavar="STEPS",
                    help="instead of the force maps: run the whole 3D ensemble (65,536 particles, "
                         "STEPS leapfrog steps, e.g. 30000) in 1000-step resumed chunks and print "
                         "its own JSON line (about 160 s at 30000 steps)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.traj3d_full:
        return traj3d_full_run(args.traj3d_full)

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
        # parameters and grid axes host->device, maps device->host in 256-set
        # chunks whose copies overlap the next chunk's computation
        b2 = BeamSets(*params_h)
        vv = torch.as_tensor(v_h).to(dev)
        zz = torch.as_tensor(z_h).to(dev)
        return force_maps_to_host(pack, b2, vv, zz, out=pinned_F, precision="fp32", chunk_sets=256)

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

    secondary = (secondary_measurements(torch, mol, pack, dev)
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

    if rank == 0:
        total = n_pts * world
        line = {
            "metric": METRIC, "value": total / (ms32 * 1e-3), "unit": "force evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": f"SrOH (12 ground + 4 excited) batched force maps: {n_sets} "
                                   f"parameter sets x {NV}x{NZ} (v, z) grid per GPU, 8-beam DC MOT, "
                                   "FP32 Lorentzians, FP64 sums, FP64 excited-chain population solve",
                       "points_per_step_per_gpu": n_pts, "parallelism": f"sets sharded, {world} GPU(s)",
                       "l2": "256 MB buffer written between timed steps (> 126 MB L2)"},
            "plain_fp64": {"value": total / (ms64 * 1e-3), "unit": "force evals/s",
                           "ms_per_step": ms64, "ratio_fp32_over_fp64": ms64 / ms32,
                           "roofline": {"bound": "fp64", "achieved": achieved64,
                                        "peak": peaks["fp64"], "unit": "TFLOP/s",
                                        "frac": achieved64 / peaks["fp64"]}},
            "fp64_reduced": {"value": total / (ms64r * 1e-3), "unit": "force evals/s",
                             "ms_per_step": ms64r,
                             "max_rel_diff_vs_plain_fp64_per_set": err64r,
                             "form": "FP64 rates in the plain form's order, populations from the "
                                     "FP64 excited-chain solve"},
            "roofline": {"bound": "fp64+fp32", "achieved": achieved32, "peak": peak32,
                         "unit": "TFLOP/s", "frac": achieved32 / peak32,
                         # DRAM read + write of one full launch, ncu capture in
                         # profiles/force_reduced_kernel_sroh_maps.md (4096 sets)
                         "traffic": TRAFFIC_PER_LAUNCH if n_sets == N_SETS else None,
                         "traffic_unit": "bytes per launch",
                         "algorithmic_bytes": 8 * n_pts,
                         "hbm": hbm_figure(8 * n_pts, ms32),
                         "peak_source": "mm_peak_probe FMA loop on this GPU: "
                                        f"fp64 {peaks['fp64']:.2f}, fp32 {peaks['fp32']:.2f} TFLOP/s",
                         "flops_per_point": {"fp64": f64_32, "fp32": f32_32},
                         "reference_algorithm_equivalent_tflops": f64_64 * n_pts / (ms32 * 1e-3) / 1e12},
            "e2e": {"value": total / (ms_e2e * 1e-3), "unit": "force evals/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": ms_e2e,
                    "api": "molmot_b200.engine.force_maps_to_host (256-set chunks, copies "
                           "overlapped with computation)"},
            "accuracy": accuracy,
            "secondary": secondary,
            "gpu_launches": args.steps * 3,
            "clocks": clk,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
