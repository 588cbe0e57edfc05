"""Multi-rank logic on CPU with the gloo backend (world_size 2): sharding,
gathering force maps in unit order, ensemble means, and a rank failure
detected on the host.  The per-unit compute here is the CPU oracle, standing
in for each rank's GPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from molmot_b200.distributed import shard


def test_shard_covers_units_once():
    for n in (0, 1, 5, 4096, 4097):
        for ws in (1, 2, 3, 8):
            blocks = [shard(n, r, ws) for r in range(ws)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(ws - 1))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        from molmot_b200.distributed import sharded_apply, ensemble_mean
        from molmot_b200.molecules import load_sroh_from_julia
        from oracle import rate_eq as orc
        import bench
        mol = load_sroh_from_julia()
        n_sets = 5
        kdir, freq, pol, s0, B = bench.make_params(mol, n_sets, 42)
        v = np.linspace(-5, 5, 4)
        z = np.linspace(-3e-3, 3e-3, 3)

        def compute(lo, hi):
            F = orc.force_batch(mol, kdir[lo:hi], freq[lo:hi], pol[lo:hi], s0[lo:hi], B[lo:hi],
                                v, z, grid=True, want_pop=False, n_threads=1)[0]
            return torch.as_tensor(F.reshape(hi - lo, 4, 3))

        full = sharded_apply(n_sets, compute, gather=True)
        vals = torch.arange(10, dtype=torch.float64) + 10 * rank
        m = ensemble_mean(vals)
        out_q.put((rank, full.numpy(), m))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_and_mean():
    from molmot_b200.molecules import load_sroh_from_julia
    from oracle import rate_eq as orc
    import bench
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mol = load_sroh_from_julia()
    kdir, freq, pol, s0, B = bench.make_params(mol, 5, 42)
    ref = orc.force_batch(mol, kdir, freq, pol, s0, B, np.linspace(-5, 5, 4),
                          np.linspace(-3e-3, 3e-3, 3), grid=True, want_pop=False)[0].reshape(5, 4, 3)
    for rank, full, m in res:
        assert np.array_equal(full, ref)
        assert m == pytest.approx(np.mean(np.concatenate([np.arange(10), 10 + np.arange(10)])))


def _dying_worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=5))
    if rank == 1:
        os._exit(3)  # leaves between steps, with no collective in flight
    t = torch.ones(1)
    try:
        dist.all_reduce(t)
        q.put("no error")
    except Exception as e:  # the survivor learns of the failure through the timeout
        q.put(type(e).__name__)


def test_rank_failure_is_detected_on_host():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dying_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    msg = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert msg != "no error"
    assert procs[1].exitcode == 3
