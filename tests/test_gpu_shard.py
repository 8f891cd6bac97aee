"""Batched systems sharded over ranks, on the GPU batch kernel (cgb_batch).

Two ranks (gloo process group for the gather) each build and solve their
shard of an uneven batch (npbcg.batch_shard: greedy by size, no exchange
during the solve) with libcgb's persistent batch kernel, and rank 0
gathers the per-system results (npbcg.gather_shards).  This machine has one
GPU, so both ranks use cuda:0 and take turns on it (a gloo barrier between
turns): each rank's launch runs alone, none waits on another's kernels.
The gathered zetas must equal, bit for bit, a one-process batch of all
systems (every system on one CTA -- no teams -- so a system's arithmetic
does not depend on which batch it is in), in the FP64 reference algorithm
and in the mixed mode with its FP64 fallback.
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPEC = dict(nsys=12, seed=11, n_range=(1400, 4000))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def solve(npbcg, specs, idx):
    systems = [npbcg.makea(specs[i][0], specs[i][1], npbcg.RCOND, specs[i][2], specs[i][3])
               for i in idx]
    with npbcg.Batch(systems, [specs[i][2] for i in idx], device=0) as b:
        b.set_team_frac(0.0)
        ref = b.solve(niter=15)
        mix = b.solve(niter=15, mode=npbcg.MODE_MIXED, tol=1e-12, cgitmax=200)
    return {"zeta": ref["zeta"], "rnorm": ref["rnorm"], "zeta_mixed": mix["zeta"],
            "status_mixed": mix["status"], "device_ms": ref["device_ms"]}


def worker(rank, world, port, out_path):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "npb-gpu_b200"))
    import npbcg
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    specs = npbcg.uneven_batch_specs(**SPEC)
    mine = npbcg.batch_shard(specs, rank, world)
    local = None
    for turn in range(world):  # one GPU: the ranks' launches take turns
        if turn == rank:
            local = solve(npbcg, specs, mine)
        dist.barrier()
    g = npbcg.gather_shards(local, mine, len(specs), dist, rank)
    if rank == 0:
        np.savez(out_path, **{k: v for k, v in g.items() if k != "device_ms_per_rank"},
                 ms=np.array(g["device_ms_per_rank"]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_match_one_batch(tmp_path, cgb):
    import torch.multiprocessing as mp
    out = str(tmp_path / "gathered.npz")
    mp.start_processes(worker, args=(2, free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    specs = cgb.uneven_batch_specs(**SPEC)
    parts = [cgb.batch_shard(specs, r, 2) for r in range(2)]
    assert parts[0] and parts[1]
    assert sorted(parts[0] + parts[1]) == list(range(len(specs)))
    want = solve(cgb, specs, list(range(len(specs))))
    assert np.array_equal(got["zeta"], want["zeta"])
    assert np.array_equal(got["rnorm"], want["rnorm"])
    assert np.array_equal(got["zeta_mixed"], want["zeta_mixed"])
    assert np.array_equal(got["status_mixed"], want["status_mixed"])
    assert np.all(got["ms"] > 0)
