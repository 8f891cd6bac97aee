"""Multi-rank batched solving: systems are split over ranks by a greedy
stored-entry balance (npbcg.shard_systems) with no data-path collective, and
the per-system results are gathered on rank 0 (npbcg.batch_shard,
npbcg.gather_shards).  Run here as two gloo ranks on the CPU, each solving
its shard with the CPU oracle (test_gpu_shard runs the same split on the
GPU batch kernel); the gathered zetas and residuals must equal a
one-process solve of all systems."""
import os
import socket

import numpy as np
import pytest


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out_path):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "npb-gpu_b200"))
    sys.path.insert(0, os.path.join(root, "tests"))
    import npbcg
    from oracle_py import Oracle
    import datetime
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    specs = npbcg.uneven_batch_specs(nsys=10, seed=3, n_range=(150, 600), nonzer_range=(3, 6))
    mine = npbcg.batch_shard(specs, rank, world)
    o = Oracle(os.path.join(root, "oracle", "liboracle.so"))
    zeta, rnorm = [], []
    for i in mine:
        n, nz, shift, seed = specs[i]
        rs, ci, a = o.makea(n, nz, 0.1, shift, seed)
        r = o.power_iterate(rs, ci, a, shift, 5)
        zeta.append(float(r["zeta"][-1]))
        rnorm.append(float(r["rnorm"][-1]))
    g = npbcg.gather_shards({"zeta": zeta, "rnorm": rnorm, "device_ms": 1.0 + rank}, mine,
                            len(specs), dist, rank)
    if rank == 0:
        assert g["device_ms_per_rank"] == [1.0 + r for r in range(world)]
        np.save(out_path, np.stack([g["zeta"], g["rnorm"]]))
    else:
        assert g is None
    dist.barrier()
    dist.destroy_process_group()


def test_shard_balance():
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "npb-gpu_b200"))
    import npbcg
    w = [100, 90, 80, 30, 20, 10, 5, 5]
    parts = npbcg.shard_systems(w, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(w)))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)


def test_two_rank_gloo_batch(tmp_path, oracle):
    import torch.multiprocessing as mp
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "npb-gpu_b200"))
    import npbcg
    out = str(tmp_path / "zeta.npy")
    mp.start_processes(worker, args=(2, free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    specs = npbcg.uneven_batch_specs(nsys=10, seed=3, n_range=(150, 600), nonzer_range=(3, 6))
    want_z, want_r = [], []
    for n, nz, shift, seed in specs:
        rs, ci, a = oracle.makea(n, nz, 0.1, shift, seed)
        r = oracle.power_iterate(rs, ci, a, shift, 5)
        want_z.append(r["zeta"][-1])
        want_r.append(r["rnorm"][-1])
    assert np.array_equal(got[0], np.array(want_z))
    assert np.array_equal(got[1], np.array(want_r))
    # every system solved exactly once
    parts = [npbcg.batch_shard(specs, r, 2) for r in range(2)]
    assert sorted(parts[0] + parts[1]) == list(range(len(specs)))
