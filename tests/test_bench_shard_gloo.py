"""The multi-rank path of bench.py's batched section, on the CPU.

Under torchrun bench.py shards the batched workload over the ranks
(npbcg.batch_shard), each rank solves its shard, and rank 0 gathers the
per-system results (npbcg.gather_shards) and the ranks' device times.  This
test runs that code (bench.batched_section) as two gloo ranks with a
stand-in for the GPU batch solver that solves each system with the CPU
oracle, so the sharding, the gather and the aggregate figures are checked
without a GPU; the GPU batch kernel itself is covered by test_gpu_batch and
test_gpu_shard.
"""
import json
import os
import socket
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NSYS = 6


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class FakeGnn:
    def __init__(self, device=0):
        pass

    def load(self, path=None):
        pass

    def close(self):
        pass


def fake_npbcg(npbcg, oracle, learned):
    """npbcg with small systems and an oracle-backed Batch (no GPU); with
    `learned` the learned rows run too (the stand-in solves them alike)."""

    class OracleBatch:
        def __init__(self, systems, shifts, device=0):
            self.systems, self.shifts = systems, list(shifts)

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def tune(self, **kw):
            return {"block": 0, "thresholds": (0, 0, 0), "best_ms": 1.0}

        def attach_learned(self, model):
            pass

        def attach_identity(self):
            pass

        def fallbacks(self):
            return np.zeros(len(self.systems), np.int32)

        def solve(self, niter=15, **kw):
            z, r = [], []
            for (rs, ci, a), sh in zip(self.systems, self.shifts):
                out = oracle.power_iterate(rs, ci, a, sh, niter)
                z.append(out["zeta"][-1])
                r.append(out["rnorm"][-1])
            k = len(self.systems)
            return dict(zeta=np.array(z), rnorm=np.array(r), iters=np.full(k, 25 * niter, np.int32),
                        status=np.zeros(k, np.int32), device_ms=1.0 + 0.5 * k)

    fake = types.SimpleNamespace(**{k: getattr(npbcg, k) for k in dir(npbcg) if not k.startswith("__")})
    fake.Batch = OracleBatch
    fake.Gnn = FakeGnn
    fake.WEIGHTS_PATH = os.path.abspath(__file__) if learned else os.path.join(ROOT, "no-weights.f32")
    fake.uneven_batch_specs = lambda nsys=NSYS: npbcg.uneven_batch_specs(
        nsys=nsys, seed=5, n_range=(150, 500), nonzer_range=(3, 5))
    return fake


def worker(rank, world, port, out_path, learned):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "npb-gpu_b200"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import bench
    import npbcg
    from oracle_py import Oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    fake = fake_npbcg(npbcg, Oracle(os.path.join(ROOT, "oracle", "liboracle.so")), learned)
    out = bench.batched_section(fake, 0, nsys=NSYS, niter=3, rank=rank, world=world, dist=dist)
    if rank == 0:
        with open(out_path, "w") as f:
            json.dump(out, f)
    else:
        assert out is None
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("learned", [False, True])
def test_bench_batched_section_two_ranks(tmp_path, learned):
    import torch.multiprocessing as mp
    out_path = str(tmp_path / "batched.json")
    mp.start_processes(worker, args=(2, free_port(), out_path, learned), nprocs=2, join=True,
                       start_method="spawn")
    with open(out_path) as f:
        out = json.load(f)
    sh = out["sharding"]
    assert sh["ranks"] == 2 and sum(sh["systems_per_rank"]) == NSYS
    assert min(sh["systems_per_rank"]) >= 1
    # every system solved once and compared with itself (the stand-in's FP64
    # and mixed runs are the same oracle solve)
    assert out["within_1e-10_all"] == NSYS
    assert out["mixed"]["refit_in_fp64"] == 0
    # aggregate rate: all systems over the slowest rank's device time
    slowest = max(sh["fp64_ms_per_rank"])
    assert abs(out["fp64_reference"]["solves_per_s"] - NSYS / slowest * 1e3) < 1e-9
    if not learned:
        assert out["mixed_learned"] is None  # no weights: the learned rows are left out
    else:
        ml = out["mixed_learned"]
        assert ml["within_1e-10_all"] == NSYS and ml["refit_in_fp64"] == 0
        assert ml["systems_with_plain_cg_fallback"] == 0
        assert ml["identity_factor"]["inner_iterations_preconditioned_systems"] == 25 * 3 * NSYS
