"""The multi-rank path of bench.py's row-partitioned section, on the CPU.

Under torchrun every rank builds its row block of one class-D system with
the NCCL id rank 0 made (broadcast over the process group), all ranks solve
together, and rank 0 reports the slowest rank's device time and the sum of
the blocks' entries.  Two gloo ranks run that code (bench.row_partitioned_
section) here with a stand-in for npbcg.Part that records what it was given;
the GPU solver itself is covered by test_gpu_part.
"""
import json
import os
import socket
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def fake_npbcg(npbcg, rank, seen, fail_rank=-1):
    class FakePart:
        @classmethod
        def generated(cls, n, nonzer, shift, world=1, rank=0, nccl_id=None, device=0):
            assert nccl_id is None  # the communicator is joined after every block is built
            if rank == fail_rank:
                raise npbcg.CgbError(npbcg.ERR_NOMEM, "out of device memory")
            seen.update(n=n, nonzer=nonzer, shift=shift, world=world, rank=rank)
            self = cls()
            self.rank = rank
            return self

        def join(self, nccl_id):
            seen["id"] = nccl_id.hex()

        def set_wait_limit(self, seconds):
            seen["limit"] = seconds

        @property
        def nnz(self):
            return 1000 + self.rank

        def power_iterate(self, niter, shift, cgitmax=25):
            import numpy as np
            seen.setdefault("calls", []).append(niter)
            return dict(zeta=np.full(niter, 52.514532105794), rnorm=np.zeros(niter),
                        device_ms=100.0 + 10.0 * self.rank)

        def close(self):
            seen["closed"] = True

    fake = types.SimpleNamespace(**{k: getattr(npbcg, k) for k in dir(npbcg) if not k.startswith("__")})
    fake.Part = FakePart
    fake.nccl_unique_id = lambda: bytes([rank + 7]) * 128
    return fake


def worker(rank, world, port, out_path, fail_rank=-1):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "npb-gpu_b200"))
    import bench
    import npbcg
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    seen = {}
    out = bench.row_partitioned_section(fake_npbcg(npbcg, rank, seen, fail_rank), 0, rank, world,
                                        dist)
    with open(f"{out_path}.{rank}", "w") as f:
        json.dump({"out": out, "seen": seen}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_row_partitioned_section_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    out_path = str(tmp_path / "part.json")
    mp.start_processes(worker, args=(2, free_port(), out_path), nprocs=2, join=True,
                       start_method="spawn")
    got = [json.load(open(f"{out_path}.{r}")) for r in range(2)]
    # rank 0's id reached every rank; each built its own block of class D
    assert got[0]["seen"]["id"] == got[1]["seen"]["id"] == (bytes([7]) * 128).hex()
    for r in range(2):
        s = got[r]["seen"]
        assert (s["n"], s["nonzer"], s["shift"], s["world"], s["rank"]) == (1500000, 21, 500.0, 2, r)
        assert s["calls"] == [1, 100] and s["closed"]
    assert got[1]["out"] is None
    o = got[0]["out"]
    assert o["ranks"] == 2 and o["seconds"] == pytest.approx(0.110)  # the slowest rank
    assert "nnz=2001" in o["what"] and o["verified"]


def test_row_partitioned_section_rank_fails_to_build(tmp_path):
    """A rank that cannot build its block: no rank joins the communicator or
    enters a collective of the solve; rank 0 reports the section unavailable."""
    import torch.multiprocessing as mp
    out_path = str(tmp_path / "part.json")
    mp.start_processes(worker, args=(2, free_port(), out_path, 1), nprocs=2, join=True,
                       start_method="spawn")
    got = [json.load(open(f"{out_path}.{r}")) for r in range(2)]
    assert "unavailable" in got[0]["out"] and got[1]["out"] is None
    for r in range(2):
        assert "id" not in got[r]["seen"] and "calls" not in got[r]["seen"]
    assert got[0]["seen"].get("closed")  # rank 0 built its block and released it
