"""One system split by rows over ranks (cgb_part), on the CPU.

The GPU path (part.cu) keeps rank r's rows [r m, min((r+1) m, n)),
m = ceil(n / world), and per CG step exchanges the search vector once (an
all-gather of the ranks' row blocks) and two scalars (all-reduces of p.q and
r.r); after the CG steps it gathers z once for ||x - A z|| and reduces
(||x - A z||^2, x.z, z.z) together.  Here two and three gloo ranks run that
exchange plan step for step in numpy, on the row blocks the library's own
split gives (npbcg.part_rows, npbcg.row_block), and the trace must match the
reference algorithm (the oracle's power iteration) to the reference's
verification epsilon.  The kernels themselves are covered by test_gpu_part.
"""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_row_blocks_reassemble(cgb):
    rs, ci, a = cgb.makea(1001, 5, cgb.RCOND, 10.0)
    for world in (1, 2, 3, 4, 7):
        m = -(-1001 // world)
        bounds = [cgb.part_rows(1001, world, r) for r in range(world)]
        assert bounds[0][0] == 0 and bounds[-1][1] == 1001
        assert all(b[1] == c[0] for b, c in zip(bounds, bounds[1:]))
        assert all(b[1] - b[0] == m for b in bounds[:-1])
        blocks = [cgb.row_block(rs, ci, a, *b) for b in bounds]
        assert all(b[0][0] == 0 for b in blocks)
        got_rs = np.concatenate([[0]] + [b[0][1:] + sum(len(x[1]) for x in blocks[:i])
                                         for i, b in enumerate(blocks)])
        assert np.array_equal(got_rs, rs)
        assert np.array_equal(np.concatenate([b[1] for b in blocks]), ci)
        assert np.array_equal(np.concatenate([b[2] for b in blocks]), a)


def test_part_rows_rejects_bad_worlds(cgb):
    for args in ((0, 1, 0), (10, 0, 0), (10, 2, 2), (10, 2, -1)):
        with pytest.raises(cgb.CgbError) as e:
            cgb.part_rows(*args)
        assert e.value.status == cgb.ERR_INVALID


def test_part_needs_a_device(cgb):
    """No CPU path: without a GPU the partitioned solver reports NO_DEVICE."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    rs, ci, a = cgb.makea(100, 5, cgb.RCOND, 10.0)
    with pytest.raises(cgb.CgbError) as e:
        cgb.Part(rs, ci, a, world=2, rank=0)
    assert e.value.status == cgb.ERR_NO_DEVICE


def spmv(rs, ci, a, v):
    rows = np.repeat(np.arange(len(rs) - 1), np.diff(rs))
    return np.bincount(rows, weights=a * v[ci], minlength=len(rs) - 1)


def partitioned_power(rs, ci, a, n, world, rank, dist, shift, niter, cgitmax):
    """The GPU path's exchange plan, one numpy step per kernel."""
    import torch
    m = -(-n // world)
    own = len(rs) - 1

    def allreduce(vals):
        t = torch.tensor(vals, dtype=torch.float64)
        dist.all_reduce(t)
        return t.numpy()

    def allgather(block):
        buf = np.zeros(m)
        buf[:own] = block
        out = [torch.zeros(m, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(out, torch.from_numpy(buf))
        return torch.cat(out).numpy()[:n]

    x = np.ones(own)
    zeta, rnorm = [], []
    for _ in range(niter):
        z, r, p = np.zeros(own), x.copy(), x.copy()
        rho = allreduce([x @ x])[0]
        pfull = allgather(p)
        for _ in range(cgitmax):
            q = spmv(rs, ci, a, pfull)
            alpha = rho / allreduce([p @ q])[0]
            z = z + alpha * p
            r = r - alpha * q
            rho_new = allreduce([r @ r])[0]
            p = r + (rho_new / rho) * p
            rho = rho_new
            pfull = allgather(p)
        az = spmv(rs, ci, a, allgather(z))
        res, xz, zz = allreduce([np.sum((x - az) ** 2), x @ z, z @ z])
        zeta.append(shift + 1.0 / xz)
        rnorm.append(np.sqrt(res))
        x = z / np.sqrt(zz)
    return np.array(zeta), np.array(rnorm)


def worker(rank, world, port, out_path):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "npb-gpu_b200"))
    import npbcg
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    rs, ci, a = npbcg.makea(1400, 7, npbcg.RCOND, 10.0)
    block = npbcg.row_block(rs, ci, a, *npbcg.part_rows(1400, world, rank))
    zeta, rnorm = partitioned_power(*block, 1400, world, rank, dist, 10.0, 15, 25)
    if rank == 0:
        np.save(out_path, np.stack([zeta, rnorm]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_plan_matches_reference(tmp_path, golden, world):
    import torch.multiprocessing as mp
    out = str(tmp_path / "trace.npy")
    mp.start_processes(worker, args=(world, free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    zeta, rnorm = np.load(out)
    e = golden["S"]["seeds"]["314159265.0"]
    ref = np.array(e["zeta"])
    assert np.max(np.abs(zeta - ref) / ref) <= 1e-10
    assert np.max(np.abs(rnorm - np.array(e["rnorm"]))) <= 1e-10
    assert abs(zeta[-1] - golden["verify"]["S"]) / golden["verify"]["S"] <= 1e-10


def test_nccl_choice_agrees_with_torch():
    """libcgb loads NCCL on first use; a process holds one libnccl.so.2, so
    loading a different one than torch's would leave torch unable to load
    its own.  In a fresh process: libcgb's NCCL first, torch afterwards."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import npbcg; npbcg.nccl_unique_id(); "
            "import torch.distributed; print('ok')" % os.path.join(ROOT, "npb-gpu_b200"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]
