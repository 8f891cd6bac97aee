"""One system split by rows over ranks (cgb_part), on the GPU.

The ranks of a world are driven from this process on one device
(cgb_part_group_power_iterate): the same kernels and the same exchanges as
one rank per GPU over NCCL, with the all-gather of the search vector done by
device copies and the scalar all-reduces by a summing kernel.  A world of
one also runs through NCCL itself (a one-rank communicator).  Each rank's
sums are ordered differently from the single-GPU solver's, so the bar is the
reference's verification epsilon: zeta relative 1e-10 and rnorm absolute
1e-10 against the reference's own traces (cg.cu:534-537), and the NPB
verification value of the class.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = {"S": (1400, 7, 15, 10.0), "W": (7000, 8, 15, 12.0), "A": (14000, 11, 15, 20.0),
          "B": (75000, 13, 75, 60.0), "C": (150000, 15, 75, 110.0)}
VERIFY = {"S": 8.5971775078648, "W": 10.362595087124, "A": 17.130235054029,
          "B": 22.712745482631, "C": 28.973605592845}


def world_of(cgb, csr, k):
    return [cgb.Part(*csr, world=k, rank=r) for r in range(k)]


def check_trace(out, e, cls):
    ref_zeta = np.array(e["zeta"])
    assert np.max(np.abs(out["zeta"] - ref_zeta) / np.abs(ref_zeta)) <= 1e-10
    assert np.max(np.abs(out["rnorm"] - np.array(e["rnorm"]))) <= 1e-10
    assert abs(out["zeta"][-1] - VERIFY[cls]) / VERIFY[cls] <= 1e-10


@pytest.mark.parametrize("cls", ["S", "W", "A"])
@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_group_matches_reference(cgb, golden, cls, k):
    n, nonzer, niter, shift = PARAMS[cls]
    csr = cgb.makea(n, nonzer, cgb.RCOND, shift)
    parts = world_of(cgb, csr, k)
    out = cgb.group_power_iterate(parts, niter, shift)
    check_trace(out, golden[cls]["seeds"]["314159265.0"], cls)
    assert out["device_ms"] > 0
    for p in parts:
        p.close()


def test_group_class_b_three_ranks(cgb, golden):
    n, nonzer, niter, shift = PARAMS["B"]
    csr = cgb.makea(n, nonzer, cgb.RCOND, shift)
    parts = world_of(cgb, csr, 3)
    check_trace(cgb.group_power_iterate(parts, niter, shift), golden["B"]["seeds"]["314159265.0"], "B")


@pytest.mark.slow
def test_group_class_c_two_ranks(cgb, golden):
    n, nonzer, niter, shift = PARAMS["C"]
    csr = cgb.makea(n, nonzer, cgb.RCOND, shift)
    parts = world_of(cgb, csr, 2)
    check_trace(cgb.group_power_iterate(parts, niter, shift), golden["C"]["seeds"]["314159265.0"], "C")


def test_repeatable_bitwise(cgb):
    n, nonzer, niter, shift = PARAMS["W"]
    csr = cgb.makea(n, nonzer, cgb.RCOND, shift)
    parts = world_of(cgb, csr, 3)
    a = cgb.group_power_iterate(parts, niter, shift)
    b = cgb.group_power_iterate(parts, niter, shift)
    assert np.array_equal(a["zeta"], b["zeta"]) and np.array_equal(a["rnorm"], b["rnorm"])


def test_world_of_one_over_nccl_equals_group(cgb, golden):
    """A one-rank NCCL communicator: the all-reduce of one rank's value is
    that value, so the trace is the group path's bit for bit."""
    n, nonzer, niter, shift = PARAMS["A"]
    csr = cgb.makea(n, nonzer, cgb.RCOND, shift)
    with cgb.Part(*csr, world=1, rank=0, nccl_id=cgb.nccl_unique_id()) as p:
        nc = p.power_iterate(niter, shift)
    with cgb.Part(*csr) as q:
        alone = q.power_iterate(niter, shift)
        grp = cgb.group_power_iterate([q], niter, shift)
    assert np.array_equal(nc["zeta"], grp["zeta"]) and np.array_equal(nc["rnorm"], grp["rnorm"])
    assert np.array_equal(alone["zeta"], grp["zeta"])
    check_trace(nc, golden["A"]["seeds"]["314159265.0"], "A")


def test_other_cgitmax(cgb, oracle):
    """cgitmax other than 25 against the oracle's power iteration."""
    n, nonzer, niter, shift = PARAMS["S"]
    csr = cgb.makea(n, nonzer, cgb.RCOND, shift)
    parts = world_of(cgb, csr, 2)
    for cgitmax in (1, 7, 40):
        got = cgb.group_power_iterate(parts, 4, shift, cgitmax=cgitmax)
        want = oracle.power_iterate(*csr, shift, 4, cgitmax=cgitmax)
        assert np.max(np.abs(got["zeta"] - want["zeta"]) / np.abs(want["zeta"])) <= 1e-10
        assert np.max(np.abs(got["rnorm"] - want["rnorm"])) <= 1e-10


def test_ragged_last_rank(cgb, oracle):
    """n not a multiple of the world: the last rank owns fewer rows."""
    csr = cgb.makea(1001, 5, cgb.RCOND, 10.0)
    parts = world_of(cgb, csr, 4)
    assert [p.rows for p in parts] == [(0, 251), (251, 502), (502, 753), (753, 1001)]
    got = cgb.group_power_iterate(parts, 5, 10.0)
    want = oracle.power_iterate(*csr, 10.0, 5)
    assert np.max(np.abs(got["zeta"] - want["zeta"]) / np.abs(want["zeta"])) <= 1e-10


def test_invalid_worlds(cgb):
    csr = cgb.makea(1400, 7, cgb.RCOND, 10.0)
    small = cgb.makea(5, 2, cgb.RCOND, 10.0)
    with pytest.raises(cgb.CgbError) as e:  # rank 6 of 7 owns no row of n = 5
        cgb.Part(*small, world=7, rank=6)
    assert e.value.status == cgb.ERR_INVALID
    p0, p1 = world_of(cgb, csr, 2)
    with pytest.raises(cgb.CgbError) as e:  # a rank of two without a communicator
        p0.power_iterate(2, 10.0)
    assert e.value.status == cgb.ERR_STATE
    with pytest.raises(cgb.CgbError) as e:  # ranks out of order
        cgb.group_power_iterate([p1, p0], 2, 10.0)
    assert e.value.status == cgb.ERR_INVALID
    with pytest.raises(cgb.CgbError) as e:  # not the whole world
        cgb.group_power_iterate([p0], 2, 10.0)
    assert e.value.status == cgb.ERR_INVALID
    rs, ci, a = csr
    bad = ci.copy()
    bad[3] = 1400
    with pytest.raises(cgb.CgbError) as e:
        cgb.Part(rs, bad, a, world=2, rank=0)
    assert e.value.status == cgb.ERR_BAD_MATRIX


def test_generated_blocks_equal_uploaded(cgb):
    """Each rank's rows generated on the device are the rows of the host
    generator's matrix: the traces agree bit for bit with parts made from
    the host CSR (the same kernels on the same data)."""
    n, nonzer, niter, shift = PARAMS["A"]
    csr = cgb.makea(n, nonzer, cgb.RCOND, shift)
    up = world_of(cgb, csr, 3)
    gen = [cgb.Part.generated(n, nonzer, shift, world=3, rank=r) for r in range(3)]
    a = cgb.group_power_iterate(up, 4, shift)
    b = cgb.group_power_iterate(gen, 4, shift)
    assert np.array_equal(a["zeta"], b["zeta"]) and np.array_equal(a["rnorm"], b["rnorm"])


@pytest.mark.slow
def test_class_d_generated_two_ranks(cgb):
    """Class D (n = 1.5 M, 100 outer steps) from generated row blocks: the
    NPB verification value (cg.cu:389-390) within the reference's epsilon."""
    n, nonzer, niter, shift = 1500000, 21, 100, 500.0
    parts = [cgb.Part.generated(n, nonzer, shift, world=2, rank=r) for r in range(2)]
    out = cgb.group_power_iterate(parts, niter, shift)
    assert abs(out["zeta"][-1] - 52.514532105794) / 52.514532105794 <= 1e-10
    assert np.all(out["rnorm"] < 1e-10)
