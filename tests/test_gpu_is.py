"""GPU parity of NPB IS (npb-gpu_b200/csrc/is.cu) through the C ABI.

Against the oracle (oracle/is_oracle.c, which verifies against the
reference's own test-key tables): the generated keys bit for bit, the last
ranking pass's counts exactly, the sorted keys exactly.  Every class S-C
(D marked slow) must pass all 51 of the reference's checks (is.cu:157-190,
rank_gpu_kernel_7, full_verify), and a second run must give the same.
"""
import numpy as np
import pytest

from test_is_oracle import IS_CLASSES as ORACLE_TABLES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cls", ["S", "W"])
def test_is_matches_oracle(cgb, oracle, cls):
    tl, ml, ti, tr = ORACLE_TABLES[cls]
    with cgb.IntSort(cls) as s:
        keys0 = s.read("keys")
        assert np.array_equal(keys0, oracle.is_keys(tl, ml))
        out = s.run()
        below = s.read("below")
        srt = s.read("sorted")
        keys = s.read("keys")
    passed, incl = oracle.is_run(cls, tl, ml, ti, tr, counts=True)
    assert out["passed"] == passed == 51
    # after the run's full check the counts hold, per value, the keys below it
    assert below[0] == 0 and np.array_equal(below[1:].astype(np.int64), incl[:-1])
    assert np.array_equal(srt, np.sort(keys))


@pytest.mark.parametrize("cls", ["S", "W", "A", "B", "C", pytest.param("D", marks=pytest.mark.slow)])
def test_is_class_verifies(cgb, cls):
    with cgb.IntSort(cls) as s:
        a = s.run()
        b = s.run()
    assert a["passed"] == cgb.IS_PASSED and b["passed"] == cgb.IS_PASSED
    assert a["device_ms"] > 0


def test_is_custom_size_and_invalid(cgb):
    with cgb.IntSort("U", 18, 12) as s:
        out = s.run()
        keys, srt = s.read("keys"), s.read("sorted")
    assert out["passed"] == 1  # no class table: only the full check
    assert np.array_equal(srt, np.sort(keys))
    with pytest.raises(cgb.CgbError) as e:
        cgb.lib()  # the class's sizes are fixed
        s = cgb.IntSort.__new__(cgb.IntSort)
        h = __import__("ctypes").c_void_p()
        cgb._check(cgb.lib().cgb_is_create(0, b"S", 20, 11, __import__("ctypes").byref(h)))
    assert e.value.status == cgb.ERR_INVALID


def test_reference_gpu_is_agrees(cgb):
    """The reference's own IS kernels (compiled from its sources into
    oracle/_ref) on the same GPU pass all 51 of their checks, as ours do."""
    import os
    from conftest import REF_DIR
    from oracle_py import RefIsLib
    path = os.path.join(REF_DIR, "libref_is_S.so")
    if not os.path.exists(path):
        pytest.skip("the reference's IS library was not built (make -C oracle)")
    ref = RefIsLib(path).gpu()
    assert ref["passed"] == cgb.IS_PASSED and ref["seconds"] > 0
    with cgb.IntSort("S") as s:
        assert s.run()["passed"] == cgb.IS_PASSED


@pytest.mark.parametrize("total_log2,max_log2", [(12, 8), (12, 26), (16, 20), (20, 10), (14, 14), (22, 8),
                                                 (24, 8)])
def test_is_bucket_edges_count_exactly(cgb, total_log2, max_log2):
    """Custom sizes at the bucket pass's edges: one bucket of 256 values
    (2^8), thousands of nearly empty buckets (2^12 keys below 2^26), runs of
    keys shorter than the grid (2^12 keys: CTAs with no keys), square sizes,
    and values holding tens of thousands of keys each (2^22 and 2^24 keys
    below 2^8).
    After a run the counts below each value and the sorted keys must equal
    an independent count of the keys the run left."""
    with cgb.IntSort("U", total_log2, max_log2) as s:
        out = s.run()
        keys, below, srt = s.read("keys"), s.read("below"), s.read("sorted")
    maxk = 1 << max_log2
    assert keys.min() >= 0 and keys.max() < maxk
    counts = np.bincount(keys, minlength=maxk)
    want = np.concatenate(([0], np.cumsum(counts)[:-1]))
    assert np.array_equal(below.astype(np.int64), want)
    assert np.array_equal(srt, np.sort(keys))
    assert out["passed"] == 1


def test_is_instances_of_different_sizes_coexist(cgb):
    """Two live instances, the larger made first: the smaller one's set-up
    must not leave the larger one unable to launch (the kernels' shared
    memory limit is per process)."""
    with cgb.IntSort("W") as big:
        with cgb.IntSort("S") as small:
            assert small.run()["passed"] == cgb.IS_PASSED
            assert big.run()["passed"] == cgb.IS_PASSED
        assert big.run()["passed"] == cgb.IS_PASSED
    with cgb.IntSort("U", 16, 27) as wide:  # 4096 buckets: the largest scatter tables
        with cgb.IntSort("U", 16, 10) as narrow:
            assert narrow.run()["passed"] == 1
            assert wide.run()["passed"] == 1
