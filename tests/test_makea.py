"""The product generator (cgb_makea in libcgb.so) is bit-exact with the
reference makea (cg.cu:1303-1368 + sparse :1611-1785).  Host code: CPU only."""
import ctypes

import numpy as np
import pytest

PARAMS = {"S": (1400, 7, 15, 10.0), "W": (7000, 8, 15, 12.0), "A": (14000, 11, 15, 20.0),
          "B": (75000, 13, 75, 60.0), "C": (150000, 15, 75, 110.0)}


@pytest.mark.parametrize("cls", ["S", "W", "A", "B"])
def test_makea_bit_exact(cgb, oracle, golden, cls):
    n, nonzer, _, shift = PARAMS[cls]
    for key, e in golden[cls]["seeds"].items():
        rs, ci, a = cgb.makea(n, nonzer, 0.1, shift, e["seed"])
        assert len(a) == e["nnz"]
        assert oracle.csr_hash(rs, ci, a) == e["csr_hash"]


@pytest.mark.slow
def test_makea_class_c_bit_exact(cgb, oracle, golden):
    if "C" not in golden:
        pytest.skip("class C golden not generated")
    n, nonzer, _, shift = PARAMS["C"]
    e = golden["C"]["seeds"]["314159265.0"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    assert len(a) == e["nnz"]
    assert oracle.csr_hash(rs, ci, a) == e["csr_hash"]


@pytest.mark.parametrize("seed", [3.0, 12345.0 * 2 + 1, 2.0 ** 46 - 1, 987654321.0])
@pytest.mark.parametrize("shape", [(50, 3, 2.0), (777, 5, 7.5), (2000, 9, 11.0)])
def test_makea_matches_oracle_any_size(cgb, oracle, seed, shape):
    n, nonzer, shift = shape
    got = cgb.makea(n, nonzer, 0.1, shift, seed)
    want = oracle.makea(n, nonzer, 0.1, shift, seed)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_makea_rejects_bad_arguments(cgb):
    lib = cgb.lib()
    rs = np.zeros(101, np.int32)
    ci = np.zeros(100 * 64, np.int32)
    a = np.zeros(100 * 64)
    nnz = ctypes.c_longlong()
    for seed in (2.0, 1.0, 0.0, -5.0, 2.0 ** 46 + 1, 3.5):   # even, out of range, fractional
        assert lib.cgb_makea(100, 7, 0.1, 10.0, seed, rs, ci, a, len(a), ctypes.byref(nnz)) == cgb.ERR_INVALID
    assert lib.cgb_makea(1, 7, 0.1, 10.0, 3.0, rs, ci, a, len(a), ctypes.byref(nnz)) == cgb.ERR_INVALID
    assert lib.cgb_makea(100, 100, 0.1, 10.0, 3.0, rs, ci, a, len(a), ctypes.byref(nnz)) == cgb.ERR_INVALID
    assert lib.cgb_makea(100, 7, 0.0, 10.0, 3.0, rs, ci, a, len(a), ctypes.byref(nnz)) == cgb.ERR_INVALID
    assert b"seed" in lib.cgb_last_error() or b"rcond" in lib.cgb_last_error()


def test_makea_capacity_reported(cgb):
    lib = cgb.lib()
    n, nonzer = 200, 5
    rs = np.zeros(n + 1, np.int32)
    ci = np.zeros(10, np.int32)
    a = np.zeros(10)
    nnz = ctypes.c_longlong()
    st = lib.cgb_makea(n, nonzer, 0.1, 10.0, 314159265.0, rs, ci, a, 10, ctypes.byref(nnz))
    assert st == cgb.ERR_CAPACITY
    full = cgb.makea(n, nonzer, 0.1, 10.0)
    assert nnz.value == len(full[2])
    assert nnz.value <= cgb.nz_bound(n, nonzer)


def test_makea_matrix_properties(cgb):
    n, nonzer, shift = 1400, 7, 10.0
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    # symmetric up to rounding: the reference forms entry (j, k) as
    # aelt[k] * (size * aelt[j]), so (j, k) and (k, j) may differ in the last bit
    import scipy.sparse as sp
    A = sp.csr_matrix((a, ci, rs), shape=(n, n))
    assert abs(A - A.T).max() <= 4e-16 * abs(A).max()
    assert (A != A.T).nnz > 0
    d = A.diagonal()
    assert np.all(d < 0)  # shift dominates: negative definite classes
