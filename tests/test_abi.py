"""libcgb.so loads and exports every symbol include/cgb.h declares; host-only
entry points behave on a machine without a GPU.  No compute call here."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cgb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cgb_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported(cgb):
    lib = cgb.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name


def test_binding_covers_header(cgb):
    assert set(declared_symbols()) <= set(cgb._SIGNATURES)


def test_status_strings(cgb):
    lib = cgb.lib()
    for code in range(0, 10):
        assert lib.cgb_status_string(code)
    assert lib.cgb_version() >= 100


def test_defaults(cgb):
    o = cgb.default_options()
    assert o.device == 0 and o.lanes_per_row == 0 and o.use_graph == 1
    P = cgb.SolveParams()
    cgb.lib().cgb_default_solve_params(ctypes.byref(P))
    assert P.cgitmax == 25 and P.mode == cgb.MODE_FP64


def test_create_validates_before_device(cgb):
    """A malformed CSR is rejected on the host, GPU or not."""
    lib = cgb.lib()
    rs = np.array([0, 2, 1], np.int32)
    ci = np.array([0, 1], np.int32)
    a = np.array([1.0, 2.0])
    h = ctypes.c_void_p()
    st = lib.cgb_create(2, rs, ci, a, None, ctypes.byref(h))
    assert st == cgb.ERR_BAD_MATRIX
    rs = np.array([0, 1, 2], np.int32)
    ci = np.array([0, 5], np.int32)
    assert lib.cgb_create(2, rs, ci, a, None, ctypes.byref(h)) == cgb.ERR_BAD_MATRIX
    ci = np.array([0, 1], np.int32)
    a = np.array([np.nan, 1.0])
    assert lib.cgb_create(2, rs, ci, a, None, ctypes.byref(h)) == cgb.ERR_NUMERIC


def test_no_silent_cpu_fallback(cgb):
    """Without a GPU, the solver reports NO_DEVICE instead of computing on the CPU."""
    import torch
    if torch.cuda.is_available():
        import pytest
        pytest.skip("a GPU is present")
    rs, ci, a = cgb.makea(100, 5, 0.1, 10.0)
    h = ctypes.c_void_p()
    st = cgb.lib().cgb_create(100, rs, ci, a, None, ctypes.byref(h))
    assert st == cgb.ERR_NO_DEVICE


def test_validation_reports_first_bad_entry_of_large_csr(cgb):
    """The entry checks run in parallel chunks; the reported entry is still
    the first bad one (lowest index), across chunk boundaries."""
    lib = cgb.lib()
    n, per_row = 1000, 3000
    rs = (np.arange(n + 1, dtype=np.int32) * per_row).astype(np.int32)
    ci = np.tile(np.arange(per_row, dtype=np.int32) % n, n)
    a = np.ones(n * per_row)
    ci[2_500_000] = n          # out of range, later chunk
    a[1_900_000] = np.nan      # not finite, earlier chunk
    h = ctypes.c_void_p()
    assert lib.cgb_create(n, rs, ci, a, None, ctypes.byref(h)) == cgb.ERR_NUMERIC
    assert b"1900000" in lib.cgb_last_error()
    a[1_900_000] = 1.0
    assert lib.cgb_create(n, rs, ci, a, None, ctypes.byref(h)) == cgb.ERR_BAD_MATRIX
    assert b"2500000" in lib.cgb_last_error()
