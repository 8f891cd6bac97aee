"""Shared test set-up: the `gpu` marker, import paths and oracle handles.

CPU tests (``-m "not gpu"``) cover the oracle against the reference's golden
values, the bit-exact generator, and that libcgb.so loads and exports every
symbol include/cgb.h declares.  GPU tests (``-m gpu``) are the parity tests
proper: they call libcgb.so through its C ABI and compare with the oracle
(oracle/liboracle.so) and the reference's own code (oracle/_ref/).
"""
import ctypes
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "npb-gpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_cg.json")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device")
    config.addinivalue_line("markers", "slow: larger sizes (still minutes at most)")


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    from oracle_py import Oracle
    return Oracle(ORACLE_SO)


@pytest.fixture(scope="session")
def cgb():
    import npbcg
    npbcg.lib()
    return npbcg


def ref_lib_path(cls):
    return os.path.join(REF_DIR, f"libref_{cls}.so")
