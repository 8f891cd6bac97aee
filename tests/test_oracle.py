"""The CPU oracle against the reference's own outputs (CPU only).

Pins oracle/cg_oracle.c: its CSR hash, nnz and per-step zeta / rnorm traces
must equal what the reference code produced (tests/golden/reference_cg.json,
written by tests/golden/make_golden.py from oracle/_ref), and its final zeta
must pass the reference's own verification (cg.cu:373-396, :534-552).
"""
import os

import numpy as np
import pytest

from conftest import ref_lib_path

VERIFY = {"S": 8.5971775078648, "W": 10.362595087124, "A": 17.130235054029,
          "B": 22.712745482631, "C": 28.973605592845}
PARAMS = {"S": (1400, 7, 15, 10.0), "W": (7000, 8, 15, 12.0), "A": (14000, 11, 15, 20.0),
          "B": (75000, 13, 75, 60.0), "C": (150000, 15, 75, 110.0)}


def test_randlc_sequence(oracle):
    """x <- 5^13 x mod 2^46: the oracle's 23-bit split equals exact integer math."""
    import ctypes
    x = ctypes.c_double(314159265.0)
    xi = 314159265
    for _ in range(2000):
        v = oracle.lib.orc_randlc(ctypes.byref(x), 1220703125.0)
        xi = (xi * 1220703125) % (1 << 46)
        assert x.value == float(xi)
        assert v == xi * 2.0 ** -46


def test_golden_verify_values_match_reference_table(golden):
    for cls, z in VERIFY.items():
        assert golden["verify"][cls] == z


@pytest.mark.parametrize("cls", ["S", "W", "A"])
def test_oracle_makea_matches_reference(oracle, golden, cls):
    n, nonzer, _, shift = PARAMS[cls]
    for key, e in golden[cls]["seeds"].items():
        rs, ci, a = oracle.makea(n, nonzer, 0.1, shift, e["seed"])
        assert len(a) == e["nnz"]
        assert oracle.csr_hash(rs, ci, a) == e["csr_hash"]
        # CSR invariants: sorted unique columns per row, diagonal present
        for j in range(0, n, max(1, n // 50)):
            row = ci[rs[j]:rs[j + 1]]
            assert np.all(np.diff(row) > 0)
            assert j in row


@pytest.mark.parametrize("cls", ["S", "W", "A"])
def test_oracle_power_trace_matches_reference(oracle, golden, cls):
    n, nonzer, niter, shift = PARAMS[cls]
    e = golden[cls]["seeds"]["314159265.0"]
    rs, ci, a = oracle.makea(n, nonzer, 0.1, shift)
    out = oracle.power_iterate(rs, ci, a, shift, niter)
    # same operations in the same order as the reference: bit-identical traces
    assert out["zeta"].tolist() == e["zeta"]
    assert out["rnorm"].tolist() == e["rnorm"]
    assert abs(out["zeta"][-1] - VERIFY[cls]) / VERIFY[cls] <= 1e-10


def test_oracle_other_seeds_traces(oracle, golden):
    for cls in ("S", "A"):
        n, nonzer, niter, shift = PARAMS[cls]
        for key, e in golden[cls]["seeds"].items():
            if key == "314159265.0":
                continue
            rs, ci, a = oracle.makea(n, nonzer, 0.1, shift, e["seed"])
            out = oracle.power_iterate(rs, ci, a, shift, niter)
            assert out["zeta"].tolist() == e["zeta"]


def test_oracle_openmp_agrees(oracle):
    n, nonzer, niter, shift = PARAMS["A"]
    rs, ci, a = oracle.makea(n, nonzer, 0.1, shift)
    serial = oracle.power_iterate(rs, ci, a, shift, niter, threads=1)
    par = oracle.power_iterate(rs, ci, a, shift, niter, threads=4)
    rel = np.abs(par["zeta"] - serial["zeta"]) / np.abs(serial["zeta"])
    assert rel.max() <= 1e-10
    assert np.abs(par["rnorm"] - serial["rnorm"]).max() <= 1e-10


def test_oracle_conj_grad_matches_fixture(oracle):
    path = os.path.join(os.path.dirname(__file__), "golden", "conj_grad_S.npz")
    g = np.load(path)
    n, nonzer, _, shift = PARAMS["S"]
    rs, ci, a = oracle.makea(n, nonzer, 0.1, shift)
    z, p, q, r, rn = oracle.conj_grad(rs, ci, a, np.ones(n))
    assert np.array_equal(z[:n], g["z"])
    assert np.array_equal(r[:n], g["r"])
    assert np.array_equal(p[:n], g["p"])
    assert np.array_equal(q[:n], g["q"])
    assert rn == g["rnorm"][0]


@pytest.mark.skipif(not os.path.exists(ref_lib_path("S")), reason="oracle/_ref not built")
def test_reference_library_agrees_with_oracle(oracle):
    from oracle_py import RefLib
    ref = RefLib(ref_lib_path("S"))
    n, nonzer, niter, shift = PARAMS["S"]
    rs, ci, a = ref.makea(271828183.0)
    rs2, ci2, a2 = oracle.makea(n, nonzer, 0.1, shift, 271828183.0)
    assert np.array_equal(rs, rs2) and np.array_equal(ci, ci2) and np.array_equal(a, a2)
    x = np.linspace(0.5, 1.5, n)
    zr = ref.conj_grad(x)
    zo = oracle.conj_grad(rs2, ci2, a2, x)
    assert np.array_equal(zr[0], zo[0][:n])
    assert zr[4] == zo[4]


def test_reference_library_takes_the_product_csr(cgb, golden):
    """ref_set_matrix loads a CSR into the reference's arrays in place of
    its makea (the bench hands it the product generator's class-C matrix
    rather than spending the reference's 13 s on generating it): with the
    product's bit-identical class-S CSR the reference's own CPU loop
    reproduces its golden trace bit for bit."""
    import os
    path = ref_lib_path("S")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built")
    from oracle_py import RefLib
    ref = RefLib(path)
    rs, ci, a = cgb.makea(1400, 7, 0.1, 10.0)
    assert ref.set_matrix(rs, ci, a) == len(a)
    out = ref.power(15)
    e = golden["S"]["seeds"]["314159265.0"]
    assert np.array_equal(out["zeta"], np.array(e["zeta"]))
    assert np.array_equal(out["rnorm"], np.array(e["rnorm"]))


def test_oracle_zeta_converges_with_outer_steps(golden):
    """Documents how fast the power iteration settles (time-to-zeta depends on it)."""
    z = np.array(golden["S"]["seeds"]["314159265.0"]["zeta"])
    rel = np.abs(z - z[-1]) / z[-1]
    assert rel[-1] == 0.0 and rel[0] > 1e-3
