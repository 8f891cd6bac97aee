"""The NPB-style driver `npb-gpu_b200/bin/cg`, a drop-in for the reference's
cg.<CLASS> binary (GMAP/NPB-GPU CUDA/CG/cg.cu main, :337-645).

Its report is diffed against the reference's own trace (tests/golden,
generated from oracle/_ref): the per-iteration "||r||  zeta" lines in the
reference format (cg.cu:515-516, zeta relative 1e-10, rnorm absolute 1e-10),
the verification block (cg.cu:534-552, epsilon 1e-10) and the Mop/s figure,
recomputed here from the reported time with the reference's operation
count (cg.cu:553-561).  The CPU tests check the argument handling and that
without a GPU the driver fails loudly (no CPU fallback).
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CG = os.path.join(ROOT, "npb-gpu_b200", "bin", "cg")

PARAMS = {"S": (1400, 7, 15, 10.0), "C": (150000, 15, 75, 110.0)}
ITER_LINE = re.compile(r"^\s+(\d+)\s+(\S+e[+-]\d+)\s*(\S+e[+-]\d+)\s*$")


def run_cg(*args, timeout=600):
    if not os.path.exists(CG):
        pytest.skip("npb-gpu_b200/bin/cg not built")
    return subprocess.run([CG, *args], capture_output=True, text=True, timeout=timeout)


def reference_mops(niter, n, nonzer, seconds):
    """The reference's Mop/s (cg.cu:553-561)."""
    nz1 = float(nonzer * (nonzer + 1))
    return 2.0 * niter * n * (3.0 + nz1 + 25.0 * (5.0 + nz1) + 3.0) / seconds / 1e6


def parse_trace(text):
    its, rn, ze = [], [], []
    for line in text.splitlines():
        m = ITER_LINE.match(line)
        if m:
            its.append(int(m.group(1)))
            rn.append(float(m.group(2)))
            ze.append(float(m.group(3)))
    return its, np.array(rn), np.array(ze)


def field(text, name):
    m = re.search(r"^\s*" + re.escape(name) + r"\s*=\s*(.+?)\s*$", text, re.M)
    assert m, f"no '{name}' line in the report"
    return m.group(1)


# ------------------------------------------------------------------ CPU
def test_driver_rejects_bad_arguments():
    for args in ([], ["X"], ["S", "--mode", "nope"], ["U", "--n", "1"], ["S", "--spmv", "x"]):
        r = run_cg(*args, timeout=60)
        assert r.returncode == 2, (args, r.returncode)
        assert "usage: cg" in r.stderr


def test_driver_row_blocks_take_the_reference_algorithm_only():
    r = run_cg("S", "--ranks", "2", "--mode", "mixed", timeout=60)
    assert r.returncode == 2 and "--ranks" in r.stderr
    r = run_cg("S", "--ranks", "-1", timeout=60)
    assert r.returncode == 2


def test_driver_fails_loudly_without_a_gpu():
    import npbcg
    try:
        npbcg.device_info(0)
        pytest.skip("a CUDA device is present")
    except npbcg.CgbError:
        pass
    r = run_cg("S", timeout=120)
    assert r.returncode == 1
    assert "cg: create failed" in r.stderr
    assert "VERIFICATION" not in r.stdout


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_driver_class_s_report_matches_reference(golden):
    n, nonzer, niter, shift = PARAMS["S"]
    r = run_cg("S")
    assert r.returncode == 0, r.stderr
    its, rn, ze = parse_trace(r.stdout)
    e = golden["S"]["seeds"]["314159265.0"]
    assert its == list(range(1, niter + 1))
    ref_z, ref_r = np.array(e["zeta"]), np.array(e["rnorm"])
    # the report prints 13-14 significant digits: compare at 1e-10
    assert np.max(np.abs(ze - ref_z) / ref_z) <= 1e-10
    assert np.max(np.abs(rn - ref_r)) <= 1e-10
    assert " VERIFICATION SUCCESSFUL" in r.stdout
    zeta = float(re.search(r"Zeta is\s+(\S+)", r.stdout).group(1))
    err = float(re.search(r"Error is\s+(\S+)", r.stdout).group(1))
    verify = golden["verify"]["S"]
    assert abs(zeta - verify) / verify <= 1e-10
    assert err <= 1e-10
    assert field(r.stdout, "class_npb") == "S"
    assert int(field(r.stdout, "Size")) == n
    assert int(field(r.stdout, "Iterations")) == niter
    assert field(r.stdout, "Verification") == "SUCCESSFUL"
    t = float(field(r.stdout, "Time in seconds"))
    mops = float(field(r.stdout, "Mop/s total"))
    assert t > 0
    # the time is printed to 1e-6 s: the recomputed figure agrees to that
    want = reference_mops(niter, n, nonzer, t)
    assert abs(mops - want) <= want * (1e-6 / t + 1e-6) + 0.01


@pytest.mark.gpu
def test_driver_other_seed_is_unverified_and_matches_reference(golden):
    n, nonzer, niter, shift = PARAMS["S"]
    e = golden["S"]["seeds"]["271828183.0"]
    r = run_cg("S", "--seed", "271828183")
    assert r.returncode == 0, r.stderr
    _, rn, ze = parse_trace(r.stdout)
    assert np.max(np.abs(ze - np.array(e["zeta"])) / np.array(e["zeta"])) <= 1e-10
    assert np.max(np.abs(rn - np.array(e["rnorm"]))) <= 1e-10
    assert "NO VERIFICATION PERFORMED" in r.stdout
    assert field(r.stdout, "Verification") == "NOT PERFORMED"


@pytest.mark.gpu
@pytest.mark.slow
def test_driver_class_c_json(golden):
    n, nonzer, niter, shift = PARAMS["C"]
    r = run_cg("C", "--json", "--gpu-makea")
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["class"] == "C" and line["n"] == n and line["niter"] == niter
    assert line["verified"] is True and line["rel_err"] <= 1e-10
    assert line["nnz"] == golden["C"]["seeds"]["314159265.0"]["nnz"]
    ref_z = golden["C"]["seeds"]["314159265.0"]["zeta"][-1]
    assert abs(line["zeta"] - ref_z) / ref_z <= 1e-10
    assert line["inner_total"] == 25 * niter
    want = reference_mops(niter, n, nonzer, line["seconds"])
    assert abs(line["mops"] - want) <= 1e-5 * want


@pytest.mark.gpu
def test_driver_row_blocks_class_s_match_reference(golden):
    """`cg S --ranks 3`: the row-partitioned solver (three row blocks
    generated on the device) prints the reference's trace and verifies."""
    n, nonzer, niter, shift = PARAMS["S"]
    r = run_cg("S", "--ranks", "3")
    assert r.returncode == 0, r.stderr
    its, rn, ze = parse_trace(r.stdout)
    e = golden["S"]["seeds"]["314159265.0"]
    assert its == list(range(1, niter + 1))
    assert np.max(np.abs(ze - np.array(e["zeta"])) / np.array(e["zeta"])) <= 1e-10
    assert np.max(np.abs(rn - np.array(e["rnorm"]))) <= 1e-10
    assert field(r.stdout, "Verification") == "SUCCESSFUL"
    assert int(field(r.stdout, "Nonzeros")) == e["nnz"]
    assert int(field(r.stdout, "Row blocks")) == 3
