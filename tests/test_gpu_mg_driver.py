"""The NPB-style MG, EP, IS and FT drivers `npb-gpu_b200/bin/mg`, `bin/ep`,
`bin/is` and `bin/ft`, drop-ins for the reference's mg.<CLASS>, ep.<CLASS>,
is.<CLASS> and ft.<CLASS> binaries (GMAP/NPB-GPU CUDA/MG/mg.cu main
:356-623, CUDA/EP/ep.cu main :114-275, CUDA/IS/is.cu main :335-505,
CUDA/FT/ft.cu main :335-505).

Its report must carry the reference's verification block (mg.cu:526-552,
epsilon 1e-8 on the L2 norm) and its Mop/s, recomputed here from the
reported time with the reference's operation count 58 nit n^3
(mg.cu:554-559).  The CPU tests check the argument handling and that
without a GPU the driver fails loudly (no CPU fallback).
"""
import json
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MG = os.path.join(ROOT, "npb-gpu_b200", "bin", "mg")
VERIFY = {"S": (32, 4, 0.5307707005734e-04), "W": (128, 4, 0.6467329375339e-05),
          "B": (256, 20, 0.1800564401355e-05)}


def run_mg(*args, timeout=600):
    if not os.path.exists(MG):
        pytest.skip("npb-gpu_b200/bin/mg not built")
    return subprocess.run([MG, *args], capture_output=True, text=True, timeout=timeout)


def field(text, name):
    m = re.search(r"^\s*" + re.escape(name) + r"\s*=\s*(.+?)\s*$", text, re.M)
    assert m, f"no '{name}' line in the report"
    return m.group(1)


def test_mg_driver_rejects_bad_arguments():
    for args in ([], ["X"], ["SS"], ["S", "--nit", "0"], ["S", "--what"]):
        r = run_mg(*args, timeout=60)
        assert r.returncode == 2, (args, r.returncode)
        assert "usage: mg" in r.stderr


def test_mg_driver_fails_loudly_without_a_gpu():
    import npbcg
    try:
        npbcg.device_info(0)
        pytest.skip("a CUDA device is present")
    except npbcg.CgbError:
        pass
    r = run_mg("S", timeout=120)
    assert r.returncode == 1 and "mg: create failed" in r.stderr
    assert "VERIFICATION" not in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("cls", ["S", "W"])
def test_mg_driver_report_verifies(cls):
    n, nit, want = VERIFY[cls]
    r = run_mg(cls)
    assert r.returncode == 0, r.stderr
    assert " VERIFICATION SUCCESSFUL" in r.stdout
    norm = float(re.search(r"L2 Norm is\s+(\S+)", r.stdout).group(1))
    assert abs(norm - want) / want <= 1e-8
    assert field(r.stdout, "class_npb") == cls
    assert int(field(r.stdout, "Iterations")) == nit
    assert field(r.stdout, "Verification") == "SUCCESSFUL"
    t = float(field(r.stdout, "Time in seconds"))
    mops = float(field(r.stdout, "Mop/s total"))
    expect = 58.0 * nit * n ** 3 * 1e-6 / t
    assert abs(mops - expect) <= expect * (1e-6 / t + 1e-6) + 0.01


@pytest.mark.gpu
def test_mg_driver_json_class_b():
    n, nit, want = VERIFY["B"]
    r = run_mg("B", "--json")
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["class"] == "B" and line["n"] == n and line["nit"] == nit
    assert line["verified"] is True and line["rel_err"] <= 1e-8
    assert abs(line["mops"] - 58.0 * nit * n ** 3 * 1e-6 / line["seconds"]) <= 1e-5 * line["mops"]


@pytest.mark.gpu
def test_mg_driver_other_iteration_count_is_unverified():
    r = run_mg("S", "--nit", "2")
    assert r.returncode == 0, r.stderr
    assert "NO VERIFICATION PERFORMED" in r.stdout
    assert field(r.stdout, "Verification") == "NOT PERFORMED"


# ------------------------------------------------------------------ EP driver
EP = os.path.join(ROOT, "npb-gpu_b200", "bin", "ep")


def run_ep(*args, timeout=600):
    if not os.path.exists(EP):
        pytest.skip("npb-gpu_b200/bin/ep not built")
    return subprocess.run([EP, *args], capture_output=True, text=True, timeout=timeout)


def test_ep_driver_rejects_bad_arguments():
    for args in ([], ["X"], ["SS"], ["S", "--what"]):
        r = run_ep(*args, timeout=60)
        assert r.returncode == 2 and "usage: ep" in r.stderr


@pytest.mark.gpu
def test_ep_driver_report_verifies():
    r = run_ep("W")
    assert r.returncode == 0, r.stderr
    assert field(r.stdout, "Verification") == "SUCCESSFUL"
    sums = re.search(r"Sums =\s+(\S+)\s+(\S+)", r.stdout)
    sx, sy = float(sums.group(1)), float(sums.group(2))
    assert abs(sx + 2.863319731645753e+3) / 2.863319731645753e+3 <= 1e-8
    assert abs(sy + 6.320053679109499e+3) / 6.320053679109499e+3 <= 1e-8
    t = float(field(r.stdout, "Time in seconds"))
    mops = float(field(r.stdout, "Mop/s total"))
    expect = 2.0 ** 26 / t / 1e6
    assert abs(mops - expect) <= expect * (1e-6 / t + 1e-6) + 0.01
    line = json.loads(run_ep("S", "--json").stdout.strip().splitlines()[-1])
    assert line["verified"] is True and line["m"] == 24


# ------------------------------------------------------------------ IS driver
IS = os.path.join(ROOT, "npb-gpu_b200", "bin", "is")


def run_is(*args, timeout=600):
    if not os.path.exists(IS):
        pytest.skip("npb-gpu_b200/bin/is not built")
    return subprocess.run([IS, *args], capture_output=True, text=True, timeout=timeout)


def test_is_driver_rejects_bad_arguments():
    for args in ([], ["E"], ["SS"], ["S", "--what"]):
        r = run_is(*args, timeout=60)
        assert r.returncode == 2 and "usage: is" in r.stderr


@pytest.mark.gpu
def test_is_driver_report_verifies():
    r = run_is("W")
    assert r.returncode == 0, r.stderr
    assert field(r.stdout, "Verification") == "SUCCESSFUL"
    assert field(r.stdout, "Checks passed") == "51 of 51"
    t = float(field(r.stdout, "Time in seconds"))
    mops = float(field(r.stdout, "Mop/s total"))
    expect = 10 * 2.0 ** 20 / t / 1e6  # is.cu:484
    assert abs(mops - expect) <= expect * (1e-6 / t + 1e-6) + 0.01
    line = json.loads(run_is("S", "--json").stdout.strip().splitlines()[-1])
    assert line["verified"] is True and line["passed"] == 51 and line["keys"] == 2 ** 16


# ------------------------------------------------------------------ FT driver
FT = os.path.join(ROOT, "npb-gpu_b200", "bin", "ft")


def run_ft(*args, timeout=600):
    if not os.path.exists(FT):
        pytest.skip("npb-gpu_b200/bin/ft not built")
    return subprocess.run([FT, *args], capture_output=True, text=True, timeout=timeout)


def test_ft_driver_rejects_bad_arguments():
    for args in ([], ["E"], ["SS"], ["S", "--what"]):
        r = run_ft(*args, timeout=60)
        assert r.returncode == 2 and "usage: ft" in r.stderr


@pytest.mark.gpu
def test_ft_driver_report_verifies():
    import math
    r = run_ft("W")
    assert r.returncode == 0, r.stderr
    assert field(r.stdout, "Verification") == "SUCCESSFUL"
    lines = re.findall(r"^T =\s+(\d+)\s+Checksum =\s+(\S+)\s+(\S+)$", r.stdout, re.M)
    assert [int(t) for t, _, _ in lines] == list(range(1, 7))
    assert abs(float(lines[0][1]) - 5.673612178944E+02) <= 1e-9 * 5.673612178944E+02
    t = float(field(r.stdout, "Time in seconds"))
    mops = float(field(r.stdout, "Mop/s total"))
    nt = 128.0 * 128 * 32
    expect = 1e-6 * nt * (14.8157 + 7.19641 * math.log(nt) + (5.23518 + 7.21113 * math.log(nt)) * 6) / t
    assert abs(mops - expect) <= expect * (1e-6 / t + 1e-6) + 0.01
    line = json.loads(run_ft("S", "--json").stdout.strip().splitlines()[-1])
    assert line["verified"] is True and line["niter"] == 6 and line["max_rel_err"] <= 1e-12


@pytest.mark.parametrize("name,runner", [("ep", run_ep), ("is", run_is), ("ft", run_ft)])
def test_npb_drivers_fail_loudly_without_a_gpu(name, runner):
    """No CPU fallback: without a CUDA device each driver exits 1 with the
    library's error and prints no verification."""
    import npbcg
    try:
        npbcg.device_info(0)
        pytest.skip("a CUDA device is present")
    except npbcg.CgbError:
        pass
    r = runner("S", timeout=120)
    assert r.returncode == 1 and f"{name}: run failed" in r.stderr
    assert "SUCCESSFUL" not in r.stdout
