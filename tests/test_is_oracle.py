"""The IS oracle (oracle/is_oracle.c) pinned against the reference.

The reference's IS (GMAP/NPB-GPU CUDA/IS/is.cu) carries, for each class, the
indices of five keys and their ranks at every iteration (is.cu:157-190,
checked by rank_gpu_kernel_7 with per-class offsets), and a full check that
the keys sort.  A run verifies when all 5 x 10 partial checks and the full
check pass: 51.  The oracle must verify at S, W, A and B (B: 2^25 keys, a
few seconds).
"""
import pytest

# (TOTAL_KEYS_LOG_2, MAX_KEY_LOG_2) is.cu:86-140; test arrays is.cu:157-190
IS_CLASSES = {
    "S": (16, 11, [48427, 17148, 23627, 62548, 4431], [0, 18, 346, 64917, 65463]),
    "W": (20, 16, [357773, 934767, 875723, 898999, 404505], [1249, 11698, 1039987, 1043896, 1048018]),
    "A": (23, 19, [2112377, 662041, 5336171, 3642833, 4250760], [104, 17523, 123928, 8288932, 8388264]),
    "B": (25, 21, [41869, 812306, 5102857, 18232239, 26860214], [33422937, 10244, 59149, 33135281, 99]),
}


@pytest.mark.parametrize("cls", ["S", "W", "A", "B"])
def test_is_oracle_verifies(oracle, cls):
    tl, ml, ti, tr = IS_CLASSES[cls]
    assert oracle.is_run(cls, tl, ml, ti, tr) == 51


def test_is_oracle_fails_a_wrong_table(oracle):
    """A rank off by one in the table fails that test key at every iteration."""
    tl, ml, ti, tr = IS_CLASSES["S"]
    wrong = list(tr)
    wrong[3] += 1
    assert oracle.is_run("S", tl, ml, ti, wrong) == 41
