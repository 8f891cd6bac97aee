"""GPU parity of NPB EP (npb-gpu_b200/csrc/ep.cu) through the C ABI.

Against the oracle (oracle/ep_oracle.c, pinned to the reference's sums):
the sums agree to relative 1e-12 (they add billions of terms in another
order; log is CUDA's, not the C library's) and the ten counts exactly.
Every class S-D must verify against the reference's sums at its epsilon,
1e-8 (ep.cu:189-212), and repeated runs agree bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m", [24, 25])
def test_ep_matches_oracle(cgb, oracle, m):
    got = cgb.ep_run(m)
    want = oracle.ep_run(m)
    assert abs(got["sx"] - want["sx"]) <= 1e-12 * abs(want["sx"])
    assert abs(got["sy"] - want["sy"]) <= 1e-12 * abs(want["sy"])
    assert np.array_equal(got["q"], want["q"])


@pytest.mark.parametrize("cls", ["S", "W", "A", "B", "C", "D"])
def test_ep_class_verifies(cgb, cls):
    c = cgb.EP_CLASSES[cls]
    out = cgb.ep_run(c["m"])
    assert abs(out["sx"] - c["sx"]) / abs(c["sx"]) <= cgb.EP_VERIFY_EPSILON
    assert abs(out["sy"] - c["sy"]) / abs(c["sy"]) <= cgb.EP_VERIFY_EPSILON
    assert abs(out["q"].sum() / 2.0 ** c["m"] - np.pi / 4) < 1e-3
    assert out["device_ms"] > 0


def test_ep_repeatable_and_invalid(cgb):
    a, b = cgb.ep_run(24), cgb.ep_run(24)
    assert a["sx"] == b["sx"] and a["sy"] == b["sy"] and np.array_equal(a["q"], b["q"])
    for m in (19, 41):
        with pytest.raises(cgb.CgbError) as e:
            cgb.ep_run(m)
        assert e.value.status == cgb.ERR_INVALID


def test_reference_gpu_ep_agrees(cgb):
    """The reference's own EP kernel (compiled from its sources into
    oracle/_ref) on the same GPU: its sums verify, and ours agree with them."""
    import os
    from conftest import REF_DIR
    from oracle_py import RefEpLib
    path = os.path.join(REF_DIR, "libref_ep_S.so")
    if not os.path.exists(path):
        pytest.skip("the reference's EP library was not built (make -C oracle)")
    ref = RefEpLib(path).gpu()
    c = cgb.EP_CLASSES["S"]
    assert abs(ref["sx"] - c["sx"]) / abs(c["sx"]) <= cgb.EP_VERIFY_EPSILON
    ours = cgb.ep_run(c["m"])
    assert abs(ours["sx"] - ref["sx"]) <= 1e-10 * abs(ref["sx"])
    assert abs(ours["sy"] - ref["sy"]) <= 1e-10 * abs(ref["sy"])
