"""The EP oracle (oracle/ep_oracle.c) pinned against the reference.

The reference's EP (GMAP/NPB-GPU CUDA/EP/ep.cu) hard-codes the two sums of
the Gaussian deviates for each class (ep.cu:189-212) and accepts a run
within relative 1e-8 of them.  They are printed to 16 significant digits;
the oracle, a plain-C restatement of the reference's serial loop with its
own LCG arithmetic, must match them to 1e-13.  Classes S and W run on the
CPU in a few seconds.
"""
import numpy as np
import pytest

EP_VERIFY = {24: (-3.247834652034740e+3, -6.958407078382297e+3),
             25: (-2.863319731645753e+3, -6.320053679109499e+3)}


@pytest.mark.parametrize("m", [24, 25])
def test_ep_oracle_matches_reference_sums(oracle, m):
    vx, vy = EP_VERIFY[m]
    out = oracle.ep_run(m)
    assert abs(out["sx"] - vx) / abs(vx) <= 1e-13
    assert abs(out["sy"] - vy) / abs(vy) <= 1e-13
    q = out["q"]
    # every accepted pair is counted once; about pi/4 of the 2^m pairs
    assert np.all(q == np.round(q)) and abs(q.sum() / 2.0 ** m - np.pi / 4) < 1e-3
    assert q[9] == 0.0
