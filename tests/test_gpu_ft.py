"""GPU parity of NPB FT (npb-gpu_b200/csrc/ft.cu) through the C ABI.

Against the oracle (oracle/ft_oracle.c, which reproduces the reference's
checksums, ft.cu:1655-1810): every iteration's checksum within relative
1e-13, the last inverse transform u1 and the evolved field u0 within 1e-12
of their largest element, the twiddle factors within an ulp (CUDA's exp
against the C library's, the same argument).  Shapes cover every line
length 32 .. 2048 and the radix-4 and radix-2 last stages.  Every class
S-D must verify at the reference's 1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def check_against_oracle(cgb, oracle, nx, ny, nz, niter):
    with cgb.Ft(nx, ny, nz) as f:
        out = f.run(niter)
        u1, u0, tw = f.read("u1"), f.read("u0"), f.read("twiddle")
    sums, want_u1 = oracle.ft_run(nx, ny, nz, niter, field=True)
    for a, b in zip(out["sums"], sums):
        assert abs(complex(*a) - complex(*b)) <= 1e-13 * abs(complex(*b))
    assert np.abs(u1 - want_u1).max() <= 1e-12 * np.abs(want_u1).max()
    want_tw = oracle.ft_indexmap(nx, ny, nz)
    assert np.allclose(tw, want_tw, rtol=3e-16, atol=0)
    want_u0 = oracle.ft_fft3d(1, oracle.ft_initial(nx, ny, nz))
    for _ in range(niter):
        want_u0 = want_u0 * want_tw
    assert np.abs(u0 - want_u0).max() <= 1e-12 * np.abs(want_u0).max()


@pytest.mark.parametrize("cls", ["S", "W"])
def test_ft_matches_oracle(cgb, oracle, cls):
    check_against_oracle(cgb, oracle, *cgb.FT_CLASSES[cls])


@pytest.mark.parametrize("dims", [(32, 64, 128, 2), (128, 32, 64, 2), (2048, 32, 32, 1), (32, 1024, 32, 1),
                                  (32, 32, 1024, 1), (32, 2048, 32, 1)])
def test_ft_shapes_match_oracle(cgb, oracle, dims):
    check_against_oracle(cgb, oracle, *dims)


@pytest.mark.parametrize("cls", ["S", "W", "A", "B", "C", "D"])
def test_ft_class_verifies(cgb, cls):
    nx, ny, nz, niter = cgb.FT_CLASSES[cls]
    with cgb.Ft(nx, ny, nz) as f:
        out = f.run(niter)
    assert cgb.ft_verify(cls, out["sums"]) <= cgb.FT_VERIFY_EPSILON
    assert out["device_ms"] > 0


def test_ft_repeatable_and_invalid(cgb):
    with cgb.Ft(64, 64, 64) as f:
        a, b = f.run(6), f.run(6)
        assert a["sums"] == b["sums"]
        for niter in (0, 65):
            with pytest.raises(cgb.CgbError) as e:
                f.run(niter)
            assert e.value.status == cgb.ERR_INVALID
    for dims in [(48, 64, 64), (16, 64, 64), (64, 64, 4096)]:
        with pytest.raises(cgb.CgbError) as e:
            cgb.Ft(*dims)
        assert e.value.status == cgb.ERR_INVALID


def test_reference_gpu_ft_agrees(cgb):
    """The reference's own FT kernels (compiled from its sources into
    oracle/_ref) on the same GPU verify, and ours agree with them."""
    import os
    from conftest import REF_DIR
    from oracle_py import RefFtLib
    path = os.path.join(REF_DIR, "libref_ft_S.so")
    if not os.path.exists(path):
        pytest.skip("the reference's FT library was not built (make -C oracle)")
    ref = RefFtLib(path).gpu()
    assert cgb.ft_verify("S", ref["sums"]) <= cgb.FT_VERIFY_EPSILON
    with cgb.Ft(64, 64, 64) as f:
        ours = f.run(6)["sums"]
    for a, b in zip(ours, ref["sums"]):
        assert abs(complex(*a) - complex(*b)) <= 1e-12 * abs(complex(*b))


def test_ft_runs_of_different_lengths_agree(cgb):
    """A run is main's whole timed region, so its checksums do not depend on
    the runs before it: 6 iterations after a 2-iteration run (the region
    captured again for the new length) equal a fresh instance's 6, and the
    first 2 of them equal the 2-iteration run's."""
    with cgb.Ft(64, 64, 64) as f:
        two = f.run(2)["sums"]
        six = f.run(6)["sums"]
    with cgb.Ft(64, 64, 64) as g:
        fresh = g.run(6)["sums"]
    assert six == fresh
    assert six[:2] == two
