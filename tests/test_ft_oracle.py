"""The FT oracle (oracle/ft_oracle.c) pinned against the reference.

The reference's FT (GMAP/NPB-GPU CUDA/FT/ft.cu) hard-codes every
iteration's checksum for each class (ft.cu:1655-1810) and accepts a run
within relative 1e-12 of them.  The oracle, a plain-C restatement of the
reference's initial conditions, index map, radix-2 Stockham line transform
and checksum, must match them at S and W (a fraction of a second each).
Its pieces are also held to independent restatements here: the initial
conditions to an integer LCG, the 3-D transform to numpy's FFT (the
reference's is = 1 is numpy's unnormalised inverse), the index map to its
formula.
"""
import numpy as np
import pytest

from npbcg import FT_CHECKSUMS


@pytest.mark.parametrize("cls,dims", [("S", (64, 64, 64, 6)), ("W", (128, 128, 32, 6))])
def test_ft_oracle_matches_reference_checksums(oracle, cls, dims):
    sums = oracle.ft_run(*dims)
    ref = FT_CHECKSUMS[cls]
    err = max(abs(complex(*s) - complex(*r)) / abs(complex(*r)) for s, r in zip(sums, ref))
    assert err <= 1e-12, err


def test_ft_initial_conditions_are_the_lcg_stream(oracle):
    nx, ny, nz = 32, 16, 8
    u = oracle.ft_initial(nx, ny, nz).ravel()
    x, a, m = 314159265, 1220703125, (1 << 46) - 1
    want = []
    for _ in range(2 * u.size):
        x = (x * a) & m
        want.append(x * 2.0 ** -46)
    want = np.array(want)
    assert np.array_equal(u.real, want[0::2]) and np.array_equal(u.imag, want[1::2])


def test_ft_transform_is_numpys(oracle):
    rng = np.random.default_rng(5)
    a = rng.standard_normal((8, 16, 32)) + 1j * rng.standard_normal((8, 16, 32))
    fwd = oracle.ft_fft3d(1, a)
    inv = oracle.ft_fft3d(-1, a)
    scale = np.abs(a).sum()
    assert np.abs(fwd - np.fft.ifftn(a) * a.size).max() <= 1e-14 * scale
    assert np.abs(inv - np.fft.fftn(a)).max() <= 1e-14 * scale


def test_ft_indexmap_formula(oracle):
    nx, ny, nz = 32, 16, 8
    tw = oracle.ft_indexmap(nx, ny, nz)
    f = lambda n: ((np.arange(n) + n // 2) % n) - n // 2
    k2 = f(nz)[:, None, None] ** 2 + f(ny)[None, :, None] ** 2 + f(nx)[None, None, :] ** 2
    ap = -4.0 * 1.0e-6 * np.pi * np.pi
    assert np.allclose(tw, np.exp(ap * k2), rtol=1e-15, atol=0)
