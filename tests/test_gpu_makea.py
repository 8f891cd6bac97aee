"""GPU assembly of the generator (cgb_makea_device) against the host
generator and the reference's CSR hashes: bit-exact (integer and byte work),
at every NPB class S..C and at other seeds."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = {"S": (1400, 7, 10.0), "W": (7000, 8, 12.0), "A": (14000, 11, 20.0),
          "B": (75000, 13, 60.0), "C": (150000, 15, 110.0)}


@pytest.mark.parametrize("cls", ["S", "W", "A", "B", "C"])
def test_device_assembly_bit_identical(cgb, golden, oracle, cls):
    n, nonzer, shift = PARAMS[cls]
    t0 = time.perf_counter()
    host = cgb.makea(n, nonzer, 0.1, shift)
    t1 = time.perf_counter()
    dev = cgb.makea_device(n, nonzer, 0.1, shift)
    t2 = time.perf_counter()
    print(f"\n{cls}: host {1e3 * (t1 - t0):.0f} ms, device assembly {1e3 * (t2 - t1):.0f} ms")
    for h, d in zip(host, dev):
        assert h.dtype == d.dtype and np.array_equal(h, d)
    assert np.array_equal(host[2].view(np.uint64), dev[2].view(np.uint64))
    ref = golden[cls]["seeds"]["314159265.0"]
    assert len(dev[2]) == ref["nnz"]
    assert oracle.csr_hash(*dev) == ref["csr_hash"]


def test_device_assembly_other_seeds(cgb, golden, oracle):
    for cls in ("S", "A"):
        n, nonzer, shift = PARAMS[cls]
        for key, ref in golden[cls]["seeds"].items():
            seed = float(key)
            dev = cgb.makea_device(n, nonzer, 0.1, shift, seed)
            host = cgb.makea(n, nonzer, 0.1, shift, seed)
            assert all(np.array_equal(h, d) for h, d in zip(host, dev))
            assert len(dev[2]) == ref["nnz"]
            assert oracle.csr_hash(*dev) == ref["csr_hash"]


@pytest.mark.parametrize("n,nonzer,shift", [(2, 1, 1.0), (64, 5, 3.0), (1024, 9, 5.0),
                                            (33, 31, 4.0), (40, 31, 4.0), (4097, 20, 8.0)])
def test_device_draw_edge_sizes(cgb, n, nonzer, shift):
    """The parallel vector draw against the host's sequential one: n a power
    of two, n just above one (half the candidates rejected), nonzer close to
    n (many duplicates: the pair buffer overflows and is doubled)."""
    for seed in (314159265.0, 271828183.0):
        host = cgb.makea(n, nonzer, 0.1, shift, seed)
        dev = cgb.makea_device(n, nonzer, 0.1, shift, seed)
        assert all(np.array_equal(h, d) for h, d in zip(host, dev))
        assert np.array_equal(host[2].view(np.uint64), dev[2].view(np.uint64))


@pytest.mark.parametrize("cls", ["S", "B", "C"])
def test_session_on_generated_matrix(cgb, golden, cls):
    """A session built on the device generator's CSR (never on the host)
    runs the same power iteration, bit for bit, as one created from the host
    generator's arrays with the same plan; a later conj_grad on host arrays
    uploads them."""
    n, nonzer, shift = PARAMS[cls]
    niter = {"S": 15, "B": 75, "C": 75}[cls]
    t0 = time.perf_counter()
    with cgb.Session.generated(n, nonzer, shift, spmv_kernel=2 if n >= 24576 else 1) as g:
        t1 = time.perf_counter()
        out_g = g.power_iterate(niter, shift)
        host = cgb.makea(n, nonzer, 0.1, shift)
        z, *_ = g.conj_grad(np.ones(n), matrix=host)
    with cgb.Session(*host, spmv_kernel=2 if n >= 24576 else 1) as h:
        out_h = h.power_iterate(niter, shift)
        zh, *_ = h.conj_grad(np.ones(n))
    print(f"\n{cls}: generated session in {1e3 * (t1 - t0):.0f} ms")
    assert np.array_equal(out_g["zeta"], out_h["zeta"])
    assert np.array_equal(out_g["rnorm"], out_h["rnorm"])
    assert np.array_equal(z, zh)
    ref = golden[cls]["seeds"]["314159265.0"]
    assert abs(out_g["zeta"][-1] - ref["zeta"][-1]) <= 1e-10 * abs(ref["zeta"][-1])


def test_device_assembly_rejects_bad_arguments(cgb):
    with pytest.raises(cgb.CgbError):
        cgb.makea_device(1400, 7, 0.1, 10.0, 314159264.0)   # even seed
    with pytest.raises(cgb.CgbError):
        cgb.makea_device(1400, 40, 0.1, 10.0)                # nonzer > 31
