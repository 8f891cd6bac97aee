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


def test_device_assembly_rejects_bad_arguments(cgb):
    with pytest.raises(cgb.CgbError):
        cgb.makea_device(1400, 7, 0.1, 10.0, 314159264.0)   # even seed
    with pytest.raises(cgb.CgbError):
        cgb.makea_device(1400, 40, 0.1, 10.0)                # nonzer > 31
