"""Regenerate tests/golden/reference_cg.json from the reference's own code.

Run in a container that holds the reference tree, after `make -C oracle`
built oracle/_ref/libref_<class>.so from it:

    python tests/golden/make_golden.py            # all classes (B, C take minutes)
    python tests/golden/make_golden.py S W A      # a subset

For every NPB class it records, from the reference makea and its CPU
conj_grad outer loop (CUDA/CG/cg.cu:403-520): nnz, a FNV-1a-64 hash of the
CSR (definition in oracle/cg_oracle.c: orc_csr_hash), the per-step zeta and
rnorm traces, and the loop's wall time on this host.  It also records the
CSR hash and zeta trace at a few other odd LCG seeds (classes S and A), and
one conj_grad call from x = 1 at class S (z and r vectors, npz).
"""
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFDIR = os.path.join(ROOT, "oracle", "_ref")

I32 = np.ctypeslib.ndpointer(np.int32, flags="C")
F64 = np.ctypeslib.ndpointer(np.float64, flags="C")
SEED = 314159265.0
EXTRA_SEEDS = {"S": [271828183.0, 123456789.0], "A": [161803399.0]}


def csr_hash(n, rowstr, colidx, a):
    """FNV-1a-64 exactly as orc_csr_hash (ints widened to u64)."""
    mask = (1 << 64) - 1
    h = 0xCBF29CE484222325
    prime = 0x100000001B3
    for v in rowstr[: n + 1].astype(np.int64):
        h = ((h ^ (int(v) & mask)) * prime) & mask
    nnz = int(rowstr[n])
    bits = a[:nnz].view(np.uint64)
    cols = colidx[:nnz].astype(np.int64)
    for c, b in zip(cols.tolist(), bits.tolist()):
        h = ((h ^ (c & mask)) * prime) & mask
        h = ((h ^ b) * prime) & mask
    return h


def load(cls):
    lib = ctypes.CDLL(os.path.join(REFDIR, f"libref_{cls}.so"))
    lib.ref_info.argtypes = [ctypes.POINTER(ctypes.c_int)] * 3 + [
        ctypes.POINTER(ctypes.c_double)] * 2 + [ctypes.POINTER(ctypes.c_longlong)]
    lib.ref_makea.argtypes = [ctypes.c_double, I32, I32, F64]
    lib.ref_makea.restype = ctypes.c_int
    lib.ref_power.argtypes = [ctypes.c_int, F64, F64]
    lib.ref_power.restype = ctypes.c_double
    lib.ref_conj_grad.argtypes = [F64, F64, F64, F64, F64, F64]
    lib.ref_conj_grad.restype = ctypes.c_int
    na, nz, ni = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    sh, rc, bound = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
    lib.ref_info(ctypes.byref(na), ctypes.byref(nz), ctypes.byref(ni), ctypes.byref(sh),
                 ctypes.byref(rc), ctypes.byref(bound))
    return lib, dict(n=na.value, nonzer=nz.value, niter=ni.value, shift=sh.value,
                     rcond=rc.value, nz_bound=bound.value)


def run_class(cls, out):
    lib, p = load(cls)
    n = p["n"]
    rowstr = np.zeros(n + 1, np.int32)
    colidx = np.zeros(p["nz_bound"], np.int32)
    a = np.zeros(p["nz_bound"], np.float64)
    entry = dict(p)
    seeds = {}
    for seed in [SEED] + EXTRA_SEEDS.get(cls, []):
        t0 = time.time()
        nnz = lib.ref_makea(seed, rowstr, colidx, a)
        tgen = time.time() - t0
        h = csr_hash(n, rowstr, colidx, a)
        zt = np.zeros(p["niter"])
        rt = np.zeros(p["niter"])
        secs = lib.ref_power(p["niter"], zt, rt)
        seeds[repr(seed)] = dict(seed=seed, nnz=int(nnz), csr_hash=f"{h:016x}",
                                 zeta=zt.tolist(), rnorm=rt.tolist(),
                                 makea_seconds=tgen, solve_seconds=secs)
        print(cls, seed, nnz, f"{h:016x}", f"{zt[-1]:.13f}", f"gen {tgen:.2f}s solve {secs:.2f}s",
              flush=True)
        if cls == "S" and seed == SEED:
            lib.ref_makea(seed, rowstr, colidx, a)
            z = np.zeros(n); r = np.zeros(n); pp = np.zeros(n); q = np.zeros(n)
            rn = np.zeros(1)
            lib.ref_conj_grad(np.ones(n), z, r, pp, q, rn)
            np.savez_compressed(os.path.join(HERE, "conj_grad_S.npz"), z=z, r=r, p=pp, q=q,
                                rnorm=rn)
    entry["seeds"] = seeds
    out[cls] = entry


def main(argv):
    classes = argv or ["S", "W", "A", "B", "C"]
    path = os.path.join(HERE, "reference_cg.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for cls in classes:
        run_class(cls, out)
        json.dump(out, open(path, "w"), indent=1)
    # the verification zetas hard-coded in the reference (CUDA/CG/cg.cu:373-396)
    out["verify"] = {"S": 8.5971775078648, "W": 10.362595087124, "A": 17.130235054029,
                     "B": 22.712745482631, "C": 28.973605592845, "epsilon": 1.0e-10}
    json.dump(out, open(path, "w"), indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
