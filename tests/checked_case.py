"""One run of the solver paths against a given libcgb build, for
test_gpu_checked.py: the normal library and the bounds-checked one
(lib/libcgb_checked.so, -DCGB_CHECKED) each run this in a fresh process,
and the test compares their outputs bit for bit and reads the checked
build's check word after every path.

    python tests/checked_case.py LIBRARY OUT.npz
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "npb-gpu_b200"))
import npbcg  # noqa: E402


def check_word():
    w = ctypes.c_int()
    npbcg._check(npbcg.lib().cgb_check_status(ctypes.byref(w)))
    return w.value


def main():
    npbcg.LIB_PATH = sys.argv[1]
    out, words = {}, {}
    # row plan (class S) and a CSR whose entry count is odd (n = 1401); the
    # plan is fixed (the autotuner's pick between lane counts and grid sizes
    # may differ between the two libraries' runs, and with it the order of
    # the sums), so the two libraries' results compare bit for bit
    for name, n, nonzer, shift in (("S", 1400, 7, 10.0), ("odd", 1401, 7, 10.0)):
        rs, ci, a = npbcg.makea(n, nonzer, npbcg.RCOND, shift)
        with npbcg.Session(rs, ci, a, spmv_kernel=1, lanes_per_row=8) as s:
            r = s.power_iterate(15, shift)
            z, *_ = s.conj_grad(np.ones(n))
        out[f"{name}_zeta"], out[f"{name}_z"] = r["zeta"], z
        words[name] = check_word()
    # caller-owned unpadded buffers (the odd-nnz matrix: the last pair load)
    import torch
    dev = torch.device("cuda", 0)
    rs, ci, a = npbcg.makea(1401, 7, npbcg.RCOND, 10.0)
    d = [torch.from_numpy(v).to(dev) for v in (rs, ci, a, np.ones(1402))]
    d_z = torch.empty(1402, dtype=torch.float64, device=dev)
    d_rn = torch.empty(1, dtype=torch.float64, device=dev)
    d_st = torch.zeros(1, dtype=torch.int32, device=dev)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    st = npbcg.lib().cgb_conj_grad_noalloc(1401, len(a), *[p(t) for t in d], p(d_z), p(d_rn),
                                            p(d_st), None)
    torch.cuda.synchronize(dev)
    assert st == 0 and int(d_st.item()) == 0
    out["noalloc_z"] = d_z.cpu().numpy()
    words["noalloc"] = check_word()
    # sliced plans (class B): both instances, an L2 keep, FP64 and mixed
    rs, ci, a = npbcg.makea(75000, 13, npbcg.RCOND, 60.0)
    for kind in (2, 3):
        with npbcg.Session(rs, ci, a, spmv_kernel=kind) as s:
            s.set_l2_keep(64e6)
            out[f"B{kind}_fp64"] = s.power_iterate(4, 60.0)["zeta"]
            out[f"B{kind}_mixed"] = s.power_iterate(4, 60.0, mode=npbcg.MODE_MIXED, tol=1e-12,
                                                   cgitmax=100)["zeta"]
            if kind == 2:
                model = npbcg.Gnn()
                model.load()
                with model.graph(rs, ci, a) as g:
                    model.attach(g, s)
                out["B_learned"] = s.power_iterate(4, 60.0, mode=npbcg.MODE_MIXED_LEARNED,
                                                   tol=1e-12, cgitmax=100)["zeta"]
        words[f"B{kind}"] = check_word()
    np.savez(sys.argv[2], words=np.array([words[k] for k in sorted(words)]),
             word_names=np.array(sorted(words)), **out)


if __name__ == "__main__":
    main()
