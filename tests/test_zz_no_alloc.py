"""The allocation-free conj_grad entry point (cgb_conj_grad_noalloc).

It serves callers that may not allocate GPU memory on this path (their
device memory comes from their own pool, or the loop must never allocate):
they pass their own device buffers for inputs and outputs, and the solver's
work space lives in a fixed array inside libcgb.  Checked through the C ABI,
twice in a row (the second call runs on the array the first one left
behind), against the session entry point cgb_conj_grad on the same matrix
and against the CPU oracle's restatement of the reference conj_grad
(cg.cu:653-801), with the tolerances of the other GPU tests: z relative
1e-12, rnorm absolute 1e-10 * ||x||.  The test allocates its buffers with
torch; the entry point itself allocates nothing.  This file is collected
last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_conj_grad_matches_session(cgb, oracle):
    import torch

    n, nonzer, shift = 14000, 11, 20.0
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift, 161803399.0)
    x = np.ones(n + 1)
    x[:n] = 1.0 + 0.25 * np.cos(np.arange(n) * 0.013)
    with cgb.Session(rs, ci, a) as s:
        z_ref, _, _, _, rn_ref = s.conj_grad(x)
    z_orc, _, _, _, rn_orc = oracle.conj_grad(rs, ci, a, x[:n])

    dev = torch.device("cuda", 0)
    d_rs = torch.from_numpy(rs).to(dev)
    d_ci = torch.from_numpy(ci).to(dev)
    d_a = torch.from_numpy(a).to(dev)
    d_x = torch.from_numpy(x).to(dev)
    d_z = torch.empty(n + 1, dtype=torch.float64, device=dev)
    d_rn = torch.empty(1, dtype=torch.float64, device=dev)
    d_st = torch.empty(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    xnorm = float(np.linalg.norm(x[:n]))
    for call in range(2):
        d_z.fill_(float("nan"))
        d_rn.fill_(float("nan"))
        d_st.fill_(-1)
        torch.cuda.synchronize(dev)
        st = cgb.lib().cgb_conj_grad_noalloc(n, len(a), _ptr(d_rs), _ptr(d_ci), _ptr(d_a),
                                              _ptr(d_x), _ptr(d_z), _ptr(d_rn), _ptr(d_st),
                                              ctypes.c_void_p(stream.cuda_stream))
        assert st == cgb.OK, cgb.lib().cgb_last_error()
        torch.cuda.synchronize(dev)
        assert int(d_st.item()) == 0, f"call {call}: device status {int(d_st.item())}"
        z = d_z.cpu().numpy()
        err = np.linalg.norm(z[:n] - z_ref[:n]) / np.linalg.norm(z_ref[:n])
        assert err <= 1e-12, f"call {call}: z differs from the session's by {err:.3e}"
        err = np.linalg.norm(z[:n] - z_orc[:n]) / np.linalg.norm(z_orc[:n])
        assert err <= 1e-12, f"call {call}: z differs from the oracle's by {err:.3e}"
        assert z[n] == 0.0
        rn = float(d_rn.item())
        assert abs(rn - rn_ref) <= 1e-10 * xnorm, f"call {call}: rnorm vs the session"
        assert abs(rn - rn_orc) <= 1e-10 * xnorm, f"call {call}: rnorm vs the oracle"


def test_noalloc_rejects_misaligned(cgb):
    """The SpMV reads entry pairs: values must be 16-byte, columns 8-byte
    aligned (as cudaMalloc returns them); anything else is refused before
    any launch."""
    st = cgb.lib().cgb_conj_grad_noalloc(100, 10, ctypes.c_void_p(256), ctypes.c_void_p(260),
                                          ctypes.c_void_p(264), ctypes.c_void_p(256),
                                          ctypes.c_void_p(256), ctypes.c_void_p(256), None, None)
    assert st == cgb.ERR_INVALID
    assert b"aligned" in cgb.lib().cgb_last_error()


def test_noalloc_rejects_oversize(cgb):
    n = 262145
    null = ctypes.c_void_p(1)
    st = cgb.lib().cgb_conj_grad_noalloc(n, 10, null, null, null, null, null, null, None, None)
    assert st == cgb.ERR_CAPACITY
    assert b"262144" in cgb.lib().cgb_last_error()
