"""GPU parity of the FP64 CG path through the C ABI (libcgb.so).

Compared with the reference's own outputs (tests/golden, oracle/_ref) and
the CPU oracle.  Tolerances:
  * zeta: relative 1e-10, the reference's verification epsilon (cg.cu:534-537);
  * rnorm: absolute 1e-10 * ||x|| (rnorm itself is roundoff, ~1e-13);
  * vectors after one conj_grad: relative 1e-12 of the vector norm (the GPU
    sums in a different order and with FMA).
"""
import os

import numpy as np
import pytest

from conftest import ref_lib_path

pytestmark = pytest.mark.gpu

PARAMS = {"S": (1400, 7, 15, 10.0), "W": (7000, 8, 15, 12.0), "A": (14000, 11, 15, 20.0),
          "B": (75000, 13, 75, 60.0), "C": (150000, 15, 75, 110.0)}
VERIFY = {"S": 8.5971775078648, "W": 10.362595087124, "A": 17.130235054029,
          "B": 22.712745482631, "C": 28.973605592845}


def session_for(cgb, cls, seed=314159265.0, **opts):
    n, nonzer, niter, shift = PARAMS[cls]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift, seed)
    return cgb.Session(rs, ci, a, **opts), (rs, ci, a)


def test_device_is_b200_class(cgb):
    info = cgb.device_info(0)
    assert info["cc"][0] == 10
    assert info["sm_count"] >= 100


def test_conj_grad_matches_reference_fixture(cgb):
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "conj_grad_S.npz"))
    s, (rs, ci, a) = session_for(cgb, "S")
    n = PARAMS["S"][0]
    z, p, q, r, rn = s.conj_grad(np.ones(n))
    xnorm = np.sqrt(n)
    # z and r = A z are converged quantities: relative agreement
    for name, got in (("z", z), ("r", r)):
        want = g[name]
        err = np.linalg.norm(got[:n] - want) / np.linalg.norm(want)
        assert err <= 1e-12, (name, err)
    # after 25 steps CG sits at roundoff: the last p and q are noise of size
    # ~1e-13 ||x||, comparable only in absolute terms (like rnorm)
    for name, got in (("p", p), ("q", q)):
        assert np.linalg.norm(got[:n] - g[name]) <= 1e-10 * xnorm, name
    assert abs(rn - g["rnorm"][0]) <= 1e-10
    # entry n, as the reference leaves it (cg.cu:670-675)
    assert z[n] == 0.0 and q[n] == 0.0 and r[n] == 1.0 and p[n] == 1.0


@pytest.mark.parametrize("cls", ["S", "W", "A", "B"])
def test_power_iterate_matches_reference(cgb, golden, cls):
    n, nonzer, niter, shift = PARAMS[cls]
    e = golden[cls]["seeds"]["314159265.0"]
    s, _ = session_for(cgb, cls)
    out = s.power_iterate(niter, shift)
    zeta = out["zeta"]
    ref_zeta = np.array(e["zeta"])
    assert np.max(np.abs(zeta - ref_zeta) / np.abs(ref_zeta)) <= 1e-10
    assert np.max(np.abs(out["rnorm"] - np.array(e["rnorm"]))) <= 1e-10
    assert abs(zeta[-1] - VERIFY[cls]) / VERIFY[cls] <= 1e-10
    assert np.all(out["iters"] == 25)
    assert out["device_ms"] > 0


@pytest.mark.slow
def test_power_iterate_class_c(cgb, golden):
    """The reference algorithm (fixed 25 CG steps) at class C against the
    reference's own trace, every outer step: zeta relative 1e-10, rnorm
    absolute 1e-10 (||x|| = 1 after the first step)."""
    n, nonzer, niter, shift = PARAMS["C"]
    e = golden["C"]["seeds"]["314159265.0"]
    s, _ = session_for(cgb, "C")
    out = s.power_iterate(niter, shift)
    ref_zeta = np.array(e["zeta"])
    assert len(ref_zeta) == niter
    assert np.max(np.abs(out["zeta"] - ref_zeta) / np.abs(ref_zeta)) <= 1e-10
    assert np.max(np.abs(out["rnorm"] - np.array(e["rnorm"]))) <= 1e-10
    assert np.all(out["iters"] == 25)
    assert abs(out["zeta"][-1] - VERIFY["C"]) / VERIFY["C"] <= 1e-10


def test_other_seeds_match_reference(cgb, golden):
    for cls in ("S", "A"):
        n, nonzer, niter, shift = PARAMS[cls]
        for key, e in golden[cls]["seeds"].items():
            s, _ = session_for(cgb, cls, seed=e["seed"])
            out = s.power_iterate(niter, shift)
            ref = np.array(e["zeta"])
            assert np.max(np.abs(out["zeta"] - ref) / np.abs(ref)) <= 1e-10


@pytest.mark.parametrize("lpr", [2, 4, 8, 16, 32])
def test_lane_counts_agree(cgb, golden, lpr):
    n, nonzer, niter, shift = PARAMS["W"]
    s, _ = session_for(cgb, "W", lanes_per_row=lpr)
    out = s.power_iterate(niter, shift)
    ref = np.array(golden["W"]["seeds"]["314159265.0"]["zeta"])
    assert np.max(np.abs(out["zeta"] - ref) / np.abs(ref)) <= 1e-10


def test_graph_and_direct_launch_agree_bitwise(cgb):
    n, nonzer, niter, shift = PARAMS["S"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    # the same kernel plan in both sessions (the autotuner may time two plans
    # within noise of each other), so the summation order is the same
    g = cgb.Session(rs, ci, a, use_graph=1, spmv_kernel=1, lanes_per_row=8).power_iterate(
        niter, shift, want_x=True)
    d = cgb.Session(rs, ci, a, use_graph=0, spmv_kernel=1, lanes_per_row=8).power_iterate(
        niter, shift, want_x=True)
    assert np.array_equal(g["zeta"], d["zeta"])
    assert np.array_equal(g["x"], d["x"])


def test_repeatable_bitwise(cgb):
    s, _ = session_for(cgb, "A")
    n, nonzer, niter, shift = PARAMS["A"]
    a1 = s.power_iterate(niter, shift, want_x=True)
    a2 = s.power_iterate(niter, shift, want_x=True)
    assert np.array_equal(a1["zeta"], a2["zeta"]) and np.array_equal(a1["x"], a2["x"])


def test_conj_grad_against_reference_library(cgb, oracle):
    path = ref_lib_path("S")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built")
    from oracle_py import RefLib
    ref = RefLib(path)
    n = ref.n
    rs, ci, a = ref.makea(123456789.0)
    s = cgb.Session(rs, ci, a)
    x = np.cos(np.arange(n) * 0.37) + 1.5
    zr, pr, qr, rr, rnr = ref.conj_grad(x)
    z, p, q, r, rn = s.conj_grad(x)
    assert np.linalg.norm(z[:n] - zr) <= 1e-12 * np.linalg.norm(zr)
    assert np.linalg.norm(r[:n] - rr) <= 1e-12 * np.linalg.norm(rr)
    assert np.linalg.norm(p[:n] - pr) <= 1e-10 * np.linalg.norm(x)
    assert np.linalg.norm(q[:n] - qr) <= 1e-10 * np.linalg.norm(x)
    assert abs(rn - rnr) <= 1e-10 * np.linalg.norm(x)


def test_reference_gpu_loop_matches_reference_trace(golden):
    """The reference's own GPU loop (conj_grad_gpu, compiled from its
    sources into oracle/_ref), which the bench times beside ours, computes
    the reference's trace: zeta relative 1e-10, rnorm absolute 1e-10."""
    path = ref_lib_path("S")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built")
    from oracle_py import RefLib
    ref = RefLib(path)
    ref.makea(copy_out=False)
    out = ref.power_gpu(ref.niter)
    e = golden["S"]["seeds"]["314159265.0"]
    assert out["seconds"] > 0
    assert np.max(np.abs(out["zeta"] - np.array(e["zeta"])) / np.array(e["zeta"])) <= 1e-10
    assert np.max(np.abs(out["rnorm"] - np.array(e["rnorm"]))) <= 1e-10


def test_conj_grad_reuploads_changed_matrix(cgb, oracle):
    n, nonzer, _, shift = PARAMS["S"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    s = cgb.Session(rs, ci, a)
    rs2, ci2, a2 = cgb.makea(n, nonzer, 0.1, shift, 271828183.0)
    s.upload(rs2, ci2, a2)
    z, *_ , rn = s.conj_grad(np.ones(n))
    zo, *_ = oracle.conj_grad(rs2, ci2, a2, np.ones(n))
    assert np.linalg.norm(z[:n] - zo[:n]) <= 1e-12 * np.linalg.norm(zo[:n])


def test_conj_grad_sees_in_place_edit_after_matrix_changed(cgb, oracle):
    """cgb_conj_grad re-uploads when the arrays' pointers change; an edit in
    place needs cgb_matrix_changed (the reference's CPU conj_grad reads a[]
    on every call)."""
    n, nonzer, _, shift = PARAMS["S"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    s = cgb.Session(rs, ci, a)
    x = np.ones(n)
    z0, *_ = s.conj_grad(x)
    held = s._keep[2]              # the very array the session was given
    held *= 1.5                    # still negative definite
    z_stale, *_ = s.conj_grad(x)   # same pointers: not seen
    assert np.array_equal(z_stale, z0)
    s.matrix_changed()
    z1, *_, rn1 = s.conj_grad(x)
    zo, *_, rno = oracle.conj_grad(rs, ci, held, x)
    assert np.linalg.norm(z1[:n] - zo[:n]) <= 1e-12 * np.linalg.norm(zo[:n])
    assert abs(rn1 - rno) <= 1e-10 * np.sqrt(n)
    # z of 1.5 A is z of A over 1.5
    assert np.linalg.norm(1.5 * z1[:n] - z0[:n]) <= 1e-11 * np.linalg.norm(z0[:n])


def test_tolerance_mode_reaches_reference_zeta(cgb, golden):
    n, nonzer, niter, shift = PARAMS["A"]
    s, _ = session_for(cgb, "A")
    out = s.power_iterate(niter, shift, mode=cgb.MODE_FP64_TOL, tol=1e-12, cgitmax=60)
    assert abs(out["zeta"][-1] - VERIFY["A"]) / VERIFY["A"] <= 1e-10
    assert out["total_inner"] < 25 * niter


def test_tiny_and_ragged_systems(cgb, oracle):
    """Edge shapes: fewer rows than CTAs, rows of very uneven length."""
    for n, nonzer, shift in ((40, 3, 2.0), (300, 2, 3.0), (1500, 20, 30.0)):
        rs, ci, a = cgb.makea(n, nonzer, 0.1, shift, 271828183.0)
        s = cgb.Session(rs, ci, a)
        out = s.power_iterate(5, shift)
        ref = oracle.power_iterate(rs, ci, a, shift, 5)
        assert np.max(np.abs(out["zeta"] - ref["zeta"]) / np.abs(ref["zeta"])) <= 1e-10


def test_empty_rows_handled(cgb):
    """A CSR with empty rows (the generator never makes one) still solves."""
    import scipy.sparse as sp
    n = 64
    d = -np.linspace(2.0, 3.0, n)
    d[::7] = -1.0
    A = sp.diags(d).tocsr()
    rs, ci, a = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data
    s = cgb.Session(rs, ci, a)
    z, p, q, r, rn = s.conj_grad(np.ones(n))
    assert np.allclose(z[:n], 1.0 / d, rtol=1e-14)


def test_wait_timeout_selftest_leaves_session_usable(cgb):
    s, _ = session_for(cgb, "S")
    st, dev = s.selftest_wait_timeout(50_000_000)  # 50 ms limit on a wait nobody ends
    assert st == cgb.ERR_TIMEOUT and dev == 1
    n, nonzer, niter, shift = PARAMS["S"]
    out = s.power_iterate(niter, shift)
    assert abs(out["zeta"][-1] - VERIFY["S"]) / VERIFY["S"] <= 1e-10


def test_barrier_timer_and_solve_after_it(cgb, golden):
    """The grid barrier's timer runs on the plan's grid, and the solve after
    it (the barrier count has moved on) still matches the reference trace."""
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a) as s:
        us = s.time_barrier(5000)
        assert 0.2 < us < 20.0
        out = s.power_iterate(niter, shift)
    ref = np.array(golden["B"]["seeds"]["314159265.0"]["zeta"])
    assert np.max(np.abs(out["zeta"] - ref) / np.abs(ref)) <= 1e-10


def test_spmv_timer_runs(cgb):
    s, _ = session_for(cgb, "A")
    ms = s.time_spmv(5)
    assert 0 < ms < 50


@pytest.mark.parametrize("kind,lpr", [(1, 8), (1, 16), (1, 32), (2, 0), (3, 0)])
def test_spmv_kernels_agree_class_b(cgb, golden, kind, lpr):
    """Row and sliced SpMV policies (sliced with and without the L2 prefetch)
    reproduce the reference trace."""
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a, spmv_kernel=kind, lanes_per_row=lpr) as s:
        plan = s.plan()
        assert plan["kind"] == {1: "row", 2: "sliced", 3: "sliced"}[kind]
        assert plan["l2_prefetch"] == (kind == 3)
        out = s.power_iterate(niter, shift)
        z, p, q, r, rn = s.conj_grad(np.ones(n))
    ref = np.array(golden["B"]["seeds"]["314159265.0"]["zeta"])
    assert np.max(np.abs(out["zeta"] - ref) / np.abs(ref)) <= 1e-10
    assert np.max(np.abs(out["rnorm"] - np.array(golden["B"]["seeds"]["314159265.0"]["rnorm"]))) <= 1e-10


def test_sliced_spmv_matches_oracle_product(cgb, oracle):
    """One sliced conj_grad against the oracle's on a non-constant x (class C)."""
    n, nonzer, niter, shift = PARAMS["C"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    x = 1.0 + 0.5 * np.sin(np.arange(n) * 0.001)
    with cgb.Session(rs, ci, a, spmv_kernel=2) as s:
        assert s.plan()["layout_entries"] >= len(a)
        z, p, q, r, rn = s.conj_grad(x)
    zo, po, qo, ro, rno = oracle.conj_grad(rs, ci, a, x)
    assert np.linalg.norm(z[:n] - zo[:n]) <= 1e-12 * np.linalg.norm(zo[:n])
    assert np.linalg.norm(r[:n] - ro[:n]) <= 1e-12 * np.linalg.norm(ro[:n])


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_l2_prefetch_changes_no_result(cgb, mode):
    """The prefetch only moves lines toward L2: the sliced plan with it gives
    bit-identical zeta and rnorm traces to the plan without it (class B)."""
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    kw = dict(mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=100) if mode == "mixed" else {}
    outs = []
    for kind in (2, 3):
        with cgb.Session(rs, ci, a, spmv_kernel=kind) as s:
            outs.append(s.power_iterate(5, shift, **kw))
    assert np.array_equal(outs[0]["zeta"], outs[1]["zeta"])
    assert np.array_equal(outs[0]["rnorm"], outs[1]["rnorm"])


@pytest.mark.parametrize("cls", ["B", "C"])
def test_l2_keep_changes_no_result(cgb, cls):
    """Keeping part of the matrix stream in L2 (evict_last loads) changes
    cache priorities only: zeta and rnorm traces are bit-identical with and
    without it, in the FP64 and the mixed mode."""
    n, nonzer, niter, shift = PARAMS[cls]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a, spmv_kernel=2) as s:
        outs = {}
        for keep in (0.0, 96e6):
            s.set_l2_keep(keep)
            assert abs(s.plan()["l2_keep_mb"] - keep / 1e6) < 1e-9
            outs[keep] = (s.power_iterate(4, shift),
                          s.power_iterate(4, shift, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=100))
    for k in (0, 1):
        assert np.array_equal(outs[0.0][k]["zeta"], outs[96e6][k]["zeta"])
        assert np.array_equal(outs[0.0][k]["rnorm"], outs[96e6][k]["rnorm"])


def test_row_panels_change_no_result(cgb):
    """Row panels -- a CTA walking its rows in pieces, every column block
    once per piece, as class D's 10 K rows a CTA need -- sum every row in
    the same order as one walk; only the fused dot products (p.q, r.y) add
    a CTA's rows in another order.  Forced at class B (panel_rows = 160),
    the z of one conj_grad and the FP64 zeta trace agree with the one-walk
    layout's to 1e-12 (rounding).  The mixed and preconditioned solves stop
    where the residual passes the tolerance, so rounding can move the stop
    by an iteration: their zetas agree to the parity bar, 1e-10.  A second
    session with panels repeats the first bit for bit (no race between a
    panel's output rows and the threads that read them next)."""
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    factor = cgb.jacobi_factor(rs, ci, a)
    outs, zs = [], []
    for rows in (0, 160, 160):
        with cgb.Session(rs, ci, a, spmv_kernel=2, panel_rows=rows) as s:
            pl = s.plan()
            assert pl["kind"] == "sliced"
            if rows:
                assert pl["panels"] >= 3 and pl["prec_panels"] >= 3, pl
            else:
                assert pl["panels"] == 1 and pl["prec_panels"] == 1, pl
            zs.append(s.conj_grad(np.ones(n))[0][:n])
            r = [s.power_iterate(4, shift),
                 s.power_iterate(4, shift, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=100)]
            s.set_preconditioner(*factor)
            r.append(s.power_iterate(4, shift, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=100))
            outs.append(r)
    assert np.linalg.norm(zs[0] - zs[1]) <= 1e-12 * np.linalg.norm(zs[0])
    for k in range(3):
        assert np.array_equal(outs[1][k]["zeta"], outs[2][k]["zeta"]), k
        assert outs[1][k]["total_inner"] == outs[2][k]["total_inner"], k
    for k, bound in enumerate((1e-12, 1e-10, 1e-10)):
        z0, z1 = outs[0][k]["zeta"], outs[1][k]["zeta"]
        assert np.max(np.abs(z0 - z1) / np.abs(z0)) <= bound, k
        assert np.all(outs[1][k]["rnorm"] <= 1e-10 * np.sqrt(n)), k  # 1e-10 ||x||, x = 1 first


def test_class_d_sliced_row_panels(cgb):
    """Class D (n = 1.5 M, 694 M entries; 10 K rows a CTA) on the sliced
    plan walks row panels; its first outer steps agree with the row plan's
    to 1e-12 (FP64, different summation order within rows)."""
    n, nonzer, shift = 1500000, 21, 500.0
    out = {}
    for kind in (1, 2):
        with cgb.Session.generated(n, nonzer, shift, spmv_kernel=kind) as s:
            pl = s.plan()
            assert pl["kind"] == ("row" if kind == 1 else "sliced")
            if kind == 2:
                assert pl["panels"] >= 4, pl
            out[kind] = s.power_iterate(2, shift)
    assert np.max(np.abs(out[1]["zeta"] - out[2]["zeta"]) / np.abs(out[1]["zeta"])) <= 1e-12
    assert np.all(out[2]["rnorm"] < 1e-10)


def test_sliced_refused_for_small_or_unsorted(cgb):
    n, nonzer, niter, shift = PARAMS["W"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with pytest.raises(cgb.CgbError) as e:
        cgb.Session(rs, ci, a, spmv_kernel=2)
    assert e.value.status == cgb.ERR_INVALID
    # a large CSR with one row's columns out of order: the autotuner must not pick sliced
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    ci = ci.copy()
    k0 = rs[10]
    ci[k0], ci[k0 + 1] = ci[k0 + 1], ci[k0]
    a = a.copy()
    a[k0], a[k0 + 1] = a[k0 + 1], a[k0]
    with cgb.Session(rs, ci, a) as s:
        assert s.plan()["kind"] == "row"
        out = s.power_iterate(3, shift)
    ok = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(*ok, spmv_kernel=1, lanes_per_row=16) as s2:
        ref = s2.power_iterate(3, shift)
    assert np.max(np.abs(out["zeta"] - ref["zeta"]) / np.abs(ref["zeta"])) <= 1e-12


def test_autotuned_plan_reported(cgb):
    n, nonzer, niter, shift = PARAMS["C"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a) as s:
        plan = s.plan()
    assert plan["kind"] in ("row", "sliced") and plan["grid"] >= 148


def test_reupload_same_structure_keeps_plan(cgb, oracle):
    """cgb_upload of new values under the same pattern rebuilds the sliced copy."""
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a, spmv_kernel=2) as s:
        a2 = a * 1.5
        s.upload(rs, ci, a2)
        assert s.plan()["kind"] == "sliced"
        x = np.ones(n)
        z, *_ = s.conj_grad(x)
    zo, *_ = oracle.conj_grad(rs, ci, a2, x)
    assert np.linalg.norm(z[:n] - zo[:n]) <= 1e-12 * np.linalg.norm(zo[:n])


def test_rejected_upload_keeps_the_matrix(cgb):
    """A re-upload is checked while it crosses to the device: a bad entry is
    reported (first bad index, as at create) and the session keeps solving
    with its previous matrix, bit-identically; a good upload then replaces
    it (reusing the captured graph)."""
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a) as s:
        ref = s.power_iterate(3, shift)
        bad_c = ci.copy()
        bad_c[len(ci) // 2] = n + 5
        with pytest.raises(cgb.CgbError) as e:
            s.upload(rs, bad_c, a)
        assert e.value.status == cgb.ERR_BAD_MATRIX
        assert f"colidx[{len(ci) // 2}]" in str(e.value)
        bad_a = a.copy()
        bad_a[7] = np.nan
        with pytest.raises(cgb.CgbError) as e:
            s.upload(rs, ci, bad_a)
        assert e.value.status == cgb.ERR_NUMERIC
        again = s.power_iterate(3, shift)
        assert np.array_equal(again["zeta"], ref["zeta"])
        s.upload(rs, ci, a * 2.0)
        doubled = s.power_iterate(3, shift)
    # the same sliced plan on a fresh session of 2A gives the same bits
    with cgb.Session(rs, ci, a * 2.0, spmv_kernel=2) as s2:
        fresh = s2.power_iterate(3, shift)
    assert np.array_equal(doubled["zeta"], fresh["zeta"])


@pytest.mark.parametrize("kind", [1, 2])
def test_mixed_precision_class_c(cgb, golden, kind):
    """FP32 SpMV inside FP64 refinement reaches the FP64 reference zeta.

    Config: n=150000, nonzer=15, shift=110, 75 outer steps; tolerance 1e-12
    on the true residual, warm start.  zeta error against the reference's
    FP64 trace: relative 1e-10 at every outer step; rnorm absolute 1e-10."""
    n, nonzer, niter, shift = PARAMS["C"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    ref = golden["C"]["seeds"]["314159265.0"]
    with cgb.Session(rs, ci, a, spmv_kernel=kind) as s:
        out = s.power_iterate(niter, shift, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=100)
    zeta_ref = np.array(ref["zeta"])
    assert np.max(np.abs(out["zeta"] - zeta_ref) / np.abs(zeta_ref)) <= 1e-10
    # rnorm: absolute 1e-10 * ||x_k|| (x_0 = ones, later x_k has unit norm)
    xnorm = np.r_[np.sqrt(n), np.ones(niter - 1)]
    assert np.all(np.abs(out["rnorm"] - np.array(ref["rnorm"])) <= 1e-10 * xnorm)
    assert out["refreshes"] >= niter          # every step ends on a true residual
    assert out["total_inner"] < 25 * niter


def test_mixed_precision_cold_start_class_b(cgb, golden):
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a) as s:
        out = s.power_iterate(niter, shift, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=100)
    zeta_ref = np.array(golden["B"]["seeds"]["314159265.0"]["zeta"])
    assert np.max(np.abs(out["zeta"] - zeta_ref) / np.abs(zeta_ref)) <= 1e-10


def test_fp32_spmv_close_to_fp64(cgb):
    """The FP32 SpMV of the session computes A p to FP32 accuracy (timing helper path)."""
    n, nonzer, niter, shift = PARAMS["C"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    for kind in (1, 2):
        with cgb.Session(rs, ci, a, spmv_kernel=kind) as s:
            assert s.time_spmv(3, fp32=True) > 0
            assert s.time_spmv(3, fp32=False) > 0


@pytest.mark.parametrize("mode", ["tol", "mixed"])
def test_galerkin_start_on_previous_iterates(cgb, golden, mode):
    """Tolerance modes start each solve from the Galerkin solution on the
    last 4 power-iteration iterates.  Config: class C (n=150000, nonzer=15,
    shift=110), 75 outer steps, tol 1e-12.  Against the reference's FP64
    trace: zeta relative 1e-10 at every step and rnorm absolute 1e-10*||x||,
    with and without the recycled start; the recycled start needs fewer
    inner iterations."""
    n, nonzer, niter, shift = PARAMS["C"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    ref = golden["C"]["seeds"]["314159265.0"]
    m = cgb.MODE_FP64_TOL if mode == "tol" else cgb.MODE_MIXED
    zr, rr = np.array(ref["zeta"]), np.array(ref["rnorm"])
    xnorm = np.r_[np.sqrt(n), np.ones(niter - 1)]
    inner = {}
    with cgb.Session(rs, ci, a) as s:
        for rec in (0, 4):
            out = s.power_iterate(niter, shift, mode=m, tol=1e-12, cgitmax=100, recycle=rec)
            assert np.max(np.abs(out["zeta"] - zr) / np.abs(zr)) <= 1e-10, rec
            assert np.all(np.abs(out["rnorm"] - rr) <= 1e-10 * xnorm), rec
            inner[rec] = out["total_inner"]
    print(f"\n{mode}: inner iterations without / with the recycled start: {inner[0]} / {inner[4]}")
    assert inner[4] < 0.85 * inner[0], inner


def test_recycle_rejects_out_of_range(cgb):
    n, nonzer, niter, shift = PARAMS["S"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a) as s:
        with pytest.raises(cgb.CgbError):
            s.power_iterate(2, shift, mode=cgb.MODE_FP64_TOL, recycle=5)
        # the reference mode ignores it
        out = s.power_iterate(niter, shift, recycle=4)
    assert abs(out["zeta"][-1] - VERIFY["S"]) / VERIFY["S"] <= 1e-10


def test_sessions_of_different_sizes_coexist(cgb):
    """A class-C session on the sliced plan, then a class-B one beside it (a
    smaller shared-memory need: fewer rows a CTA): the kernels' shared
    memory limit is one per process, and setting up the smaller session must
    not leave the larger one unable to launch.  Its results stay
    bit-identical."""
    n, nonzer, _, shift = PARAMS["C"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    na, nza, _, sha = PARAMS["B"]
    rsa, cia, aa = cgb.makea(na, nza, 0.1, sha)
    with cgb.Session(rs, ci, a, spmv_kernel=2) as big:
        first = big.power_iterate(2, shift)
        with cgb.Session(rsa, cia, aa, spmv_kernel=2) as small:
            small.power_iterate(2, sha)
            again = big.power_iterate(2, shift)
    assert np.array_equal(first["zeta"], again["zeta"])
    assert np.array_equal(first["rnorm"], again["rnorm"])
