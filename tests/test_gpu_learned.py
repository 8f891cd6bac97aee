"""GPU tests of the learned preconditioner (network kernels and the
preconditioned mixed-precision solver).

Network kernels against the CPU oracle oracle/gnn_oracle.py (float64):
forward G relative 1e-4, loss relative 1e-4, gradients norm-wise relative
2e-3 per parameter group (the GPU accumulates in FP32).  Solver results
against the reference's FP64 traces: zeta relative 1e-10, rnorm absolute
1e-10 * ||x||.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

pytestmark = pytest.mark.gpu

PARAMS = {"S": (1400, 7, 15, 10.0), "W": (7000, 8, 15, 12.0), "A": (14000, 11, 15, 20.0),
          "B": (75000, 13, 75, 60.0), "C": (150000, 15, 75, 110.0)}
VERIFY = {"S": 8.5971775078648, "B": 22.712745482631, "C": 28.973605592845}


def group_errors(go, g_gpu, g_ref):
    out = {}
    k = 0
    for name, shape in go.param_layout():
        size = int(np.prod(shape)) if shape else 1
        a, b = g_gpu[k:k + size].astype(np.float64), np.atleast_1d(g_ref[name]).ravel()
        out[name] = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        k += size
    return out


@pytest.fixture(scope="module")
def small_case(cgb):
    rs, ci, a = cgb.makea(1400, 7, 0.1, 10.0, 271828183.0)
    return rs, ci, a


def test_gnn_forward_matches_oracle(cgb, small_case):
    import gnn_oracle as go
    rs, ci, a = small_case
    model = cgb.Gnn(seed=7)
    p = go.unflatten(model.params)
    with model.graph(rs, ci, a) as g:
        goff, gdiag = model.infer(g)
        gref = go.Graph(rs, ci, a)
        G, _ = go.forward(p, gref)
        assert np.allclose(g.dscale, gref.dscale, rtol=1e-15)
    Gd = G.diagonal()
    low = __import__("scipy.sparse", fromlist=["tril"]).tril(G, k=-1).tocsr()
    low.sort_indices()
    assert len(goff) == low.nnz
    assert np.linalg.norm(gdiag - Gd) / np.linalg.norm(Gd) <= 1e-4
    assert np.linalg.norm(goff - low.data) / np.linalg.norm(low.data) <= 1e-4


def test_gnn_gradient_matches_oracle(cgb, small_case):
    import gnn_oracle as go
    rs, ci, a = small_case
    model = cgb.Gnn(seed=11)
    rng = np.random.default_rng(5)
    # perturb the initial weights so every path of the network is active
    model.params = model.params + rng.normal(0, 0.05, model.n_params).astype(np.float32)
    probes = rng.normal(size=(len(rs) - 1, 32)).astype(np.float32)
    with model.graph(rs, ci, a) as g:
        loss, grad = model.loss_grad(g, probes=probes)
    Lref, gref, _ = go.loss_and_grad(go.unflatten(model.params), go.Graph(rs, ci, a),
                                     probes.astype(np.float64))
    assert abs(loss - Lref) <= 1e-4 * abs(Lref)
    errs = group_errors(go, grad, gref)
    bad = {k: v for k, v in errs.items() if v > 2e-3}
    assert not bad, bad


def test_gnn_generated_probes_and_training_lowers_loss(cgb):
    model = cgb.Gnn(seed=3)
    mats = [cgb.makea(2000, 7, 0.1, 10.0, s) for s in (1000003.0, 1000005.0)]
    graphs = [model.graph(*m) for m in mats]
    first, last = [], []
    for step in range(60):
        g = graphs[step % 2]
        loss = model.train_step(g, seed=step, cg_steps=(0, 2, 4, 8)[step % 4], lr=2e-3)
        assert np.isfinite(loss)
        if step < 8:
            first.append(loss)
        elif step >= 52:
            last.append(loss)
    assert np.mean(last) < 0.8 * np.mean(first), (np.mean(first), np.mean(last))
    for g in graphs:
        g.close()


def test_pcg_with_identity_factor_is_plain_cg(cgb, golden):
    n, nonzer, niter, shift = PARAMS["S"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a) as s:
        s.set_preconditioner(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
                             np.ones(n))
        out = s.power_iterate(niter, shift, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
    ref = np.array(golden["S"]["seeds"]["314159265.0"]["zeta"])
    assert np.max(np.abs(out["zeta"] - ref) / np.abs(ref)) <= 1e-10
    assert out["fallbacks"] == 0


def test_pcg_rejects_bad_factor(cgb):
    n, nonzer, niter, shift = PARAMS["S"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a) as s:
        with pytest.raises(cgb.CgbError):
            s.power_iterate(3, shift, mode=cgb.MODE_MIXED_LEARNED)  # nothing installed
        with pytest.raises(cgb.CgbError):  # upper-triangular entry
            s.set_preconditioner(np.array([0, 1] + [2] * (n - 1), np.int32),
                                 np.array([1, 1], np.int32), np.ones(2))
        with pytest.raises(cgb.CgbError):  # non-positive diagonal
            s.set_preconditioner(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
                                 -np.ones(n))


def test_stalling_preconditioner_falls_back(cgb, golden):
    """A badly scaled SPD factor stalls PCG; the step falls back to plain CG
    and still reaches the reference zeta."""
    n, nonzer, niter, shift = PARAMS["S"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    d = np.where(np.arange(n) % 2 == 0, 1.0, 1e-3)
    with cgb.Session(rs, ci, a) as s:
        s.set_preconditioner(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), d)
        out = s.power_iterate(niter, shift, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=300)
    ref = np.array(golden["S"]["seeds"]["314159265.0"]["zeta"])
    assert np.max(np.abs(out["zeta"] - ref) / np.abs(ref)) <= 1e-10
    assert out["fallbacks"] > 0


def trained_model(cgb):
    """The committed weights when present, else a short training run."""
    model = cgb.Gnn()
    if os.path.exists(cgb.WEIGHTS_PATH):
        model.load()
        return model, "committed"
    for k, seed in enumerate((1000003.0, 1000005.0, 1000007.0, 1000009.0)):
        rs, ci, a = cgb.makea(14000, 11, 0.1, 20.0, seed)
        with model.graph(rs, ci, a) as g:
            for j in range(8):
                model.train_step(g, seed=8 * k + j, cg_steps=(0, 2, 4, 8)[j % 4], lr=2e-3)
    return model, "short run"


@pytest.mark.parametrize("tol", [1e-12, 1e-11, 1e-10])
def test_learned_preconditioner_class_c_unseen_seed(cgb, golden, tol):
    """Config: train on other seeds, test at n=150000, nonzer=15, shift=110
    (the NPB seed, never used in training); FP64 plain CG (the reference
    trace) is the yardstick for zeta: relative 1e-10 at every outer step, at the solver
    tolerances the benchmark reports (1e-10 is the configuration's own)."""
    model, how = trained_model(cgb)
    n, nonzer, niter, shift = PARAMS["C"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    with cgb.Session(rs, ci, a) as s, model.graph(rs, ci, a) as g:
        model.attach(g, s)
        out = s.power_iterate(niter, shift, mode=cgb.MODE_MIXED_LEARNED, tol=tol, cgitmax=200)
    ref = golden["C"]["seeds"]["314159265.0"]
    zr = np.array(ref["zeta"])
    assert np.max(np.abs(out["zeta"] - zr) / np.abs(zr)) <= 1e-10, how
    # rnorm: absolute 1e-10 * ||x_k|| (x_0 = ones, later x_k has unit norm)
    xnorm = np.r_[np.sqrt(n), np.ones(niter - 1)]
    assert np.all(np.abs(out["rnorm"] - np.array(ref["rnorm"])) <= 1e-10 * xnorm)


def test_learned_gain_over_method_without_it(cgb):
    """Ablation on an unseen matrix: the same preconditioned solver with the
    trained network's factor against the method without the network (F = I,
    i.e. plain CG) and Jacobi: inner iterations to the same tolerance and the
    training objective on fresh probes.  Records the numbers; asserts that
    training lowered the objective below the untrained network's and below
    F = I, and that the learned factor does not need more iterations than
    plain CG."""
    model, how = trained_model(cgb)
    n, nonzer, shift = 14000, 11, 20.0
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift, 987654321.0)
    kw = dict(mode=cgb.MODE_MIXED_LEARNED, tol=1e-10, cgitmax=200)
    with cgb.Session(rs, ci, a) as s, model.graph(rs, ci, a) as g:
        s.set_preconditioner(*cgb.identity_factor(n))
        plain = s.power_iterate(15, shift, **kw)
        s.set_preconditioner(*cgb.jacobi_factor(rs, ci, a))
        jac = s.power_iterate(15, shift, **kw)
        model.attach(g, s)
        lrn = s.power_iterate(15, shift, **kw)
        untrained = cgb.Gnn()
        loss_learned, _ = model.loss_grad(g, seed=99, cg_steps=4)
        loss_untrained, _ = untrained.loss_grad(g, seed=99, cg_steps=4)
        ident = cgb.Gnn()
        p = ident.params
        p[:] = 0.0
        p[ident.n_params - 34] = 0.5413249  # c_d: g_ii = softplus(c_d) = 1, g_ij = 0: G = I
        ident.params = p
        loss_identity, _ = ident.loss_grad(g, seed=99, cg_steps=4)
    for r in (jac, lrn):
        assert abs(r["zeta"][-1] - plain["zeta"][-1]) <= 1e-10 * abs(plain["zeta"][-1])
    print(f"\nablation ({how}): inner iterations plain={plain['total_inner']} "
          f"jacobi={jac['total_inner']} learned={lrn['total_inner']} "
          f"(fallbacks {lrn['fallbacks']}); loss learned={loss_learned:.4g} "
          f"untrained={loss_untrained:.4g} identity={loss_identity:.4g}")
    assert loss_learned < loss_untrained and loss_learned < loss_identity
    assert lrn["total_inner"] <= plain["total_inner"]


def test_learned_gain_in_wall_time(cgb):
    """What the network gains in time, on an unseen matrix where A is less
    well conditioned (n=7000, nonzer=8, shift=12: the NPB class W sizes at
    another seed): the same preconditioned solver (15 outer steps, tol
    1e-10) with the trained factor against F = I (the method without the
    network): fewer inner iterations and less device time, each the best
    of three solves, with zeta within 1e-10 of the FP64 reference
    algorithm.  (On class C, where A is nearly perfectly conditioned, the
    network's iterations do not pay for the factor products; the bench
    reports both.)"""
    model, how = trained_model(cgb)
    n, nonzer, shift = 7000, 8, 12.0
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift, 555555557.0)
    kw = dict(mode=cgb.MODE_MIXED_LEARNED, tol=1e-10, cgitmax=200)

    def best(s):
        s.power_iterate(15, shift, **kw)
        runs = [s.power_iterate(15, shift, **kw) for _ in range(3)]
        return min(runs, key=lambda r: r["device_ms"])

    with cgb.Session(rs, ci, a) as s, model.graph(rs, ci, a) as g:
        ref = s.power_iterate(15, shift)
        s.set_preconditioner(*cgb.identity_factor(n))
        ident = best(s)
        model.attach(g, s)
        lrn = best(s)
    for r in (ident, lrn):
        rel = np.max(np.abs(r["zeta"] - ref["zeta"]) / np.abs(ref["zeta"]))
        assert rel <= 1e-10, rel
    print(f"\nwall time ({how}): learned {lrn['device_ms']:.3f} ms / {lrn['total_inner']} its, "
          f"F = I {ident['device_ms']:.3f} ms / {ident['total_inner']} its")
    assert lrn["total_inner"] < 0.8 * ident["total_inner"]
    assert lrn["device_ms"] < 0.95 * ident["device_ms"]


def test_learned_sliced_plan_matches_row_plan(cgb, golden):
    """Class B with the trained factor under both SpMV policies: the sliced
    plan applies F and F^T through their own sliced copies (BF16 values,
    interleaved rows), the row plan through FP32 CSR rows; both reach the
    reference zeta trace."""
    model, how = trained_model(cgb)
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    zr = np.array(golden["B"]["seeds"]["314159265.0"]["zeta"])
    iters = {}
    for kind in (1, 2):
        with cgb.Session(rs, ci, a, spmv_kernel=kind) as s, model.graph(rs, ci, a) as g:
            assert s.plan()["kind"] == ("row" if kind == 1 else "sliced")
            model.attach(g, s)
            out = s.power_iterate(niter, shift, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
        assert np.max(np.abs(out["zeta"] - zr) / np.abs(zr)) <= 1e-10, (kind, how)
        iters[kind] = out["total_inner"]
    # same mathematics (the sliced copies hold F in BF16, the row plan in
    # FP32): iteration counts agree closely
    assert abs(iters[1] - iters[2]) <= 0.15 * iters[1], iters


def test_factor_rows_sorted_and_merged(cgb):
    """A factor given with unsorted rows and a repeated column equals the
    sorted, merged one (here Jacobi split into halves around an explicit
    zero), bit for bit, under the sliced plan."""
    n, nonzer, niter, shift = PARAMS["B"]
    rs, ci, a = cgb.makea(n, nonzer, 0.1, shift)
    fp, fc, fv = cgb.jacobi_factor(rs, ci, a)
    ptr, col, val = [0], [], []
    for i in range(n):
        ent = [(i, fv[i] / 2)] + ([(i - 1, 0.0)] if i > 0 else []) + [(i, fv[i] / 2)]
        for c, v in ent:
            col.append(c)
            val.append(v)
        ptr.append(len(col))
    kw = dict(mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
    with cgb.Session(rs, ci, a, spmv_kernel=2) as s:
        s.set_preconditioner(fp, fc, fv)
        ref = s.power_iterate(5, shift, **kw)
        s.set_preconditioner(np.array(ptr, np.int32), np.array(col, np.int32), np.array(val))
        out = s.power_iterate(5, shift, **kw)
    assert np.array_equal(out["zeta"], ref["zeta"])
    assert out["total_inner"] == ref["total_inner"]
