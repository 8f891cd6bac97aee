"""GPU tests of the batched persistent solver (cgb_batch).

FP64 mode is the reference algorithm, so each system must match the
single-system session (and the CPU oracle) to zeta relative 1e-10.  MIXED
mode is compared with the FP64 mode of the same batch: zeta relative 1e-10
where that FP64 solve has converged (its final rnorm <= 1e-10), and a system the
mixed iteration gives up on (status 1) is re-solved with the FP64 reference
algorithm, bit-identically.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def build(cgb, specs):
    systems, shifts = [], []
    for n, nonzer, shift, seed in specs:
        systems.append(cgb.makea(n, nonzer, 0.1, shift, seed))
        shifts.append(shift)
    return systems, np.array(shifts)


def test_batch_fp64_matches_single_system_and_oracle(cgb, oracle):
    specs = [(1400, 7, 10.0, 314159265.0), (2000, 9, 12.0, 271828183.0),
             (5000, 11, 15.0, 123456789.0), (700, 5, 8.0, 161803399.0),
             (9000, 13, 19.0, 987654321.0)]
    systems, shifts = build(cgb, specs)
    with cgb.Batch(systems, shifts) as b:
        out = b.solve(niter=15)
    for (rs, ci, a), sh, z in zip(systems, shifts, out["zeta"]):
        with cgb.Session(rs, ci, a) as s:
            ref = s.power_iterate(15, sh)["zeta"][-1]
        assert abs(z - ref) <= 1e-10 * abs(ref)
    rs, ci, a = systems[0]
    o = oracle.power_iterate(rs, ci, a, shifts[0], 15)
    assert abs(out["zeta"][0] - 8.5971775078648) / 8.5971775078648 <= 1e-10
    assert abs(out["zeta"][0] - o["zeta"][-1]) <= 1e-10 * abs(o["zeta"][-1])
    assert np.all(out["status"] == 0) and np.all(out["iters"] == 15 * 25)


def test_batch_mixed_against_fp64_reference(cgb):
    specs = cgb.uneven_batch_specs(nsys=48, seed=7, n_range=(1400, 8000))
    systems, shifts = build(cgb, specs)
    with cgb.Batch(systems, shifts) as b:
        fp64 = b.solve(niter=15)
        mixed = b.solve(niter=15, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=200)
    converged = fp64["rnorm"] <= 1e-10
    assert converged.sum() >= 10
    rel = np.abs(mixed["zeta"] - fp64["zeta"]) / np.abs(fp64["zeta"])
    ok = converged & (mixed["status"] == 0)
    assert np.all(rel[ok] <= 1e-10), rel[ok].max()
    fell = mixed["status"] == 1
    assert np.array_equal(mixed["zeta"][fell], fp64["zeta"][fell])
    assert mixed["iters"][ok].sum() < fp64["iters"][ok].sum()


def test_batch_indefinite_system_falls_back(cgb):
    """n=1400, nonzer=13, shift=11.4 is symmetric indefinite (eigenvalues
    from -11.3 to 11.4): the mixed iteration must give up on it and the
    system be solved with the reference algorithm, bit-identically."""
    specs = [(1400, 13, 11.4, 314159265.0), (1400, 7, 11.4, 314159265.0)]
    systems, shifts = build(cgb, specs)
    with cgb.Batch(systems, shifts) as b:
        fp64 = b.solve(niter=15)
        mixed = b.solve(niter=15, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=200)
    assert mixed["status"][0] == 1
    assert mixed["zeta"][0] == fp64["zeta"][0]
    assert mixed["status"][1] == 0
    assert abs(mixed["zeta"][1] - fp64["zeta"][1]) <= 1e-10 * abs(fp64["zeta"][1])


def test_batch_fallback_is_the_reference_algorithm(cgb):
    """A cap too small to converge makes every mixed solve give up; each
    system is then solved again with the FP64 reference algorithm (25 steps
    whatever the mixed cap), bit-identical to the FP64 mode."""
    specs = [(1400, 7, 10.0, 314159265.0), (3000, 11, 13.0, 271828183.0),
             (1400, 13, 11.4, 314159265.0)]
    systems, shifts = build(cgb, specs)
    with cgb.Batch(systems, shifts) as b:
        fp64 = b.solve(niter=5)
        mixed = b.solve(niter=5, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=2)
    assert np.all(mixed["status"] == 1)
    assert np.array_equal(mixed["zeta"], fp64["zeta"])
    assert np.array_equal(mixed["iters"], fp64["iters"])


def test_batch_galerkin_start(cgb):
    """The mixed mode's Galerkin start on previous iterates: the same
    answers (within 1e-10 of the FP64 fp64 where it converged) with fewer
    inner iterations than a start from z = 0."""
    specs = cgb.uneven_batch_specs(nsys=32, seed=5, n_range=(1400, 9000))
    systems, shifts = build(cgb, specs)
    with cgb.Batch(systems, shifts) as b:
        fp64 = b.solve(niter=15)
        cold = b.solve(niter=15, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=200, recycle=0)
        warm = b.solve(niter=15, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=200, recycle=4)
    conv = fp64["rnorm"] <= 1e-10
    for out in (cold, warm):
        ok = conv & (out["status"] == 0)
        rel = np.abs(out["zeta"] - fp64["zeta"]) / np.abs(fp64["zeta"])
        assert np.all(rel[ok] <= 1e-10), rel[ok].max()
        fell = out["status"] == 1
        assert np.array_equal(out["zeta"][fell], fp64["zeta"][fell])
    both = (cold["status"] == 0) & (warm["status"] == 0)
    assert both.sum() >= 8
    print(f"\nbatch inner iterations, z0 = 0 / Galerkin start: {cold['iters'][both].sum()} / "
          f"{warm['iters'][both].sum()}")
    assert warm["iters"][both].sum() < cold["iters"][both].sum()


def test_batch_tune_keeps_results(cgb):
    """Retuning changes lanes per row and block shape, hence the order of
    the row sums; converged systems keep zeta to 1e-10."""
    specs = cgb.uneven_batch_specs(nsys=24, seed=11, n_range=(1400, 6000))
    systems, shifts = build(cgb, specs)
    with cgb.Batch(systems, shifts) as b:
        before = b.solve(niter=3)
        cfg = b.tune(niter=1)
        after = b.solve(niter=3)
    assert cfg["block"] in (512, 1024) and cfg["best_ms"] > 0
    conv = before["rnorm"] <= 1e-10
    assert conv.sum() >= 12
    rel = np.abs(after["zeta"] - before["zeta"]) / np.abs(before["zeta"])
    assert np.all(rel[conv] <= 1e-10), rel[conv].max()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_batch_teams_match_single_cta(cgb, oracle, mode):
    """Systems split over teams of 2, 4 and 8 CTAs (rows shared, the search
    vector exchanged through global memory at each update) give the zeta of
    the one-CTA solve to 1e-10 (the sums only change order), and the FP64
    mode still matches the oracle."""
    specs = [(20000, 13, 30.0, 314159265.0), (9000, 11, 19.0, 271828183.0),
             (5000, 9, 15.0, 123456789.0), (1400, 7, 10.0, 314159265.0)]
    systems, shifts = build(cgb, specs)
    kw = dict(mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=200) if mode == "mixed" else {}
    with cgb.Batch(systems, shifts) as b:
        b.set_team_frac(0.0)
        alone = b.solve(niter=8, **kw)
        assert b.policy()["teams"] == 0
        b.set_team_frac(0.001)   # every system above 0.1 % of the work per CTA: teams of 8
        teams = b.solve(niter=8, **kw)
        assert b.policy()["teams"] == len(specs)
        # teams while the work per CTA is above 5 x the batch's mean per CTA:
        # the three larger systems (12.5 to 100 x), not the smallest (2.2 x)
        b.set_team_frac(5.0)
        some = b.solve(niter=8, **kw)
        assert b.policy()["teams"] == len(specs) - 1
    for out in (teams, some):
        assert np.array_equal(out["status"], alone["status"])
        rel = np.abs(out["zeta"] - alone["zeta"]) / np.abs(alone["zeta"])
        assert np.all(rel <= 1e-10), rel.max()
        if mode == "fp64":
            assert np.array_equal(out["iters"], alone["iters"])
    if mode == "fp64":
        rs, ci, a = systems[3]
        o = oracle.power_iterate(rs, ci, a, shifts[3], 8)
        assert abs(teams["zeta"][3] - o["zeta"][-1]) <= 1e-10 * abs(o["zeta"][-1])


def test_batch_rejects_oversize(cgb):
    rs = np.zeros(27002, np.int32)
    with pytest.raises(cgb.CgbError) as e:
        cgb.Batch([(rs, np.zeros(0, np.int32), np.zeros(0))], [1.0])
    assert e.value.status == cgb.ERR_CAPACITY


# ------------------------------------------------------------ learned mode
def learned_model(cgb):
    import os
    if not os.path.exists(cgb.WEIGHTS_PATH):
        pytest.skip("no trained weights")
    m = cgb.Gnn()
    m.load()
    return m


def test_batch_learned_against_fp64_reference(cgb):
    """CGB_MODE_MIXED_LEARNED with the trained network's factor per system:
    zeta relative 1e-10 against the FP64 reference algorithm of the same
    batch wherever that one converged; indefinite systems give up and are
    re-solved with the reference algorithm (bit-identical); the network
    needs fewer inner iterations than the unpreconditioned mixed mode on
    the systems both solved."""
    specs = cgb.uneven_batch_specs(nsys=48, seed=7, n_range=(1400, 8000))
    systems, shifts = build(cgb, specs)
    model = learned_model(cgb)
    with cgb.Batch(systems, shifts) as b:
        fp64 = b.solve(niter=15)
        mixed = b.solve(niter=15, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=200)
        b.attach_learned(model)
        lrn = b.solve(niter=15, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
        fb = b.fallbacks()
    model.close()
    converged = fp64["rnorm"] <= 1e-10
    rel = np.abs(lrn["zeta"] - fp64["zeta"]) / np.abs(fp64["zeta"])
    ok = converged & (lrn["status"] != 1)
    assert ok.sum() >= 10
    assert np.all(rel[ok] <= 1e-10), rel[ok].max()
    fell = lrn["status"] == 1
    assert np.array_equal(lrn["zeta"][fell], fp64["zeta"][fell])
    # the same systems are indefinite in both preconditioned and plain mixed
    assert np.array_equal(fell, mixed["status"] == 1)
    assert np.all((lrn["status"] == 2) == (fb > 0))
    both = ok & (mixed["status"] == 0)
    assert lrn["iters"][both].sum() < mixed["iters"][both].sum()


def test_batch_learned_identity_factor_is_plain_cg(cgb):
    """F = I: the preconditioned solver is plain CG, so it takes the mixed
    mode's iterations (to within a few per cent: the products round
    differently) and reaches the same zeta."""
    specs = cgb.uneven_batch_specs(nsys=24, seed=5, n_range=(1400, 6000))
    systems, shifts = build(cgb, specs)
    with cgb.Batch(systems, shifts) as b:
        b.set_team_frac(0.0)
        mixed = b.solve(niter=15, mode=cgb.MODE_MIXED, tol=1e-12, cgitmax=200)
        b.attach_identity()
        ident = b.solve(niter=15, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
    assert np.array_equal(ident["status"] == 1, mixed["status"] == 1)
    ok = mixed["status"] == 0
    rel = np.abs(ident["zeta"][ok] - mixed["zeta"][ok]) / np.abs(mixed["zeta"][ok])
    assert np.all(rel <= 1e-10)
    a, m = ident["iters"][ok].sum(), mixed["iters"][ok].sum()
    assert abs(a - m) <= 0.05 * m


def test_batch_learned_teams_agree(cgb):
    """Teams of CTAs (the largest systems split over 2-8 CTAs that exchange
    the FP32 vectors through global memory) against every system on one
    CTA: zeta relative 1e-10."""
    specs = cgb.uneven_batch_specs(nsys=16, seed=9, n_range=(6000, 20000))
    systems, shifts = build(cgb, specs)
    model = learned_model(cgb)
    with cgb.Batch(systems, shifts) as b:
        b.attach_learned(model)
        b.set_team_frac(0.0)
        solo = b.solve(niter=15, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
        b.set_team_frac(0.05)
        team = b.solve(niter=15, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
        assert b.policy()["teams"] > 0
    model.close()
    assert np.array_equal(solo["status"] == 1, team["status"] == 1)
    rel = np.abs(solo["zeta"] - team["zeta"]) / np.abs(solo["zeta"])
    assert np.all(rel <= 1e-10), rel.max()


def test_batch_learned_needs_every_factor(cgb):
    specs = [(1400, 7, 10.0, 314159265.0), (2000, 9, 12.0, 271828183.0)]
    systems, shifts = build(cgb, specs)
    with cgb.Batch(systems, shifts) as b:
        b.set_preconditioner(0, *cgb.identity_factor(1400))
        with pytest.raises(cgb.CgbError) as e:
            b.solve(niter=2, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=50)
        assert e.value.status == cgb.ERR_STATE
        with pytest.raises(cgb.CgbError) as e:
            b.set_preconditioner(1, np.zeros(2001, np.int32), np.zeros(0, np.int32), np.zeros(0))
        assert e.value.status == cgb.ERR_BAD_MATRIX


def test_batch_factor_rows_sorted_and_merged(cgb):
    """cgb_batch_set_preconditioner takes rows in any column order and sums
    repeated columns: a factor given with its rows reversed and each
    off-diagonal entry split in two halves solves bit for bit like the
    same factor given sorted."""
    specs = [(1400, 7, 10.0, 314159265.0), (2000, 9, 12.0, 271828183.0)]
    systems, shifts = build(cgb, specs)
    outs = []
    for shuffled in (False, True):
        with cgb.Batch(systems, shifts) as b:
            b.set_team_frac(0.0)
            for i, (rs, ci, a) in enumerate(systems):
                n = len(rs) - 1
                # F = I - 0.001 L (L: A's strict lower pattern, values 1)
                lptr, lcol = cgb.strict_lower_pattern(rs, ci)
                rows_p, rows_c, rows_v = [0], [], []
                for r in range(n):
                    cols = list(lcol[lptr[r]:lptr[r + 1]])
                    vals = [-1e-3] * len(cols)
                    if shuffled:
                        cols = cols[::-1] + cols
                        vals = [v / 2 for v in vals[::-1]] + [v / 2 for v in vals]
                        cols, vals = [r] + cols, [1.0] + vals
                    else:
                        cols, vals = cols + [r], vals + [1.0]
                    rows_c += cols
                    rows_v += vals
                    rows_p.append(len(rows_c))
                b.set_preconditioner(i, np.array(rows_p, np.int32), np.array(rows_c, np.int32),
                                     np.array(rows_v))
            outs.append(b.solve(niter=5, mode=cgb.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=100))
    assert np.array_equal(outs[0]["zeta"], outs[1]["zeta"])
    assert np.array_equal(outs[0]["iters"], outs[1]["iters"])
