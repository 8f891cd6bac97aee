"""Small, fixed workloads for profiling and tuning runs of libcgb.

    python npb-gpu_b200/npbcg/profile_case.py --cls B --what spmv --reps 3
    python npb-gpu_b200/npbcg/profile_case.py --cls B --what solve --niter 2
    python npb-gpu_b200/npbcg/profile_case.py --cls B --what sweep
    python npb-gpu_b200/npbcg/profile_case.py --what batch --nsys 64 --niter 2
    python npb-gpu_b200/npbcg/profile_case.py --cls B --what barrier --reps 20000
    python npb-gpu_b200/npbcg/profile_case.py --cls D --what part --ranks 1 --niter 1
    python npb-gpu_b200/npbcg/profile_case.py --what mg --mg-class A --niter 4
    python npb-gpu_b200/npbcg/profile_case.py --what ep --ep-class B
    python npb-gpu_b200/npbcg/profile_case.py --what is --is-class B
    python npb-gpu_b200/npbcg/profile_case.py --what ft --ft-class B

`spmv` launches the standalone FP64 SpMV+dot kernel `reps` times (after one
warm-up launch); `solve` runs one power iteration of `niter` outer steps;
`sweep` prints SpMV timings for every lanes-per-row choice; `part` runs the
row-partitioned solver on `ranks` device-generated row blocks, all driven
from this process; `mg` runs the MG benchmark's timed region (niter
V-cycles) of an MG class once after one warm-up run; `ep` runs the EP
kernel of an EP class once; `is` runs the IS benchmark (one untimed and ten
timed ranking passes, the full check) of an IS class once; `ft` runs the FT
benchmark's timed region of an FT class once after one warm-up run.  Each
prints one JSON line.
"""
import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import npbcg  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cls", default="B", choices=sorted(npbcg.CLASSES))
    ap.add_argument("--what", default="spmv",
                    choices=["spmv", "solve", "sweep", "batch", "barrier", "part", "mg", "ep", "is", "ft"])
    ap.add_argument("--ep-class", default="B", choices=sorted(npbcg.EP_CLASSES),
                    help="ep: the EP class")
    ap.add_argument("--ft-class", default="B", choices=sorted(npbcg.FT_CLASSES),
                    help="ft: the FT class")
    ap.add_argument("--is-class", default="B", choices=sorted(npbcg.IS_CLASSES),
                    help="is: the IS class")
    ap.add_argument("--mg-class", default="A", choices=sorted(npbcg.MG_CLASSES),
                    help="mg: the MG class")
    ap.add_argument("--ranks", type=int, default=1, help="part: row blocks")
    ap.add_argument("--mode", default="fp64", choices=["fp64", "mixed", "learned"],
                    help="solve / batch: the solver mode (mixed: tol 1e-12, cgitmax 100)")
    ap.add_argument("--nsys", type=int, default=64, help="batch: systems of the batched workload")
    ap.add_argument("--tune", action="store_true",
                    help="batch: run the autotuner first (12 launches at niter 1)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--niter", type=int, default=2)
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--kind", type=int, default=0, help="0 auto, 1 row, 2 sliced, 3 sliced with L2 prefetch")
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--panel-rows", type=int, default=0,
                    help="sliced plan: most rows a CTA sums at a time (forces row panels)")
    ap.add_argument("--keep-mb", type=float, default=None,
                    help="bytes (MB) of the sliced stream kept in L2 (default: the autotuner's)")
    a = ap.parse_args()
    kw = {} if a.mode == "fp64" else dict(
        mode=npbcg.MODE_MIXED if a.mode == "mixed" else npbcg.MODE_MIXED_LEARNED, tol=1e-12,
        cgitmax=100)
    if a.what == "batch":
        # the batched workload's first nsys systems, niter outer steps each
        specs = npbcg.uneven_batch_specs(nsys=a.nsys)
        systems = [npbcg.makea(n, nz, npbcg.RCOND, sh, seed) for n, nz, sh, seed in specs]
        with npbcg.Batch(systems, [sh for _, _, sh, _ in specs]) as b:
            if a.tune:
                b.tune(niter=1, **kw)
            r = b.solve(niter=a.niter, **kw)
            print(json.dumps({"what": "batch", "nsys": a.nsys, "niter": a.niter, "mode": a.mode,
                              "device_ms": r["device_ms"], "policy": b.policy()}), flush=True)
        return
    if a.what == "ep":
        r = npbcg.ep_run(npbcg.EP_CLASSES[a.ep_class]["m"])
        print(json.dumps({"what": "ep", "class": a.ep_class, "sx": r["sx"], "sy": r["sy"],
                          "device_ms": r["device_ms"]}), flush=True)
        return
    if a.what == "ft":
        nx, ny, nz, niter = npbcg.FT_CLASSES[a.ft_class]
        with npbcg.Ft(nx, ny, nz) as f:
            f.run(niter)
            r = f.run(niter)
        print(json.dumps({"what": "ft", "class": a.ft_class, "device_ms": r["device_ms"],
                          "max_rel_err": npbcg.ft_verify(a.ft_class, r["sums"])}), flush=True)
        return
    if a.what == "is":
        with npbcg.IntSort(a.is_class) as s:
            r = s.run()
        print(json.dumps({"what": "is", "class": a.is_class, "passed": r["passed"],
                          "device_ms": r["device_ms"]}), flush=True)
        return
    if a.what == "mg":
        with npbcg.Mg.for_class(a.mg_class) as g:
            g.run(a.niter)
            r = g.run(a.niter)
        print(json.dumps({"what": "mg", "class": a.mg_class, "niter": a.niter, **r}), flush=True)
        return
    c = npbcg.CLASSES[a.cls]
    if a.what == "part":
        parts = [npbcg.Part.generated(c["n"], c["nonzer"], c["shift"], world=a.ranks, rank=r)
                 for r in range(a.ranks)]
        r = npbcg.group_power_iterate(parts, a.niter, c["shift"])
        print(json.dumps({"cls": a.cls, "what": "part", "ranks": a.ranks, "niter": a.niter,
                          "nnz": sum(p.nnz for p in parts), "device_ms": r["device_ms"],
                          "zeta": float(r["zeta"][-1])}), flush=True)
        for p in parts:
            p.close()
        return
    rs, ci, av = npbcg.makea(c["n"], c["nonzer"], npbcg.RCOND, c["shift"])
    n, nnz = c["n"], len(av)
    out = {"cls": a.cls, "n": n, "nnz": nnz, "what": a.what}
    if a.what == "sweep":
        rows = []
        configs = [(1, l) for l in (8, 16, 32)] + [(2, 0)]
        for kind, lanes in configs:
            for fp32 in (False, True):
                try:
                    with npbcg.Session(rs, ci, av, spmv_kernel=kind, lanes_per_row=lanes) as s:
                        ms = s.time_spmv(50, fp32=fp32)
                        entries = s.plan()["layout_entries"]
                except npbcg.CgbError as e:
                    rows.append({"kind": kind, "lanes": lanes, "fp32": fp32, "error": str(e)})
                    continue
                b = (npbcg.spmv_bytes_fp32 if fp32 else npbcg.spmv_bytes_fp64)(n, nnz)
                rows.append({"kind": kind, "lanes": lanes, "fp32": fp32, "ms": ms,
                             "gbs": b / ms / 1e6, "layout_entries": entries})
        with npbcg.Session(rs, ci, av) as s:
            out["autotuned"] = s.plan()
        out["sweep"] = rows
    else:
        with npbcg.Session(rs, ci, av, lanes_per_row=a.lanes, spmv_kernel=a.kind,
                           panel_rows=a.panel_rows) as s:
            if a.keep_mb is not None:
                s.set_l2_keep(a.keep_mb * 1e6)
            out["plan"] = s.plan()
            if a.what == "barrier":
                out.update(us_per_barrier=[s.time_barrier(a.reps) for _ in range(3)])
            elif a.what == "spmv":
                ms = s.time_spmv(a.reps, fp32=a.fp32)
                b = (npbcg.spmv_bytes_fp32 if a.fp32 else npbcg.spmv_bytes_fp64)(n, nnz)
                out.update(ms=ms, gbs=b / ms / 1e6)
            else:
                if a.mode == "learned":
                    model = npbcg.Gnn()
                    model.load()
                    with model.graph(rs, ci, av) as g:
                        model.attach(g, s)
                r = s.power_iterate(a.niter, c["shift"], **kw)
                out.update(device_ms=r["device_ms"], zeta=float(r["zeta"][-1]))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
