"""Benchmark of the NPB CG inverse-power-iteration hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): the NPB class-B solve, n=75000, nonzer=13, shift=60,
rcond=0.1, seed 314159265 -- 75 outer steps x (25 CG iterations + residual)
in FP64, as the reference times it (GMAP/NPB-GPU CUDA/CG/cg.cu:491-522).
The CSR (13.7 M entries, 166 MB) is larger than the 126 MB L2, so no L2
flush is needed between steps.

Metric: SpMV-equivalent HBM GB/s = (SpMV algorithmic bytes x SpMVs per solve)
/ solve time, next to time-to-zeta (the solve's wall time with zeta within
1e-10 of the reference verification value).

Multi-GPU (torchrun, one rank per GPU): the class-B system is too small to
shard, so each rank solves its own replica (weak scaling, no data-path
collective); value = all ranks' bytes / the slowest rank's time.  Beside it,
`row_partitioned` splits one class-D system by rows over all ranks (strong
scaling: NCCL all-gather of p and two scalar all-reduces per CG step), and
`batched` shards the uneven batch by system.  `mg` runs the NPB MG
benchmark (class C) on every rank's GPU beside the reference's own GPU code
for MG, and `ep` the NPB EP benchmark (class C) likewise.

`--impl reference` times the reference's own CPU code (oracle/_ref, the
reference cg.cu compiled as is: serial, it has no threading) on the same
metric, rank 0 only.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "npb-gpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "SpMV HBM GB/s; time-to-zeta (rel err≤1e-10), learned/mixed vs plain CG"
CLASS = "B"
CGITMAX = 25
CPU_SAMPLE_STEPS = 20     # outer steps in the bounded CPU baseline sample
REF_STEP_OUTER = 4        # outer steps per reference-arm step


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def spmv_bytes(n, nnz):
    """FP64 CSR SpMV: 12 B/entry (value + int32 index), row pointers, p once, q once."""
    return 12 * nnz + 4 * (n + 1) + 8 * n + 8 * n


def outer_step_bytes(n, nnz, cgitmax=CGITMAX):
    """Algorithmic bytes of one outer-step kernel: per CG iteration the SpMV
    stream plus the fused vector work (p.q, z/r update with r.r, p update:
    12 nnz + 4(n+1) + 96 n), the residual SpMV with x.z, z.z (12 nnz +
    4(n+1) + 48 n) and the start of conj_grad (40 n)."""
    it = 12 * nnz + 4 * (n + 1) + 96 * n
    res = 12 * nnz + 4 * (n + 1) + 48 * n
    return cgitmax * it + res + 40 * n


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        busy = [v for v in sm if mx and v >= 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def physical_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",")]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


def load_traffic():
    """Per-launch DRAM bytes (ncu: dram__bytes_read.sum + dram__bytes_write.sum)
    of the kernels this bench reports, from the committed summary
    profiles/traffic_per_launch.txt -- used only when that summary was
    captured on this build: its `# build <hash>` line must equal the hash of
    the library's sources (npbcg.source_fingerprint).  Returns ({(kernel,
    workload): bytes}, a note saying where the numbers come from).  (ncu
    replays from cold caches: the L2 keep budget does not change them.)"""
    import npbcg
    path = os.path.join(ROOT, "profiles", "traffic_per_launch.txt")
    out, build = {}, None
    if os.path.exists(path):
        for line in open(path):
            parts = line.split()
            if line.startswith("# build") and len(parts) >= 3:
                build = parts[2]
            elif len(parts) >= 3 and not line.startswith("#"):
                try:
                    out[(parts[0], parts[1])] = float(parts[-1])
                except ValueError:
                    pass
    here = npbcg.source_fingerprint()
    if build != here:
        return {}, f"none: no ncu capture of this build ({here}; the summary is of {build})"
    return out, f"ncu capture of this build ({here}), profiles/traffic_per_launch.txt"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU arms
def cpu_reference_run(outer_steps, repeats=1, gpu_steps=0):
    """Times the reference's own serial CPU conj_grad loop (oracle/_ref);
    with gpu_steps > 0 also the reference's own GPU loop (conj_grad_gpu and
    its eleven kernels, cg.cu:489-522, 803-1265) on the same matrix, best of
    two runs after a warm-up: (n, nnz, CPU times, GPU run or None)."""
    from oracle_py import RefLib
    ref = RefLib(os.path.join(ROOT, "oracle", "_ref", f"libref_{CLASS}.so"))
    nnz = ref.makea(copy_out=False)
    times = []
    for _ in range(repeats):
        times.append(ref.power(outer_steps)["seconds"])
    gpu = None
    if gpu_steps > 0:
        ref.power_gpu(2)
        runs = [ref.power_gpu(gpu_steps) for _ in range(2)]
        gpu = min(runs, key=lambda r: r["seconds"])
    return ref.n, nnz, times, gpu


def cpu_openmp_run(rowstr, colidx, a, shift, outer_steps, threads):
    from oracle_py import Oracle
    o = Oracle(os.path.join(ROOT, "oracle", "liboracle.so"))
    return o.power_iterate(rowstr, colidx, a, shift, outer_steps, threads=threads)["seconds"]


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    c = CLASSES[CLASS]
    n, nnz, times, _ = cpu_reference_run(REF_STEP_OUTER, repeats=args.warmup + args.steps)
    timed = times[args.warmup:]
    per_step_bytes = REF_STEP_OUTER * (CGITMAX + 1) * spmv_bytes(n, nnz)
    total = sum(timed)
    value = per_step_bytes * len(timed) / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(timed), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference makea, seed 314159265)",
        "config": {"workload": f"NPB class {CLASS}: n={c['n']} nonzer={c['nonzer']} "
                               f"shift={c['shift']} rcond=0.1; each step {REF_STEP_OUTER} outer "
                               f"x (25 CG + residual) FP64 of the 75-step solve",
                   "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": 1, "kind": "reference",
                         "sample": f"{REF_STEP_OUTER} outer steps of class {CLASS} per step, "
                                   "reference cg.cu conj_grad compiled as is (serial)"},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------ solver modes
def solver_modes_section(npbcg, device):
    """Class C (n=150000, nonzer=15, shift=110, 75 outer steps): time to zeta
    of the FP64 reference algorithm on these kernels (fixed 25 CG steps)
    against the tolerance-stopped FP64 solver (from z = 0 and from the
    Galerkin start), the mixed-precision solver, and the preconditioned
    mixed-precision solver with F = I (the method without the network) and
    with the trained network's factor, at tolerances 1e-12, 1e-11 and 1e-10
    (the learned configuration's own); each compared with the FP64 plain
    zeta and rnorm of the same GPU run (every outer step) and the reference
    verification value."""
    c = npbcg.CLASSES["C"]
    n, niter, shift = c["n"], c["niter"], c["shift"]
    rs, ci, a = npbcg.makea(n, c["nonzer"], npbcg.RCOND, shift)
    out = {"workload": f"NPB class C: n={n} nonzer={c['nonzer']} shift={shift}, {niter} outer steps",
           "tol": 1e-12}

    def timed(s, **kw):
        s.power_iterate(niter, shift, **kw)          # builds the graph
        best = None
        for _ in range(2):
            r = s.power_iterate(niter, shift, **kw)
            if best is None or r["device_ms"] < best["device_ms"]:
                best = r
        return best

    nnz = len(a)
    # informative: the reference's own GPU loop on the same matrix, 75 steps
    # (best of two after a warm-up), before our sessions hold the device
    ref_gpu_ms = None
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libref_C.so")
    if os.path.exists(ref_path):
        from oracle_py import RefLib
        ref = RefLib(ref_path)
        ref.set_matrix(rs, ci, a)
        ref.power_gpu(2)
        ref_gpu = min((ref.power_gpu(niter) for _ in range(2)), key=lambda r: r["seconds"])
        ref_gpu_ms = 1e3 * ref_gpu["seconds"]
        out["reference_gpu_fixed25"] = {
            "ms": ref_gpu_ms, "zeta": float(ref_gpu["zeta"][-1]),
            "what": "the reference's conj_grad_gpu loop (cg.cu:489-522), wall time as its timer "
                    "takes it, on this GPU"}
    with npbcg.Session(rs, ci, a, device=device) as s:
        out["plan"] = s.plan()
        out["roofline_classC"] = class_c_roofline(npbcg, s, n, nnz, niter, shift)
        plain = timed(s)
        zp = float(plain["zeta"][-1])
        runs, tols = {"fp64_fixed25": plain}, {"fp64_fixed25": None}
        # tolerances: 1e-12, 1e-11, and 1e-10 -- the learned configuration's
        # own ("solve PCG to relative residual 1e-10 per outer step"); zeta
        # stays within 1e-10 of the FP64 reference algorithm at all three,
        # and every run states its own zeta and rnorm errors
        for tol, tag in ((1e-12, ""), (1e-11, "@tol1e-11"), (1e-10, "@tol1e-10")):
            kw = dict(tol=tol, cgitmax=100)
            if not tag:
                runs["fp64_tol_cold_start"] = timed(s, mode=npbcg.MODE_FP64_TOL, recycle=0, **kw)
                tols["fp64_tol_cold_start"] = tol
            runs["fp64_tol" + tag] = timed(s, mode=npbcg.MODE_FP64_TOL, **kw)
            runs["mixed" + tag] = timed(s, mode=npbcg.MODE_MIXED, **kw)
            # the preconditioned solver without the network: F = I
            s.set_preconditioner(*npbcg.identity_factor(n))
            runs["mixed_pcg_identity_factor" + tag] = timed(s, mode=npbcg.MODE_MIXED_LEARNED, **kw)
            if os.path.exists(npbcg.WEIGHTS_PATH):
                model = npbcg.Gnn(device=device)
                model.load()
                with model.graph(rs, ci, a) as g:
                    model.attach(g, s)
                runs["mixed_learned" + tag] = timed(s, mode=npbcg.MODE_MIXED_LEARNED, **kw)
                model.close()
            for k in runs:
                tols.setdefault(k, tol)
        for name, r in runs.items():
            z = float(r["zeta"][-1])
            out[name] = {"ms": r["device_ms"], "tol": tols[name], "zeta": z,
                         "zeta_rel_err_vs_fp64_plain": abs(z - zp) / abs(zp),
                         "zeta_rel_err_vs_verify": abs(z - c["zeta"]) / c["zeta"],
                         "max_step_zeta_rel_err_vs_fp64_plain":
                             float(np.max(np.abs(r["zeta"] - plain["zeta"]) / np.abs(plain["zeta"]))),
                         # ||x|| = 1 after the first outer step, sqrt(n) before
                         "rnorm": float(r["rnorm"][-1]),
                         "rnorm_abs_err_vs_fp64_plain": abs(float(r["rnorm"][-1]) -
                                                            float(plain["rnorm"][-1])),
                         "max_step_rnorm_abs_err_vs_fp64_plain":
                             float(np.max(np.abs(r["rnorm"] - plain["rnorm"]))),
                         "inner_iterations": int(r["total_inner"]),
                         "refreshes": int(r.get("refreshes", 0)),
                         "fallbacks": int(r.get("fallbacks", 0)),
                         "speedup_vs_fp64_fixed25": plain["device_ms"] / r["device_ms"],
                         "speedup_vs_reference_gpu": (ref_gpu_ms / r["device_ms"]
                                                      if ref_gpu_ms else None)}
    return out


def class_c_roofline(npbcg, s, n, nnz, niter, shift):
    """The SpMV roofline at class C (n=150000, nonzer=15): the plan's FP64
    outer-step kernel (25 CG iterations + the residual product a launch) and
    the standalone SpMV with the fused p.q (FP64 and FP32), each timed with
    CUDA events on the library's stream; algorithmic bytes as in
    outer_step_bytes / spmv_bytes; DRAM bytes from an ncu capture of this
    build when there is one; and what one kernel boundary costs the solve's
    CUDA graph (graphs of empty kernels of the outer step's shape)."""
    plan = s.plan()
    peak, peak_kind = peaks()
    if plan["kind"] == "sliced":
        kernel = "outer_step_fp64_sliced_pf" if plan["l2_prefetch"] else "outer_step_fp64_sliced"
        spmv_kernel = "spmv_dot_sliced_pf" if plan["l2_prefetch"] else "spmv_dot_sliced"
    else:
        kernel = f"outer_step_fp64<{plan['lanes_per_row']}>"
        spmv_kernel = f"spmv_dot_row<{plan['lanes_per_row']}>"
    kernel_ms, gap_ms = s.time_outer_steps(niter, shift)
    spmv_ms = s.time_spmv(50)
    spmv32_ms = s.time_spmv(50, fp32=True)
    table, note = load_traffic()
    ob = outer_step_bytes(n, nnz)
    sb = spmv_bytes(n, nnz)
    sb32 = 8 * nnz + 4 * (n + 1) + 8 * n
    out = {"workload": f"NPB class C: n={n} nonzer=15 nnz={nnz}", "peak": peak,
           "peak_source": peak_kind, "plan": plan}
    for name, k, ms, nbytes in (("outer_step", kernel, kernel_ms, ob),
                                ("spmv_fp64", spmv_kernel, spmv_ms, sb),
                                ("spmv_fp32", spmv_kernel.replace("spmv_dot_sliced", "spmv_dot_sliced32"),
                                 spmv32_ms, sb32)):
        gbs = nbytes / (ms / 1e3) / 1e9
        traffic = table.get((k.split("<")[0], "classC"))
        out[name] = {"kernel": k, "launch_ms": ms, "algorithmic_bytes_per_launch": nbytes,
                     "achieved_gbs": gbs, "frac": gbs / peak, "traffic": traffic,
                     "traffic_source": note if traffic is not None else
                     (note if not table else "none: kernel not in the capture")}
    out["graph_launch_overhead_ms_per_step"] = gap_ms
    return out


# -------------------------------------------------------------- batched
def batched_section(npbcg, device, nsys=512, niter=15, rank=0, world=1, dist=None):
    """512 generator systems (n log-uniform in [1400, 20000], nonzer in 7..13,
    shift = 10 + n/1000, own seeds) in one persistent launch per GPU: the
    FP64 reference algorithm (the yardstick) and the mixed-precision solver
    after the autotuner; aggregate solves/s and each system's zeta error
    against the FP64 reference algorithm.  With several ranks the systems
    are sharded by size (npbcg.batch_shard: no exchange during the solve),
    each rank solves its shard in its own launch, and rank 0 gathers the
    per-system results; the aggregate rate is all systems over the slowest
    rank's device time.  Returns None on ranks other than 0."""
    specs = npbcg.uneven_batch_specs(nsys=nsys)
    mine = list(range(nsys)) if world == 1 else npbcg.batch_shard(specs, rank, world)
    systems = [npbcg.makea(specs[i][0], specs[i][1], npbcg.RCOND, specs[i][2], specs[i][3])
               for i in mine]
    shifts = [specs[i][2] for i in mine]
    with npbcg.Batch(systems, shifts, device=device) as b:
        # the autotuner picks block shape, lanes per row and teams for each
        # mode, timing three outer steps (the tolerance modes reach their
        # Galerkin-started regime only after the first)
        tuned_fp64 = b.tune(niter=1)
        ref_run = b.solve(niter=niter)
        tuned = b.tune(niter=3, mode=npbcg.MODE_MIXED, tol=1e-12, cgitmax=200)
        mixed = b.solve(niter=niter, mode=npbcg.MODE_MIXED, tol=1e-12, cgitmax=200)
        learned = ident = tuned_l = None
        if os.path.exists(npbcg.WEIGHTS_PATH):
            # the learned preconditioner (one network inference per system),
            # then the same kernel with F = I (the method without the network)
            model = npbcg.Gnn(device=device)
            model.load()
            t0 = time.perf_counter()
            b.attach_learned(model)
            attach_s = time.perf_counter() - t0
            model.close()
            tuned_l = b.tune(niter=3, mode=npbcg.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
            learned = b.solve(niter=niter, mode=npbcg.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
            learned["fallbacks"] = b.fallbacks()
            learned["attach_s"] = attach_s
            b.attach_identity()
            ident = b.solve(niter=niter, mode=npbcg.MODE_MIXED_LEARNED, tol=1e-12, cgitmax=200)
    # algorithmic bytes of the FP64 reference algorithm: niter x (25 CG + residual) SpMVs per system
    local_bytes = sum(niter * (CGITMAX + 1) * spmv_bytes(len(s[0]) - 1, len(s[2])) for s in systems)
    local_nnz = sum(len(s[2]) for s in systems)
    has_l = learned is not None
    if world > 1:
        loc = {"zeta_ref": ref_run["zeta"], "rnorm_ref": ref_run["rnorm"], "zeta": mixed["zeta"],
               "status": mixed["status"], "iters": mixed["iters"],
               "device_ms": ref_run["device_ms"]}
        if has_l:
            loc.update(zeta_l=learned["zeta"], status_l=learned["status"], iters_l=learned["iters"],
                       fb_l=learned["fallbacks"], zeta_i=ident["zeta"], iters_i=ident["iters"])
        g_ref = npbcg.gather_shards(loc, mine, nsys, dist, rank)
        g_mix = npbcg.gather_shards({"device_ms": mixed["device_ms"]}, mine, nsys, dist, rank)
        g_l = npbcg.gather_shards({"device_ms": learned["device_ms"] if has_l else 0.0},
                                  mine, nsys, dist, rank)
        g_i = npbcg.gather_shards({"device_ms": ident["device_ms"] if has_l else 0.0},
                                  mine, nsys, dist, rank)
        tot = [None] * world if rank == 0 else None
        dist.gather_object((local_bytes, local_nnz, len(mine)), tot, dst=0)
        if rank != 0:
            return None
        ref_ms = max(g_ref["device_ms_per_rank"])
        mix_ms = max(g_mix["device_ms_per_rank"])
        if has_l:
            lrn = dict(zeta=g_ref["zeta_l"], status=g_ref["status_l"], iters=g_ref["iters_l"],
                       fallbacks=g_ref["fb_l"], device_ms=max(g_l["device_ms_per_rank"]))
            idn = dict(zeta=g_ref["zeta_i"], iters=g_ref["iters_i"],
                       device_ms=max(g_i["device_ms_per_rank"]))
        zref, rref, zmix = g_ref["zeta_ref"], g_ref["rnorm_ref"], g_ref["zeta"]
        status, iters = g_ref["status"], g_ref["iters"]
        total_bytes = sum(t[0] for t in tot)
        total_nnz = sum(t[1] for t in tot)
        shard_info = {"ranks": world, "systems_per_rank": [t[2] for t in tot],
                      "fp64_ms_per_rank": g_ref["device_ms_per_rank"],
                      "mixed_ms_per_rank": g_mix["device_ms_per_rank"]}
    else:
        ref_ms, mix_ms = ref_run["device_ms"], mixed["device_ms"]
        zref, rref, zmix = ref_run["zeta"], ref_run["rnorm"], mixed["zeta"]
        status, iters = mixed["status"], mixed["iters"]
        total_bytes, total_nnz, shard_info = local_bytes, local_nnz, None
        lrn, idn = learned, ident
    conv = rref <= 1e-10
    rel = np.abs(zmix - zref) / np.abs(zref)
    ref_gbs = total_bytes / (ref_ms / 1e3) / 1e9
    peak, _ = peaks()
    learned_out = None
    if has_l:
        rel_l = np.abs(lrn["zeta"] - zref) / np.abs(zref)
        rel_i = np.abs(idn["zeta"] - zref) / np.abs(zref)
        solved = lrn["status"] != 1
        learned_out = {
            "ms": lrn["device_ms"], "solves_per_s": nsys / lrn["device_ms"] * 1e3,
            "autotuned": tuned_l if world == 1 else "per rank",
            "attach_s": learned.get("attach_s"),
            "refit_in_fp64": int((lrn["status"] == 1).sum()),
            "systems_with_plain_cg_fallback": int((lrn["status"] == 2).sum()),
            "inner_iterations": int(lrn["iters"].sum()),
            "inner_iterations_preconditioned_systems": int(lrn["iters"][solved].sum()),
            "max_zeta_rel_err_converged": float(rel_l[conv].max()) if conv.any() else None,
            "within_1e-10_converged": int((rel_l[conv] <= 1e-10).sum()),
            "within_1e-10_all": int((rel_l <= 1e-10).sum()),
            "speedup_vs_fp64": ref_ms / lrn["device_ms"],
            "speedup_vs_mixed": mix_ms / lrn["device_ms"],
            "identity_factor": {
                "ms": idn["device_ms"], "inner_iterations_preconditioned_systems":
                    int(idn["iters"][solved].sum()),
                "max_zeta_rel_err_converged": float(rel_i[conv].max()) if conv.any() else None},
        }
    return {
        "workload": f"{nsys} systems, n log-uniform in [1400, 20000], nonzer 7..13, "
                    f"shift 10 + n/1000, {niter} outer steps each",
        "mixed_learned": learned_out,
        "total_nnz": int(total_nnz),
        "sharding": shard_info,
        "autotuned": {"fp64": tuned_fp64, "mixed": tuned} if world == 1 else "per rank",
        "fp64_reference": {"ms": ref_ms, "solves_per_s": nsys / ref_ms * 1e3,
                           "spmv_gbs": ref_gbs, "frac_of_peak": ref_gbs / (peak * world)},
        "mixed": {"ms": mix_ms, "solves_per_s": nsys / mix_ms * 1e3,
                  "refit_in_fp64": int((status == 1).sum()),
                  "inner_iterations": int(iters.sum())},
        "reference_converged_systems": int(conv.sum()),
        "max_zeta_rel_err_converged": float(rel[conv].max()) if conv.any() else None,
        "within_1e-10_converged": int((rel[conv] <= 1e-10).sum()),
        "within_1e-10_all": int((rel <= 1e-10).sum()),
        "speedup_mixed_vs_fp64": ref_ms / mix_ms,
    }


# ------------------------------------------------------------------- our arm
CLASSES = None


PART_CLASS = "D"


def row_partitioned_section(npbcg, device, rank, world, dist):
    """Class D as one system split by rows over the ranks (npbcg.Part: each
    rank generates and holds its row block; per CG step an NCCL all-gather
    of p and two scalar all-reduces, all on the device).  Every rank takes
    the same steps; the time is the slowest rank's device time."""
    import torch
    c = dict(npbcg.CLASSES[PART_CLASS], name=PART_CLASS)
    nid = npbcg.nccl_unique_id() if rank == 0 else None
    dev = "cuda" if dist is None or dist.get_backend() == "nccl" else "cpu"
    if dist is not None:
        box = [nid]
        dist.broadcast_object_list(box, src=0)
        nid = box[0]
    # every rank builds its block first; the communicator is joined only
    # when all of them have one, so a rank that failed cannot leave the
    # others waiting in a collective
    part, err = None, None
    try:
        part = npbcg.Part.generated(c["n"], c["nonzer"], c["shift"], world=world, rank=rank,
                                    device=device)
    except npbcg.CgbError as e:
        err = str(e)
    ok = torch.tensor([0.0 if part is None else 1.0], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(ok, op=dist.ReduceOp.MIN)
    if ok.item() < 1.0:
        if part is not None:
            part.close()
        return {"unavailable": err or "another rank could not build its row block"} if rank == 0 else None
    part.join(nid)
    part.set_wait_limit(300.0)
    try:
        part.power_iterate(1, c["shift"])  # warm-up (the reference's untimed step)
        if dist is not None:
            dist.barrier()
        out = part.power_iterate(c["niter"], c["shift"])
        ms, nnz = out["device_ms"], part.nnz
        if dist is not None:
            t = torch.tensor([ms, float(nnz)], dtype=torch.float64, device=dev)
            tmax = t.clone()
            dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
            dist.all_reduce(t)
            ms, nnz = float(tmax[0].item()), int(t[1].item())
    finally:
        part.close()
    if rank != 0:
        return None
    zeta = float(out["zeta"][-1])
    solve_bytes = c["niter"] * (CGITMAX + 1) * spmv_bytes(c["n"], nnz)
    return {
        "what": f"NPB class {c['name']} (n={c['n']}, nnz={nnz}) split into {world} row block(s), "
                "one per rank, generated on each rank's GPU; reference algorithm, "
                f"{c['niter']} outer steps; NCCL all-gather of p + 2 scalar all-reduces per CG step, "
                "outer step captured as a CUDA graph",
        "ranks": world, "seconds": ms / 1e3, "ms_per_outer_step": ms / c["niter"],
        "value": solve_bytes / (ms / 1e3) / 1e9, "unit": "GB/s (algorithmic, whole job)",
        "zeta": zeta, "zeta_rel_err_vs_verify": abs(zeta - c["zeta"]) / c["zeta"],
        "verified": abs(zeta - c["zeta"]) / c["zeta"] <= 1e-10,
    }


MG_CLASS = "C"


def mg_section(npbcg, device, rank, world, dist):
    """NPB MG class C (512^3, 20 V-cycles) on each rank's GPU (replicas: the
    MG grid is not split), next to the reference's own GPU code for MG on
    the same GPU and its serial CPU code (rank 0, one GPU)."""
    import torch
    c = npbcg.MG_CLASSES[MG_CLASS]
    n = 1 << c["lt"]
    with npbcg.Mg.for_class(MG_CLASS, device) as g:
        g.run(c["nit"])  # the graph's capture and a warm-up
        runs = [g.run(c["nit"]) for _ in range(3)]
    ms = max(r["device_ms"] for r in runs)
    if dist is not None:
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if rank != 0:
        return None
    rnm2 = runs[-1]["rnm2"]
    nbytes = npbcg.mg_region_bytes(c["lt"], c["nit"])
    peak, peak_kind = peaks()
    out = {
        "what": f"NPB MG class {MG_CLASS}: {n}^3 grid, {c['nit']} V-cycles (resid, psinv, rprj3, "
                "interp kernels, timed region as one CUDA graph), FP64",
        "ms": ms, "mops": 58.0 * c["nit"] * n ** 3 * 1e-6 / (ms / 1e3),
        "rnm2": rnm2, "rel_err_vs_verify": abs(rnm2 - c["rnm2"]) / c["rnm2"],
        "verified": abs(rnm2 - c["rnm2"]) / c["rnm2"] <= npbcg.MG_VERIFY_EPSILON,
        "algorithmic_bytes": nbytes, "achieved_gbs": nbytes / (ms / 1e3) / 1e9,
        "frac_of_peak": nbytes / (ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
        "replicas": world,
    }
    ref_path = os.path.join(ROOT, "oracle", "_ref", f"libref_mg_{MG_CLASS}.so")
    if world == 1 and os.path.exists(ref_path):
        from oracle_py import RefMgLib
        ref = RefMgLib(ref_path)
        ref.gpu()
        rg = min((ref.gpu() for _ in range(2)), key=lambda r: r["seconds"])
        out["reference_gpu"] = {
            "what": "the reference's timed MG region on this GPU (mg.cu:486-517: resid_gpu, "
                    "norm2u3_gpu, mg3P_gpu ...), compiled from its sources with its device flags",
            "ms": rg["seconds"] * 1e3, "rnm2": rg["rnm2"],
            "our_speedup": rg["seconds"] * 1e3 / ms,
        }
    return out


EP_CLASS = "C"


def ep_section(npbcg, device, rank):
    """NPB EP class C (2^32 pairs) on each rank's GPU, next to the reference's
    own EP kernel on the same GPU (rank 0).  The reference's timer stops right
    after its kernel launch (ep.cu:166-172); its time here is the wall time to
    its sums on the host."""
    c = npbcg.EP_CLASSES[EP_CLASS]
    npbcg.ep_run(c["m"], device)  # warm-up
    runs = [npbcg.ep_run(c["m"], device) for _ in range(3)]
    if rank != 0:
        return None
    ms = max(r["device_ms"] for r in runs)
    r = runs[-1]
    out = {
        "what": f"NPB EP class {EP_CLASS}: 2^{c['m']} pairs, one kernel, FP64 log/sqrt",
        "ms": ms, "mops": 2.0 ** (c["m"] + 1) / (ms / 1e3) / 1e6,
        "sx_rel_err": abs(r["sx"] - c["sx"]) / abs(c["sx"]),
        "sy_rel_err": abs(r["sy"] - c["sy"]) / abs(c["sy"]),
        "verified": max(abs(r["sx"] - c["sx"]) / abs(c["sx"]),
                        abs(r["sy"] - c["sy"]) / abs(c["sy"])) <= npbcg.EP_VERIFY_EPSILON,
    }
    ref_path = os.path.join(ROOT, "oracle", "_ref", f"libref_ep_{EP_CLASS}.so")
    if os.path.exists(ref_path):
        from oracle_py import RefEpLib
        ref = RefEpLib(ref_path)
        ref.gpu()
        rg = min((ref.gpu() for _ in range(2)), key=lambda x: x["seconds_wall"])
        out["reference_gpu"] = {
            "what": "the reference's EP kernel on this GPU (ep.cu:159-186: one thread per batch of "
                    "2^16 pairs), compiled from its sources with its device flags; wall time to "
                    "its sums on the host",
            "ms": rg["seconds_wall"] * 1e3, "our_speedup": rg["seconds_wall"] * 1e3 / ms,
        }
    return out


IS_CLASS = "C"


def is_section(npbcg, device, rank):
    """NPB IS class C (2^27 keys below 2^23) on each rank's GPU, next to the
    reference's own IS kernels on the same GPU (rank 0).  Both times cover the
    ten timed ranking passes (is.cu:415-430); the reference's is the wall time
    to a device synchronisation after its tenth pass."""
    total_log2, max_log2 = npbcg.IS_CLASSES[IS_CLASS]
    with npbcg.IntSort(IS_CLASS, device=device) as s:
        runs = [s.run() for _ in range(4)][1:]
    if rank != 0:
        return None
    ms = max(r["device_ms"] for r in runs)
    keys = float(1 << total_log2)
    out = {
        "what": f"NPB IS class {IS_CLASS}: 2^{total_log2} keys below 2^{max_log2}, ten ranking passes",
        "ms": ms, "mops": 10.0 * keys / (ms / 1e3) / 1e6,
        "passed": min(r["passed"] for r in runs), "verified": all(r["passed"] == npbcg.IS_PASSED for r in runs),
    }
    ref_path = os.path.join(ROOT, "oracle", "_ref", f"libref_is_{IS_CLASS}.so")
    if os.path.exists(ref_path):
        from oracle_py import RefIsLib
        ref = RefIsLib(ref_path)
        ref.gpu()
        rg = min((ref.gpu() for _ in range(2)), key=lambda x: x["seconds"])
        out["reference_gpu"] = {
            "what": "the reference's IS kernels on this GPU (is.cu rank_gpu: seven kernels a pass), "
                    "compiled from its sources with its block sizes; wall time of the ten passes",
            "ms": rg["seconds"] * 1e3, "passed": rg["passed"], "our_speedup": rg["seconds"] * 1e3 / ms,
        }
    return out


FT_CLASS = "C"


def ft_section(npbcg, device, rank):
    """NPB FT class C (512^3, 20 iterations) on each rank's GPU, next to the
    reference's own FT kernels on the same GPU (rank 0).  Both times cover
    main's timed region (ft.cu:391-412); the reference's is its wall time to
    the checksums on the host."""
    nx, ny, nz, niter = npbcg.FT_CLASSES[FT_CLASS]
    with npbcg.Ft(nx, ny, nz, device=device) as f:
        runs = [f.run(niter) for _ in range(4)][1:]
    if rank != 0:
        return None
    ms = max(r["device_ms"] for r in runs)
    nt = float(nx * ny * nz)
    # ft.cu:418-421
    mflops = 1.0e-6 * nt * (14.8157 + 7.19641 * np.log(nt) + (5.23518 + 7.21113 * np.log(nt)) * niter) / (ms / 1e3)
    # the initial conditions (16 B a point written), the forward transform
    # (3 passes, 32 B each), per iteration 3 passes of 32 B (the first reads
    # u0 and writes u1), and u0 written back once (16 B)
    algorithmic = nt * (16 + 3 * 32 + niter * 3 * 32 + 16)
    out = {
        "what": f"NPB FT class {FT_CLASS}: {nx}x{ny}x{nz}, {niter} iterations (one shared-memory "
                "Stockham pass an axis, evolve fused into the z pass), FP64",
        "ms": ms, "mflops": mflops,
        "max_rel_err": max(npbcg.ft_verify(FT_CLASS, r["sums"]) for r in runs),
        "verified": all(npbcg.ft_verify(FT_CLASS, r["sums"]) <= npbcg.FT_VERIFY_EPSILON for r in runs),
        "algorithmic_bytes": algorithmic, "achieved_gbs": algorithmic / (ms / 1e3) / 1e9,
    }
    ref_path = os.path.join(ROOT, "oracle", "_ref", f"libref_ft_{FT_CLASS}.so")
    if os.path.exists(ref_path):
        from oracle_py import RefFtLib
        ref = RefFtLib(ref_path)
        rg = ref.gpu()
        out["reference_gpu"] = {
            "what": "the reference's timed FT region on this GPU (ft.cu:391-412: radix-2 Stockham "
                    "stages in global memory), compiled from its sources with its block sizes",
            "ms": rg["seconds"] * 1e3, "our_speedup": rg["seconds"] * 1e3 / ms,
            "max_rel_err": npbcg.ft_verify(FT_CLASS, rg["sums"]),
        }
    return out


def our_arm(args, rank, world, local_rank):
    import torch
    import npbcg

    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    else:
        torch.cuda.set_device(local_rank)
    device = local_rank

    c = npbcg.CLASSES[CLASS]
    n, niter, shift = c["n"], c["niter"], c["shift"]
    rs, ci, a = npbcg.makea(n, c["nonzer"], npbcg.RCOND, shift)
    nnz = len(a)
    lib = npbcg.lib()

    # pinned host copies for the end-to-end leg
    def pinned(arr):
        p = ctypes.c_void_p()
        npbcg._check(lib.cgb_host_alloc(ctypes.byref(p), arr.nbytes))
        buf = (ctypes.c_char * arr.nbytes).from_address(p.value)
        out = np.frombuffer(buf, dtype=arr.dtype)
        out[:] = arr
        return out, p

    h_rs, p_rs = pinned(rs)
    h_ci, p_ci = pinned(ci)
    h_a, p_a = pinned(a)

    sess = npbcg.Session(h_rs, h_ci, h_a, device=device)
    solve_bytes = niter * (CGITMAX + 1) * spmv_bytes(n, nnz)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def reduce_max(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(max(args.warmup, 3)):
        out = sess.power_iterate(niter, shift)

    # ---- device-resident timed region
    sampler = ClockSampler(physical_index(local_rank))
    barrier()
    sampler.start()
    dev_ms = []
    for _ in range(args.steps):
        out = sess.power_iterate(niter, shift)
        dev_ms.append(out["device_ms"])
    barrier()
    clocks = sampler.stop()
    total_ms = reduce_max(sum(dev_ms))
    zeta = float(out["zeta"][-1])
    zeta_err = abs(zeta - c["zeta"]) / c["zeta"]
    value = world * args.steps * solve_bytes / (total_ms / 1e3) / 1e9
    ms_per_step = total_ms / args.steps

    # ---- end to end through the C ABI: H2D of the CSR from pinned memory,
    # the solve, D2H of the traces and of x, every step
    h2d = 4 * (n + 1) + 12 * nnz
    d2h = niter * (8 + 8 + 4) + 8 * n
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sess.upload(h_rs, h_ci, h_a)
        e2e_out = sess.power_iterate(niter, shift, want_x=True)
    barrier()
    e2e_s = reduce_max(time.perf_counter() - t0)
    e2e_value = world * args.steps * solve_bytes / e2e_s / 1e9

    # ---- roofline of the dominant kernel (the outer-step kernel): its
    # average launch duration from CUDA events around each launch on the
    # library's stream, algorithmic bytes per launch from outer_step_bytes
    plan = sess.plan()
    if plan["kind"] == "sliced":
        kernel = "outer_step_fp64_sliced_pf" if plan["l2_prefetch"] else "outer_step_fp64_sliced"
    else:
        kernel = f"outer_step_fp64<{plan['lanes_per_row']}>"
    kernel_ms, gap_ms = sess.time_outer_steps(niter, shift)
    bytes_launch = outer_step_bytes(n, nnz)
    achieved = bytes_launch / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic_table, traffic_note = load_traffic()
    traffic = traffic_table.get((kernel.split("<")[0], f"class{CLASS}"))
    spmv_ms = sess.time_spmv(50)
    spmv_gbs = spmv_bytes(n, nnz) / (spmv_ms / 1e3) / 1e9

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the reference makea generator, seed 314159265)",
            "config": {
                "workload": f"NPB class {CLASS}: n={n} nonzer={c['nonzer']} shift={shift} "
                            f"rcond=0.1 nnz={nnz}; {niter} outer x ({CGITMAX} CG + residual) FP64, "
                            "one persistent cooperative kernel per outer step, CUDA graph per solve",
                "l2": "inputs larger than L2 (CSR 166 MB > 126 MB L2), no flush",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            },
            "time_to_zeta_s": ms_per_step / 1e3,
            "zeta": zeta, "zeta_rel_err": zeta_err,
            "spmv_standalone": {"ms": spmv_ms, "gbs": spmv_gbs,
                                "frac_of_peak": spmv_gbs / peak},
            "outer_step_kernel_ms": kernel_ms,
            "graph_launch_overhead_ms_per_step": gap_ms,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                         "algorithmic_bytes_per_launch": bytes_launch,
                         "launch_ms": kernel_ms, "peak_source": peak_kind,
                         "traffic_source": traffic_note if traffic is not None else
                         (traffic_note if not traffic_table else "none: kernel not in the capture")},
            "plan": plan,
            "clocks": clocks,
            "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps * (niter + 1),
        }
        if not args.no_solver_modes:
            line["solver_modes"] = solver_modes_section(npbcg, device)
            line["roofline_classC"] = line["solver_modes"].pop("roofline_classC")
        if world == 1 and not args.no_cpu_baseline:
            nref, nnz_ref, times, rgpu = cpu_reference_run(CPU_SAMPLE_STEPS, gpu_steps=niter)
            sample_bytes = CPU_SAMPLE_STEPS * (CGITMAX + 1) * spmv_bytes(nref, nnz_ref)
            # informative: the reference's own CUDA code on this GPU, the same
            # 75-step solve, its wall time as the reference's timer takes it
            rg_bytes = niter * (CGITMAX + 1) * spmv_bytes(nref, nnz_ref)
            line["reference_gpu"] = {
                "what": "the reference's conj_grad_gpu loop (cg.cu:489-522, 803-1265), compiled "
                        "from its sources with its device flags for sm_100a, same matrix",
                "seconds": rgpu["seconds"], "value": rg_bytes / rgpu["seconds"] / 1e9,
                "unit": "GB/s", "zeta": float(rgpu["zeta"][-1]),
                "zeta_rel_err_vs_verify": abs(float(rgpu["zeta"][-1]) - c["zeta"]) / c["zeta"],
                "our_device_speedup": (rgpu["seconds"] * 1e3) / ms_per_step,
                "our_e2e_speedup": e2e_value / (rg_bytes / rgpu["seconds"] / 1e9),
            }
            ser = sample_bytes / times[0] / 1e9
            threads = os.cpu_count() or 1
            omp_s = cpu_openmp_run(rs, ci, a, shift, CPU_SAMPLE_STEPS, threads)
            line["cpu_baseline"] = {
                "value": ser, "unit": "GB/s", "cores": 1, "kind": "reference",
                "sample": f"{CPU_SAMPLE_STEPS} of {niter} outer steps of class {CLASS}, the "
                          "reference's serial conj_grad loop (oracle/_ref)",
                "seconds": times[0],
                "openmp_port": {"value": sample_bytes / omp_s / 1e9, "unit": "GB/s",
                                "cores": threads, "kind": "port", "seconds": omp_s},
            }
    if not args.no_mg:
        mg = mg_section(npbcg, device, rank, world, dist)
        if line is not None:
            line["mg"] = mg
        ep = ep_section(npbcg, device, rank)
        if line is not None:
            line["ep"] = ep
        is_ = is_section(npbcg, device, rank)
        if line is not None:
            line["is"] = is_
        ft = ft_section(npbcg, device, rank)
        if line is not None:
            line["ft"] = ft
    if not args.no_partitioned:
        part = row_partitioned_section(npbcg, device, rank, world, dist)
        if line is not None:
            line["row_partitioned"] = part
    if not args.no_batched:
        # every rank solves its shard of the batched workload; rank 0 gathers
        batched = batched_section(npbcg, device, rank=rank, world=world, dist=dist)
        if line is not None:
            line["batched"] = batched
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    sess.close()
    for p in (p_rs, p_ci, p_a):
        lib.cgb_host_free(p)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def main():
    global CLASSES
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solver-modes", action="store_true",
                    help="skip the class C comparison of the solver modes")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-mg", action="store_true", help="skip the NPB MG, EP, IS and FT class C sections")
    ap.add_argument("--no-partitioned", action="store_true",
                    help="skip class D split by rows over the ranks")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    import npbcg
    CLASSES = npbcg.CLASSES
    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    return our_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
