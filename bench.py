"""Benchmark: FCG to relative residual 1e-10 with the GPU V-cycle preconditioner.

Workload (the plain FP64 drop-in at scale): -Lap u + (1/sqrt3)(u_x+u_y+u_z)
on the unit cube, 7-point FD, h = 1/(idim+1), idim = 160 (4,096,000 rows,
28,518,400 nnz), b = A*1, x0 = 0.  MLD2P4 'ML' preconditioner: decoupled
smoothed aggregation (threshold 0.01, omega = 4/(3 ||D^-1 A||_inf)),
coarsening to <= 2000 rows, V-cycle with 1 pre + 1 post sweep of
block-Jacobi ILU(0) (or point Jacobi, --smoother JACOBI: 2 sweeps, damping
0.8), coarsest level 4 sweeps of block-Jacobi ILU(0).  One step = one full
FCG solve to 1e-10 (istop 2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Each rank solves its own copy of the system (weak scaling: N independent
solves, no data-path collective).  value = solves/s over the whole job,
device-timed with CUDA events (max over ranks).  The reference arm times the
CPU restatement of the reference's algorithm (the oracle) on the host cores.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

# independent systems run on their own streams: give them separate hardware queues
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "time-to-1e-10 residual (mixed vs FP64 GPU V-cycle); V-cycle apply HBM GB/s"
S3 = 1.0 / np.sqrt(3.0)
ISO = (1.0, 1.0, 1.0, S3, S3, S3, 0.0)
ANISO = (1.0, 1.0, 0.01, S3, S3, S3, 0.0)


def load_package():
    name = "mld2p4_2_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = os.path.join(ROOT, "mld2p4-2_b200")
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # CPU baseline / reference arm only
    return oracle


def profiled_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            k = json.load(f)["kernels"].get(kernel)
        if k:
            t = k["traffic_bytes_per_launch"]
            return sum(t) / len(t)
    except Exception:
        pass
    return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler run during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p is not None:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


def build_problem(mld, idim):
    a = mld.gen_pde3d(idim, 1, ISO)
    b = a.matvec(np.ones(a.nrows))
    return a, b


def make_prec(mld, a, smoother, precision="FP64", device=0):
    p = mld.MldPrec(device=device)
    p.init("ML")
    p.set("SMOOTHER_TYPE", smoother)
    if smoother == "JACOBI":
        p.set("SMOOTHER_SWEEPS", 2)
        p.set("SMOOTHER_DAMPING", 0.8)
    elif smoother == "BJAC":
        p.set("SUB_SOLVE", "ILU")
        p.set("SMOOTHER_SWEEPS", 1)
    p.set("COARSE_SOLVE", "BJAC")
    p.set("COARSE_SUBSOLVE", "ILU")
    p.set("COARSE_SWEEPS", 4)
    p.set("MIN_COARSE_SIZE", 2000)
    p.set("AGGR_THRESH", 0.01)
    p.set("PRECISION", precision)
    p.build(a)
    return p


def cpu_solve_oracle(orc, a, smoother, eps):
    sm = orc.BJAC if smoother == "BJAC" else orc.JACOBI
    par = orc.default_params(smoother=sm, sweeps_pre=2 if smoother == "JACOBI" else 1,
                             sweeps_post=2 if smoother == "JACOBI" else 1,
                             jac_damp=0.8 if smoother == "JACOBI" else 1.0,
                             coarse_solver=orc.BJAC, coarse_sweeps=4, min_coarse_size=2000)
    ao = orc.CSR(a.irp, a.ja, a.val)
    op = orc.Prec(par)
    op.build(ao)
    return ao, op


def run_reference(args, rank, world):
    """CPU reference arm: the oracle (restated reference algorithm) on host cores."""
    if rank != 0:
        return
    mld = load_package()
    orc = load_oracle()
    a, b = build_problem(mld, args.idim)
    ao, op = cpu_solve_oracle(orc, a, args.smoother, args.eps)
    for _ in range(args.warmup):
        orc.krylov("FCG", ao, op, b, eps=args.eps, itmax=500)
    t0 = time.perf_counter()
    its = []
    for _ in range(args.steps):
        _, it, rr, _ = orc.krylov("FCG", ao, op, b, eps=args.eps, itmax=500)
        its.append(it)
    dt = time.perf_counter() - t0
    value = args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config(args, a, None),
        "iterations": its[-1] if its else None,
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": orc.num_threads(),
                         "kind": "port",
                         "sample": f"{args.steps} full FCG solve(s) to {args.eps:g}, idim={args.idim}"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config(args, a, p):
    c = {"workload": f"pdegen 3D convection-diffusion idim={args.idim} FP64, "
                     f"ML V-cycle {args.smoother} smoother, FCG to {args.eps:g}",
         "idim": args.idim, "rows": a.nrows, "nnz": a.nnz, "smoother": args.smoother,
         "precision": args.precision, "parallelism": f"replicas x{args.gpus}",
         "l2": "inputs larger than L2 (hierarchy > 1 GB resident in HBM)"}
    if p is not None:
        c["levels"] = [p.level_info(l)["n"] for l in range(p.nlev)]
    return c


def time_variant(mld, a, b, smoother, precision, args, dev, torch, probe=False, dist=None):
    """Build one preconditioner form and time K FCG solves (device events)."""
    p = make_prec(mld, a, smoother, precision, device=dev)
    n = a.nrows
    bd = torch.tensor(b, dtype=torch.float64, device=f"cuda:{dev}")
    x0 = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")
    xs = torch.zeros_like(x0)
    torch.cuda.synchronize()
    p.apply(bd, xs)  # first apply captures the graph
    res = {"p": p, "bd": bd, "xs": xs}
    if probe:
        # dominant kernel: the (kind, level) group with the largest device time
        prof = p.profile("N")
        groups = {}
        for e in prof:
            g = groups.setdefault((e["kind_id"], e["level"]), [0.0, 0, 0])
            g[0] += e["ms"]
            g[1] += 1
            g[2] += e["bytes"]
        (dk, dl), (dms, _, _) = max(groups.items(), key=lambda kv: kv[1][0])
        p.probe_set(dk, dl, 0)
        res.update(dk=dk, dl=dl, share=dms / sum(e["ms"] for e in prof))

    def solve():
        xs.copy_(x0)
        torch.cuda.synchronize()
        _, it, rr = mld.krylov("FCG", a, p, bd, xs, eps=args.eps, itmax=500, use_prec_matrix=True)
        ms, nl = p.last_timing()
        return it, rr, ms, nl

    for _ in range(args.warmup):
        solve()
    p.probe_read()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    tot, launches, its, rr = 0.0, 0, [], None
    for _ in range(args.steps):
        it, rr, ms, nl = solve()
        tot += ms
        launches += nl
        its.append(it)
    torch.cuda.synchronize()
    res["probe"] = p.probe_read()
    if dist is not None:
        from mld2p4_2_b200 import dist as mdist
        tot = mdist.max_over_ranks(tot, device=f"cuda:{dev}")
    ap = []
    for _ in range(5):
        p.apply(bd, xs)
        ap.append(p.last_timing()[0])
    res.update(tot_ms=tot, launches=launches, iters=its[-1], relres=rr,
               apply_ms=min(ap), apply_bytes=p.apply_bytes())
    # solution error of the last timed solve
    xs.copy_(x0)
    torch.cuda.synchronize()
    mld.krylov("FCG", a, p, bd, xs, eps=args.eps, itmax=500, use_prec_matrix=True)
    res["err"] = float(torch.max(torch.abs(xs - 1.0)))
    return res


def time_precision_form(mld, args, dev, torch, idim=160, ref_solution=None):
    """Precision form: anisotropic -(u_xx + u_yy + 0.01 u_zz) + (1/sqrt3) grad u
    at idim=160, b uniform[-1,1] (seed 0); the FP64 V-cycle against the FP32
    V-cycle and the FP32 V-cycle with FP16 prolongator values, each inside the
    FP64 FCG loop to 1e-10, with the point-Jacobi and the FBGS smoothers
    (block-Jacobi ILU(0) FCG stagnates near 1e-3 on this problem, on the CPU
    oracle as on the GPU, and is left out).  ref_solution(a, b) gives the FP64
    CPU solution the final errors are measured against (or None)."""
    a = mld.gen_pde3d(idim, 1, ANISO)
    b = np.random.default_rng(0).uniform(-1.0, 1.0, a.nrows)
    bd = torch.tensor(b, dtype=torch.float64, device=f"cuda:{dev}")
    x = torch.zeros_like(bd)
    xref = ref_solution(a, b) if ref_solution is not None else None
    out = {"form": f"anisotropic idim={idim} (0.01 u_zz), b uniform[-1,1] seed 0, FCG to {args.eps:g}"}
    for sm in ("JACOBI", "FBGS"):
        res = {}
        for pr in ("FP64", "FP32", "FP32_P16"):
            p = make_prec(mld, a, sm, pr, device=dev)
            ms, its = [], None
            for _ in range(1 + max(1, min(args.steps, 3))):  # first solve warms (graph capture)
                x.zero_()
                torch.cuda.synchronize()
                _, its, rr = mld.krylov("FCG", a, p, bd, x, eps=args.eps, itmax=500, use_prec_matrix=True)
                ms.append(p.last_timing()[0])
            t = statistics.median(ms[1:])
            xs = x.cpu().numpy()
            r = {"time_to_1e-10_ms": t, "iterations": its, "final_relres": rr}
            if xref is not None:
                r["rel_error_vs_cpu_fp64"] = float(np.linalg.norm(xs - xref) / np.linalg.norm(xref))
            res[pr.lower()] = r
            p.free()
        f64 = res["fp64"]["time_to_1e-10_ms"]
        for pr in ("fp32", "fp32_p16"):
            res[pr]["speedup_vs_fp64"] = f64 / res[pr]["time_to_1e-10_ms"]
            res[pr]["extra_iterations"] = res[pr]["iterations"] - res["fp64"]["iterations"]
        out[sm.lower()] = res
    return out


def time_systems(mld, args, dev, torch, nsys=64, lo=24, hi=96):
    """Batching form (b): nsys independent systems, idim uniform in lo..hi
    (seed 1), each with its own hierarchy (FP32 V-cycle, FP64 FCG), solved
    together (mldg_krylov_batch) against solving them one after the other."""
    dims = np.random.default_rng(1).integers(lo, hi + 1, nsys)
    precs, bs, mats, rows = [], [], [], 0
    # throughput setting: the small levels keep their triangular solves, which
    # overlap across the concurrent systems, instead of the explicit inverses
    # (bandwidth-bound products that a single system runs faster alone) or
    # the 16-SM cluster solves (which hold SMs the other systems would use)
    prev = os.environ.get("MLDG_NO_DENSE_INV")
    prev_rep = os.environ.get("MLDG_NO_REP")
    os.environ["MLDG_NO_DENSE_INV"] = "1"
    os.environ["MLDG_NO_REP"] = "1"
    for idim in dims:
        a = mld.gen_pde3d(int(idim), 1, ISO)
        mats.append(a)
        precs.append(make_prec(mld, a, "BJAC", "FP32", device=dev))
        bs.append(torch.tensor(a.matvec(np.ones(a.nrows)), dtype=torch.float64, device=f"cuda:{dev}"))
        rows += a.nrows
    if prev is None:
        del os.environ["MLDG_NO_DENSE_INV"]
    else:
        os.environ["MLDG_NO_DENSE_INV"] = prev
    if prev_rep is None:
        del os.environ["MLDG_NO_REP"]
    else:
        os.environ["MLDG_NO_REP"] = prev_rep
    xs = [torch.zeros_like(b) for b in bs]
    mld.krylov_batch("FCG", precs, bs, xs, eps=args.eps, itmax=500)  # warm: captures the graphs
    reps = max(1, min(args.steps, 3))
    ms = []
    for _ in range(reps):
        for x in xs:
            x.zero_()
        _, its, rel, t = mld.krylov_batch("FCG", precs, bs, xs, eps=args.eps, itmax=500)
        ms.append(t)
    err = max(float(torch.max(torch.abs(x - 1.0))) for x in xs)
    seq = 0.0
    its1 = []
    for a, p, b, x in zip(mats, precs, bs, xs):
        x.zero_()
        _, it, _ = mld.krylov("FCG", a, p, b, x, eps=args.eps, itmax=500, use_prec_matrix=True)
        seq += p.last_timing()[0]
        its1.append(it)
    for p in precs:
        p.free()
    bms = statistics.median(ms)
    return {"form": f"{nsys} independent systems, idim uniform {lo}..{hi} (seed 1), own hierarchies, "
                    f"FP32 V-cycle, FP64 FCG to {args.eps:g}, b = A*1",
            "rows_total": rows, "idim_min": int(dims.min()), "idim_max": int(dims.max()),
            "batched_ms": bms, "batched_systems_per_s": nsys / (bms * 1e-3),
            "sequential_ms": seq, "sequential_systems_per_s": nsys / (seq * 1e-3),
            "speedup": seq / bms, "iterations_batched": [int(its.min()), int(its.max())],
            "iterations_single": [min(its1), max(its1)], "max_relres": float(rel.max()),
            "max_abs_err_vs_ones": err}


def time_batch(mld, args, dev, torch, nrhs=32, idim=128):
    """Batching form (a): nrhs right-hand sides (uniform[-1,1], seed 4) through
    one multi-vector V-cycle per FCG iteration (mldg_krylov_multi; FP32 V-cycle,
    FP64 FCG) against nrhs single-vector FCG solves."""
    a = mld.gen_pde3d(idim, 1, ISO)
    p = make_prec(mld, a, "BJAC", "FP32", device=dev)
    n = a.nrows
    B = np.random.default_rng(4).uniform(-1.0, 1.0, (nrhs, n))
    Bd = torch.tensor(B, dtype=torch.float64, device=f"cuda:{dev}")
    Xd = torch.zeros_like(Bd)
    p.krylov_multi("FCG", Bd, Xd, eps=args.eps, itmax=500)  # warm (captures the graphs)
    reps = max(1, min(args.steps, 3))
    ms = []
    for _ in range(reps):
        Xd.zero_()
        _, its, rel = p.krylov_multi("FCG", Bd, Xd, eps=args.eps, itmax=500)
        ms.append(p.last_timing()[0])
    single = 0.0
    its1 = []
    x = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")
    for c in range(nrhs):
        x.zero_()
        _, it, _ = mld.krylov("FCG", a, p, Bd[c], x, eps=args.eps, itmax=500, use_prec_matrix=True)
        single += p.last_timing()[0]
        its1.append(it)
    Y = torch.zeros_like(Bd)
    ap = []
    for _ in range(5):
        p.apply_block(Bd, Y)
        ap.append(p.last_timing()[0])
    ap1 = []
    for _ in range(5):
        p.apply(Bd[0].contiguous(), x)
        ap1.append(p.last_timing()[0])
    bms = statistics.median(ms)
    p.free()
    return {"form": f"{nrhs} right-hand sides, idim={idim}, BJAC FP32 V-cycle, FP64 FCG to {args.eps:g}",
            "rows": n, "batched_ms": bms, "batched_solves_per_s": nrhs / (bms * 1e-3),
            "sequential_ms": single, "sequential_solves_per_s": nrhs / (single * 1e-3),
            "speedup": single / bms, "iterations_batched": [int(its.min()), int(its.max())],
            "iterations_single": [min(its1), max(its1)], "max_relres": float(rel.max()),
            "block_apply_ms": min(ap), "single_apply_ms": min(ap1),
            "apply_per_rhs_speedup": min(ap1) * nrhs / min(ap)}


def run_ours(args, rank, world, local_rank):
    import torch
    mld = load_package()
    dev = local_rank
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_
    a, b = build_problem(mld, args.idim)
    n = a.nrows
    peak, peak_kind = peaks()
    with Clocks(dev) as clk:
        main = time_variant(mld, a, b, args.smoother, args.precision, args, dev, torch, probe=True,
                            dist=dist)
        others = {}
        if not args.no_variants:
            for sm, pr in (("JACOBI", "FP64"), ("BJAC", "FP32"), ("FBGS", "FP64")):
                if (sm, pr) == (args.smoother, args.precision):
                    continue
                r = time_variant(mld, a, b, sm, pr, args, dev, torch, dist=dist)
                others[f"{sm.lower()}_{pr.lower()}"] = r
                r["p"].free()
        precision_form = None
        if not args.no_variants and not args.no_batch:
            ref = None
            if world == 1 and not args.no_cpu_baseline:
                def ref(a, b):
                    # FP64 CPU solution of the oracle (C restatement), the checker
                    orc = load_oracle()
                    ao, op = cpu_solve_oracle(orc, a, "JACOBI", args.eps)
                    xr, _, _, _ = orc.krylov("FCG", ao, op, b, eps=args.eps, itmax=500)
                    return xr
            precision_form = time_precision_form(mld, args, dev, torch, ref_solution=ref)
        batch = None
        if not args.no_variants and not args.no_batch:
            batch = {"rhs32_idim128": time_batch(mld, args, dev, torch),
                     "systems64_idim24_96": time_systems(mld, args, dev, torch)}
    p = main["p"]
    # end-to-end through the public API with host buffers (pinned)
    bh = torch.empty(n, dtype=torch.float64, pin_memory=True)
    bh.copy_(torch.from_numpy(b))
    xh = torch.zeros(n, dtype=torch.float64, pin_memory=True)
    e2e_ms = 0.0
    for s in range(args.steps):
        xh.zero_()
        mld.krylov("FCG", a, p, bh, xh, eps=args.eps, itmax=500, use_prec_matrix=True)
        e2e_ms += p.last_timing()[0]
    if dist is not None:
        from mld2p4_2_b200 import dist as mdist
        e2e_ms = mdist.max_over_ranks(e2e_ms, device=f"cuda:{dev}")
    if rank != 0:
        return
    probe_ms, probe_cnt, probe_bytes = main["probe"]
    achieved = (probe_bytes * probe_cnt) / (probe_ms * 1e-3) / 1e9 if probe_ms > 0 else None
    kname = f"{mld.KERNEL_NAMES[main['dk']]} level {main['dl']}"

    def summary(r, label):
        return {"form": label, "time_to_1e-10_ms": r["tot_ms"] / args.steps,
                "solves_per_s": world * args.steps / (r["tot_ms"] * 1e-3),
                "iterations": r["iters"], "final_relres": r["relres"],
                "max_abs_err_vs_ones": r["err"], "apply_ms": r["apply_ms"],
                "apply_algorithmic_bytes": r["apply_bytes"],
                "apply_gbs": r["apply_bytes"] / (r["apply_ms"] * 1e-3) / 1e9,
                "apply_frac_of_peak": r["apply_bytes"] / (r["apply_ms"] * 1e-3) / 1e9 / peak}

    variants = {f"{args.smoother.lower()}_{args.precision.lower()}":
                summary(main, f"{args.smoother} smoother, {args.precision} V-cycle")}
    for k, r in others.items():
        variants[k] = summary(r, k)
    line = {
        "metric": METRIC, "value": world * args.steps / (main["tot_ms"] * 1e-3), "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": main["tot_ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "FP64" else "f32/f64",
        "data": "synthetic", "config": config(args, a, p),
        "iterations": main["iters"], "time_to_1e-10_ms": main["tot_ms"] / args.steps,
        "final_relres": main["relres"], "max_abs_err_vs_ones": main["err"],
        "apply_ms": main["apply_ms"], "apply_algorithmic_bytes": main["apply_bytes"],
        "apply_gbs": main["apply_bytes"] / (main["apply_ms"] * 1e-3) / 1e9,
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak if achieved else None,
                     "traffic": profiled_traffic(kname)
                     if args.idim == 160 and args.precision == "FP64" else None,
                     "peak_source": peak_kind, "bytes_per_launch": probe_bytes,
                     "avg_launch_ms": probe_ms / probe_cnt if probe_cnt else None,
                     "launches_timed": probe_cnt, "share_of_apply": main["share"]},
        "variants": variants,
        "batching": batch,
        "precision_form": precision_form,
        "e2e": {"value": world * args.steps / (e2e_ms * 1e-3), "unit": "solves/s",
                "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 8 * n},
        "gpu_launches": main["launches"],
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        orc = load_oracle()
        ao, op = cpu_solve_oracle(orc, a, args.smoother, args.eps)
        t0 = time.perf_counter()
        _, it_c, _, _ = orc.krylov("FCG", ao, op, b, eps=args.eps, itmax=500)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "solves/s", "cores": orc.num_threads(),
                                "kind": "port",
                                "sample": f"1 full FCG solve to {args.eps:g} ({it_c} iterations), "
                                          f"idim={args.idim}, {args.smoother} smoother, oracle (C restatement)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--idim", type=int, default=160)
    ap.add_argument("--smoother", default="BJAC", choices=["BJAC", "JACOBI"])
    ap.add_argument("--precision", default="FP64", choices=["FP64", "FP32", "FP32_P16"])
    ap.add_argument("--eps", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true",
                    help="time only the selected smoother/precision form")
    ap.add_argument("--no-batch", action="store_true", help="skip the many-right-hand-sides form")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # rank 0 alone times the CPU reference; other ranks exit without work
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
