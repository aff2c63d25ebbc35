"""Benchmark: time to relative residual 1e-10, mixed-precision V-cycle against
the FP64 GPU V-cycle, and the V-cycle apply's HBM bandwidth.

Headline workload (the precision form): anisotropic convection-diffusion
-(u_xx + u_yy + 0.01 u_zz) + (1/sqrt3)(u_x+u_y+u_z) = f on the unit cube,
7-point FD, h = 1/(idim+1), idim = 160 (4,096,000 rows, 28,518,400 nnz),
b uniform[-1,1] (numpy default_rng(0)), x0 = 0.  MLD2P4 'ML' preconditioner:
decoupled smoothed aggregation (threshold 0.01, omega = 4/(3 ||D^-1 A||_inf)),
coarsening to <= 2000 rows, V-cycle with 2 pre + 2 post sweeps of point
Jacobi (damping 0.8), coarsest level 4 sweeps of block-Jacobi ILU(0).  The
hierarchy values and the whole V-cycle run in FP32 inside FP64 flexible CG
(FP64 residual, dot products and norms), stopping on ||b - Ax||/||b|| <= 1e-10.
One step = one full solve.  The same solve with the FP64 V-cycle is timed in
the same run (key `fp64_vcycle`), and so are the plain FP64 drop-in forms of
the isotropic idim=160 problem (key `isotropic_fp64`), the batching forms
and, on one GPU, the FP64 CPU oracle solution the final errors refer to.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N GPUs: every rank solves its own copy of the headline system (replicas,
weak scaling, no data-path collective); the batching forms' independent
units (64 systems, 32 right-hand sides) are dealt to the ranks.  value =
solves/s over the whole job, device-timed with CUDA events, max over ranks.
The reference arm times the CPU restatement of the reference's algorithm (the
oracle, FP64: the reference has no other precision) on the host cores and
never loads the product library.
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
HEADLINE_SMOOTHER = "JACOBI"  # 2 sweeps, damping 0.8 (the point-Jacobi form of the drop-in)


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


def load_dist():
    """The multi-rank helpers (pure Python; loads no native code)."""
    name = "mld2p4_2_b200_dist"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "mld2p4-2_b200", "dist.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # CPU baseline / reference arm only
    return oracle


def profiled_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` (and the capture it comes from) from the
    committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            k = json.load(f)["kernels"].get(kernel)
        if k:
            t = k["traffic_bytes_per_launch"]
            return sum(t) / len(t), k.get("source")
    except Exception:
        pass
    return None, None


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
        self.lines = []

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


def headline_rhs(n):
    return np.random.default_rng(0).uniform(-1.0, 1.0, n)


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


def oracle_prec(orc, ao, smoother):
    """The oracle preconditioner with the settings of make_prec (FP64)."""
    sm = {"BJAC": orc.BJAC, "JACOBI": orc.JACOBI, "FBGS": orc.FBGS}[smoother]
    jac = smoother == "JACOBI"
    par = orc.default_params(smoother=sm, sweeps_pre=2 if jac else 1, sweeps_post=2 if jac else 1,
                             jac_damp=0.8 if jac else 1.0, coarse_solver=orc.BJAC, coarse_sweeps=4,
                             min_coarse_size=2000)
    op = orc.Prec(par)
    op.build(ao)
    return op


# the V-cycle precision forms (PRECISION keyword of the host mirror)
FORM_TEXT = {"FP64": "FP64", "FP32": "FP32",
             "FP32_P16": "FP32 with FP16 prolongator values (FP32 row scales)",
             "FP32_H16": "FP32 arithmetic on FP16 operator values (FP32 row scales for A, P, R, ND)",
             "FP64_REFERENCE": "FP64, the reference's only form, on the host cores"}


def workload_config(args, world, a=None, p=None, precision=None):
    pr = precision or args.precision
    c = {"workload": f"pdegen 3D anisotropic convection-diffusion (0.01 u_zz) idim={args.idim}, "
                     f"b uniform[-1,1] seed 0, ML V-cycle point-Jacobi 2+2 sweeps (damping 0.8) in "
                     f"{FORM_TEXT[pr]}, FP64 FCG to {args.eps:g}",
         "idim": args.idim, "rows": args.idim ** 3, "smoother": HEADLINE_SMOOTHER,
         "precision": pr, "outer": "FP64 FCG (istop 2)",
         "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
         "l2": "inputs larger than L2 (hierarchy ~1.6 GB resident in HBM)"}
    if a is not None:
        c["nnz"] = a.nnz
    if p is not None:
        c["levels"] = [p.level_info(l)["n"] for l in range(p.nlev)]
    return c


# ---------------------------------------------------------------------------
# reference arm: the oracle (C restatement of the reference algorithm), FP64

def run_reference(args, rank, world):
    """Rank 0 alone times the CPU reference on the headline workload; other
    ranks exit without work.  Each step is a bounded sample: the first
    `sample_its` FCG iterations of the solve, scaled to the solve's full
    iteration count (measured once, untimed)."""
    if rank != 0:
        return
    orc = load_oracle()
    ao = orc.gen_pde3d(args.idim, 1, ANISO)
    b = headline_rhs(ao.nrows)
    t0 = time.perf_counter()
    op = oracle_prec(orc, ao, HEADLINE_SMOOTHER)
    t_build = time.perf_counter() - t0
    _, its_full, rr_full, _ = orc.krylov("FCG", ao, op, b, eps=args.eps, itmax=1000)
    k = max(1, min(args.sample_its, its_full))
    for _ in range(args.warmup):
        orc.krylov("FCG", ao, op, b, eps=args.eps, itmax=k)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.krylov("FCG", ao, op, b, eps=args.eps, itmax=k)
    dt = time.perf_counter() - t0
    s_per_solve = dt / args.steps / k * its_full
    value = 1.0 / s_per_solve
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * s_per_solve, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, world, precision="FP64_REFERENCE"),
        "iterations": its_full, "final_relres": rr_full, "hierarchy_build_s": t_build,
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": orc.num_threads(),
                         "kind": "port",
                         "sample": f"each step: the first {k} FCG iterations of the idim={args.idim} "
                                   f"anisotropic solve, scaled to its {its_full} iterations; SpMVs, "
                                   f"vector updates and dot products on {orc.num_threads()} OpenMP "
                                   f"threads"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm

def time_solves(mld, a, p, bd, x, args, torch, dist=None, dev=0, profile_range=False):
    """W untimed, then K timed FCG solves (device events of the library);
    returns total ms (max over ranks), launches, iterations, relres.
    profile_range: bracket the timed solves with cudaProfilerStart/Stop, so
    that a profiler started with its capture off (ncu --profile-from-start
    off) sees exactly the headline's timed launches."""
    def solve():
        x.zero_()
        _, it, rr = mld.krylov("FCG", a, p, bd, x, eps=args.eps, itmax=1000, use_prec_matrix=True)
        ms, nl = p.last_timing()
        return it, rr, ms, nl

    for _ in range(args.warmup):
        solve()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    tot, launches, its, rr = 0.0, 0, [], None
    if profile_range:
        torch.cuda.profiler.start()
    for _ in range(args.steps):
        it, rr, ms, nl = solve()
        tot += ms
        launches += nl
        its.append(it)
    torch.cuda.synchronize()
    if profile_range:
        torch.cuda.profiler.stop()
    if dist is not None:
        tot = load_dist().max_over_ranks(tot, device=f"cuda:{dev}")
    return {"tot_ms": tot, "launches": launches, "iters": its[-1], "relres": rr}


def apply_stats(p, bd, y, reps=5):
    ap = []
    for _ in range(reps):
        p.apply(bd, y)
        ap.append(p.last_timing()[0])
    return min(ap), p.apply_bytes(), p.apply_impl_bytes()


def dominant_kernel(p, mld, bd, y, reps):
    """The (kind, level) group with the largest device time in one profiled
    V-cycle, then the average device time of its first launch over `reps`
    graph-replayed applies (CUDA events placed in the captured graph)."""
    prof = p.profile("N")
    groups = {}
    for e in prof:
        g = groups.setdefault((e["kind_id"], e["level"]), [0.0, 0, 0])
        g[0] += e["ms"]
        g[1] += 1
        g[2] += e["bytes"]
    (dk, dl), (dms, _, _) = max(groups.items(), key=lambda kv: kv[1][0])
    share = dms / sum(e["ms"] for e in prof)
    p.probe_set(dk, dl, 0)
    p.apply(bd, y)  # capture with the probe
    p.probe_read()
    for _ in range(reps):
        p.apply(bd, y)
    ms, cnt, nbytes = p.probe_read()
    p.probe_set(0, 0, 0)
    return {"kernel": f"{mld.KERNEL_NAMES[dk]} level {dl}", "ms": ms, "count": cnt, "bytes": nbytes,
            "share_of_vcycle": share}


def form_summary(r, apply_ms, abytes, ibytes, peak, world, steps, label):
    return {"form": label, "time_to_1e-10_ms": r["tot_ms"] / steps,
            "solves_per_s": world * steps / (r["tot_ms"] * 1e-3),
            "iterations": r["iters"], "final_relres": r["relres"], "apply_ms": apply_ms,
            "apply_algorithmic_bytes": abytes, "apply_implementation_bytes": ibytes,
            "apply_gbs": abytes / (apply_ms * 1e-3) / 1e9,
            "apply_frac_of_peak": abytes / (apply_ms * 1e-3) / 1e9 / peak}


def isotropic_forms(mld, args, dev, torch, peak, world, dist):
    """The plain FP64 drop-in at idim=160 (isotropic, b = A*1): block-Jacobi
    ILU(0) and point Jacobi V-cycles, FCG to 1e-10."""
    a = mld.gen_pde3d(args.idim, 1, ISO)
    b = a.matvec(np.ones(a.nrows))
    bd = torch.tensor(b, dtype=torch.float64, device=f"cuda:{dev}")
    x = torch.zeros_like(bd)
    out = {"form": f"isotropic idim={args.idim}, b = A*1, FP64 V-cycle, FCG to {args.eps:g}"}
    for sm in ("BJAC", "JACOBI"):
        p = make_prec(mld, a, sm, "FP64", device=dev)
        r = time_solves(mld, a, p, bd, x, args, torch, dist, dev)
        ap, ab, ib = apply_stats(p, bd, x)
        s = form_summary(r, ap, ab, ib, peak, world, args.steps, f"{sm} smoother, FP64 V-cycle")
        s["max_abs_err_vs_ones"] = float(torch.max(torch.abs(x - 1.0)))
        if sm == "BJAC":
            s["dominant_kernel"] = dominant_kernel(p, mld, bd, torch.zeros_like(bd), 10)
        out[sm.lower()] = s
        p.free()
    return out


def time_systems(mld, args, dev, torch, rank, world, nsys=64, lo=24, hi=96):
    """Batching form (b): nsys independent systems, idim uniform in lo..hi
    (seed 1), each with its own hierarchy (FP32 V-cycle, FP64 FCG), dealt to
    the ranks by size and solved together on each rank (mldg_krylov_batch),
    against solving a rank's systems one after the other."""
    md = load_dist()
    dims = [int(v) for v in np.random.default_rng(1).integers(lo, hi + 1, nsys)]
    mine = md.deal_balanced([d ** 3 for d in dims], world)[rank]
    precs, bs, mats, rows = [], [], [], 0
    # throughput setting: the small levels keep their triangular solves, which
    # overlap across the concurrent systems, instead of the explicit inverses
    # (bandwidth-bound products that a single system runs faster alone) or
    # the 16-SM cluster solves (which hold SMs the other systems would use)
    saved = {k: os.environ.get(k) for k in ("MLDG_NO_DENSE_INV", "MLDG_NO_REP")}
    os.environ.update({"MLDG_NO_DENSE_INV": "1", "MLDG_NO_REP": "1"})
    try:
        for i in mine:
            a = mld.gen_pde3d(dims[i], 1, ISO)
            mats.append(a)
            precs.append(make_prec(mld, a, "BJAC", "FP32", device=dev))
            bs.append(torch.tensor(a.matvec(np.ones(a.nrows)), dtype=torch.float64, device=f"cuda:{dev}"))
            rows += a.nrows
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
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
    seq, its1 = 0.0, []
    for a, p, b, x in zip(mats, precs, bs, xs):
        x.zero_()
        _, it, _ = mld.krylov("FCG", a, p, b, x, eps=args.eps, itmax=500, use_prec_matrix=True)
        seq += p.last_timing()[0]
        its1.append(it)
    for p in precs:
        p.free()
    bms = md.max_over_ranks(statistics.median(ms), device=f"cuda:{dev}")
    seq = md.max_over_ranks(seq, device=f"cuda:{dev}")
    merged = md.merge_results(mine, list(zip([int(v) for v in its], [float(v) for v in rel])), nsys)
    rows = int(md.sum_over_ranks(rows, device=f"cuda:{dev}"))
    err = md.max_over_ranks(err, device=f"cuda:{dev}")
    its_all = [m[0] for m in merged]
    return {"form": f"{nsys} independent systems, idim uniform {lo}..{hi} (seed 1), own hierarchies, "
                    f"FP32 V-cycle, FP64 FCG to {args.eps:g}, b = A*1, dealt to {world} rank(s) by size",
            "rows_total": rows, "idim_min": min(dims), "idim_max": max(dims),
            "batched_ms": bms, "batched_systems_per_s": nsys / (bms * 1e-3),
            "sequential_ms": seq, "speedup": seq / bms,
            "iterations_batched": [min(its_all), max(its_all)],
            "iterations_single": [min(its1), max(its1)] if its1 else None,
            "max_relres": max(m[1] for m in merged), "max_abs_err_vs_ones": err}


def time_rhs(mld, args, dev, torch, rank, world, nrhs=32, idim=128):
    """Batching form (a): nrhs right-hand sides (uniform[-1,1], seed 4), a
    contiguous block of columns per rank, advanced together through one
    multi-vector V-cycle per FCG iteration (mldg_krylov_multi; FP32 V-cycle,
    FP64 FCG), against the same columns as single-vector solves."""
    md = load_dist()
    a = mld.gen_pde3d(idim, 1, ISO)
    p = make_prec(mld, a, "BJAC", "FP32", device=dev)
    n = a.nrows
    B = np.random.default_rng(4).uniform(-1.0, 1.0, (nrhs, n))
    lo, hi = md.column_block(nrhs, rank, world)
    Bd = torch.tensor(B[lo:hi], dtype=torch.float64, device=f"cuda:{dev}")
    Xd = torch.zeros_like(Bd)
    p.krylov_multi("FCG", Bd, Xd, eps=args.eps, itmax=500)  # warm (captures the graphs)
    reps = max(1, min(args.steps, 3))
    ms = []
    for _ in range(reps):
        Xd.zero_()
        _, its, rel = p.krylov_multi("FCG", Bd, Xd, eps=args.eps, itmax=500)
        ms.append(p.last_timing()[0])
    single, its1 = 0.0, []
    x = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")
    for c in range(hi - lo):
        x.zero_()
        _, it, _ = mld.krylov("FCG", a, p, Bd[c].contiguous(), x, eps=args.eps, itmax=500,
                              use_prec_matrix=True)
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
    p.free()
    bms = md.max_over_ranks(statistics.median(ms), device=f"cuda:{dev}")
    single = md.max_over_ranks(single, device=f"cuda:{dev}")
    merged = md.merge_results(list(range(lo, hi)), list(zip([int(v) for v in its], [float(v) for v in rel])),
                              nrhs)
    its_all = [m[0] for m in merged]
    return {"form": f"{nrhs} right-hand sides, idim={idim}, BJAC FP32 V-cycle, FP64 FCG to {args.eps:g}, "
                    f"column blocks on {world} rank(s)",
            "rows": n, "batched_ms": bms, "batched_solves_per_s": nrhs / (bms * 1e-3),
            "sequential_ms": single, "speedup": single / bms,
            "iterations_batched": [min(its_all), max(its_all)],
            "iterations_single": [min(its1), max(its1)] if its1 else None,
            "max_relres": max(m[1] for m in merged),
            "block_apply_ms": min(ap), "single_apply_ms": min(ap1),
            "apply_per_rhs_speedup": min(ap1) * (hi - lo) / min(ap)}


def run_ours(args, rank, world, local_rank):
    import torch
    mld = load_package()
    dev = local_rank
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_
    peak, peak_kind = peaks()
    a = mld.gen_pde3d(args.idim, 1, ANISO)
    n = a.nrows
    b = headline_rhs(n)
    bd = torch.tensor(b, dtype=torch.float64, device=f"cuda:{dev}")
    x = torch.zeros_like(bd)
    y = torch.zeros_like(bd)
    forms = {}
    with Clocks(dev) as clk:
        # the headline form, then the FP64 V-cycle it is compared with
        order = [args.precision] + [f for f in ("FP64", "FP32", "FP32_P16", "FP32_H16")
                                    if f != args.precision and not (args.no_variants and f != "FP64")]
        sols = {}
        for pr in order:
            p = make_prec(mld, a, HEADLINE_SMOOTHER, pr, device=dev)
            r = time_solves(mld, a, p, bd, x, args, torch, dist, dev, profile_range=pr == args.precision)
            sols[pr] = x.cpu().numpy()
            ap, ab, ib = apply_stats(p, bd, y)
            forms[pr] = {"r": r, "apply": (ap, ab, ib)}
            if pr == args.precision:
                main_p = p
                forms[pr]["dom"] = dominant_kernel(p, mld, bd, y, 20)
                forms[pr]["levels"] = [p.level_info(l)["n"] for l in range(p.nlev)]
            else:
                p.free()
        iso = None
        if not args.no_variants:
            iso = isotropic_forms(mld, args, dev, torch, peak, world, dist)
        batch = None
        if not args.no_batch:
            batch = {"rhs32_idim128": time_rhs(mld, args, dev, torch, rank, world),
                     "systems64_idim24_96": time_systems(mld, args, dev, torch, rank, world)}
    # end-to-end through the public API with host buffers (pinned): the H2D
    # copies of b and x0 and the D2H copy of x are inside the timed region
    bh = torch.empty(n, dtype=torch.float64, pin_memory=True)
    bh.copy_(torch.from_numpy(b))
    xh = torch.zeros(n, dtype=torch.float64, pin_memory=True)
    e2e_ms = 0.0
    for _ in range(args.steps):
        xh.zero_()
        mld.krylov("FCG", a, main_p, bh, xh, eps=args.eps, itmax=1000, use_prec_matrix=True)
        e2e_ms += main_p.last_timing()[0]
    if dist is not None:
        e2e_ms = load_dist().max_over_ranks(e2e_ms, device=f"cuda:{dev}")
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        orc = load_oracle()
        ao = orc.CSR(a.irp, a.ja, a.val)
        op = oracle_prec(orc, ao, HEADLINE_SMOOTHER)
        t0 = time.perf_counter()
        xr, it_c, rr_c, _ = orc.krylov("FCG", ao, op, b, eps=args.eps, itmax=1000)
        dt = time.perf_counter() - t0
        cpu = {"value": 1.0 / dt, "unit": "solves/s", "cores": orc.num_threads(), "kind": "port",
               "sample": f"1 full FCG solve to {args.eps:g} ({it_c} iterations) of the idim={args.idim} "
                         f"anisotropic system, FP64 V-cycle (oracle, C restatement); SpMVs, vector "
                         f"updates and dot products on {orc.num_threads()} OpenMP threads"}
        for pr in sols:
            forms[pr]["err_vs_cpu"] = float(np.linalg.norm(sols[pr] - xr) / np.linalg.norm(xr))
    if rank != 0:
        return
    main = forms[args.precision]
    r = main["r"]
    dom = main["dom"]
    achieved = dom["bytes"] * dom["count"] / (dom["ms"] * 1e-3) / 1e9 if dom["ms"] > 0 else None
    traffic, traffic_src = profiled_traffic(dom["kernel"] + f" {args.precision}")

    def summary(pr):
        f = forms[pr]
        s = form_summary(f["r"], *f["apply"], peak, world, args.steps,
                         f"point-Jacobi V-cycle in {FORM_TEXT[pr]}, FP64 FCG")
        if "err_vs_cpu" in f:
            s["rel_error_vs_cpu_fp64"] = f["err_vs_cpu"]
        return s

    f64 = forms["FP64"]["r"]
    line = {
        "metric": METRIC, "value": world * args.steps / (r["tot_ms"] * 1e-3), "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["tot_ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"FP64": "f64", "FP32": "f32 V-cycle / f64 FCG", "FP32_P16": "f32 V-cycle (f16 P) / f64 FCG",
                  "FP32_H16": "f32 V-cycle on f16 operator values / f64 FCG"}[args.precision],
        "data": "synthetic (seeded generator, no dataset)",
        "config": workload_config(args, world, a) | {"levels": main["levels"]},
        "iterations": r["iters"], "time_to_1e-10_ms": r["tot_ms"] / args.steps,
        "final_relres": r["relres"],
        "fp64_vcycle": {"time_to_1e-10_ms": f64["tot_ms"] / args.steps, "iterations": f64["iters"],
                        "speedup_of_headline": f64["tot_ms"] / r["tot_ms"],
                        "extra_iterations_of_headline": r["iters"] - f64["iters"]},
        "forms": {pr.lower(): summary(pr) for pr in forms},
        "apply_ms": main["apply"][0], "apply_algorithmic_bytes": main["apply"][1],
        "apply_gbs": main["apply"][1] / (main["apply"][0] * 1e-3) / 1e9,
        "roofline": {"bound": "hbm", "kernel": dom["kernel"], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak if achieved else None,
                     "traffic": traffic, "traffic_source": traffic_src,
                     "peak_source": peak_kind, "bytes_per_launch": dom["bytes"],
                     "avg_launch_ms": dom["ms"] / dom["count"] if dom["count"] else None,
                     "launches_timed": dom["count"], "share_of_vcycle": dom["share_of_vcycle"]},
        "isotropic_fp64": iso,
        "batching": batch,
        "e2e": {"value": world * args.steps / (e2e_ms * 1e-3), "unit": "solves/s",
                "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 8 * n},
        "gpu_launches": r["launches"],
        "clocks": clk.summary(),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--idim", type=int, default=160)
    ap.add_argument("--precision", default="FP32_H16", choices=["FP64", "FP32", "FP32_P16", "FP32_H16"])
    ap.add_argument("--eps", type=float, default=1e-10)
    ap.add_argument("--sample-its", type=int, default=8,
                    help="reference arm: FCG iterations timed per step (scaled to the full solve)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true",
                    help="time only the headline form and the FP64 V-cycle")
    ap.add_argument("--no-batch", action="store_true", help="skip the batching forms")
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
