"""Benchmark of the neko_b200 pressure/Helmholtz solve path.

Workload (one GPU): the large FP64 pressure-type solve -- periodic box
[0, 2 pi]^3 of 32^3 hexahedra, GLL points displaced by 0.05 sin of the other
two coordinates, lx = 8 (16.8 M local points), h1 = 1, h2 = 0, mean-free
Fourier-mode right-hand side, preconditioned CG from x0 = 0 to a residual
1e-8 times the initial one.  A step is one complete solve.

    python bench.py --gpus N --steps K --warmup W [--impl native|reference]
                    [--pc jacobi|hsmg]

Under torchrun each rank solves its own copy (replicas, weak scaling; the
solve itself does not shard).  `value` is solves/s of the whole job from
device-timed steps (inputs resident in HBM); `e2e` repeats the steps through
the public API with the right-hand side copied in from pinned host memory
and the solution copied back inside the timed region.  `roofline` is the
ax_helm kernel timed with CUDA events on its own stream over the same
problem; `cpu_baseline` times the CPU oracle on a bounded sample.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


# DRAM bytes per point of ax_cg_fused_kernel measured by ncu on a 24^3-element
# case (dram__bytes_read.sum + dram__bytes_write.sum per launch over the
# points; the part of p and w still dirty in L2 when the launch ends is not
# counted).
FUSED_TRAFFIC_B_PER_POINT = {8: 85.4}

# Algorithmic bytes of one gather-scatter add per local entry (a point that
# shares its node with another element): its value read and written, and its
# 4-byte map index.
GS_B_PER_ENTRY = 20


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d, "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 100 ms during the
    timed region (one nvidia-smi process in loop mode)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._p = None
        self._t = None

    def _read(self):
        for line in self._p.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __enter__(self):
        try:
            self._p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)  # first sample before the timed work starts
        except Exception:
            self._p = None
        return self

    def __exit__(self, *a):
        if self._p is not None:
            time.sleep(0.15)
            self._p.terminate()
            try:
                self._p.wait(timeout=10)
            except Exception:
                self._p.kill()
            self._t.join(timeout=10)

    def summary(self):
        sm = []
        mx = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "interval_ms": 100}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def _reduce_device():
    import torch.distributed as dist
    return "cpu" if dist.get_backend() == "gloo" else "cuda"


def max_over_ranks(v, world):
    """Largest value over the ranks (device times: the job ends with the
    slowest rank)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard(items, rank, world):
    """This rank's share of independent work items (replicas: item i goes
    to rank i mod world)."""
    return [it for i, it in enumerate(items) if i % world == rank]


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def build_problem(nb, cfg):
    return nb.Problem(cfg["nel"], cfg["lx"], lo=cfg["lo"], hi=cfg["hi"], periodic=cfg["periodic"],
                      deform=cfg["deform"], dirichlet=cfg["dirichlet"])


def make_rhs(nb, P, seed):
    import torch
    from neko_b200 import workloads
    x, y, z, B = (P.field(k) for k in ("x", "y", "z", "B"))
    b = workloads.periodic_box_rhs(x, y, z, B, seed).contiguous()
    P.gs.op(b, P.n)
    torch.cuda.synchronize()
    return b


def host_threads():
    """Host threads the CPU oracle uses (its element-parallel loops); set
    NB_ORACLE_THREADS to this process's CPU affinity unless given."""
    if "NB_ORACLE_THREADS" not in os.environ:
        try:
            n = len(os.sched_getaffinity(0))
        except AttributeError:
            n = os.cpu_count() or 1
        os.environ["NB_ORACLE_THREADS"] = str(n)
    return int(os.environ["NB_ORACLE_THREADS"])


def oracle_problem(cfg):
    """The CPU oracle's copy of the workload's mesh and geometry."""
    host_threads()
    from oracle import oracle as orc
    O = orc.OracleProblem.box(cfg["nel"], cfg["lx"], lo=cfg["lo"], hi=cfg["hi"],
                              periodic=cfg["periodic"])
    O.deform_sine(cfg["deform"])
    O.coef()
    return O


def oracle_solve(O, b, pc, tol, coarse_tol, max_iter):
    """One complete FP64 solve of the CPU oracle (the port of the
    reference's CPU path, element loops on all host threads) from x0 = 0:
    returns (x, iterations, solve seconds, preconditioner set-up seconds)."""
    from oracle import oracle as orc
    if pc == "hsmg":
        t0 = time.perf_counter()
        H = orc.OracleHsmg(O, coarse_tol=coarse_tol)
        t_setup = time.perf_counter() - t0
        t0 = time.perf_counter()
        x, it, _, _ = H.cg(b, max_iter, tol, flexible=True)
        dt = time.perf_counter() - t0
        H.close()
    elif pc == "phmg":
        t0 = time.perf_counter()
        H = orc.OraclePhmg(O)
        t_setup = time.perf_counter() - t0
        t0 = time.perf_counter()
        x, it, _, _ = H.krylov(b, max_iter, tol, kind="cg")
        dt = time.perf_counter() - t0
        H.close()
    else:
        t_setup = 0.0
        t0 = time.perf_counter()
        x, it, _, _ = O.cg_jacobi(b, max_iter, tol)
        dt = time.perf_counter() - t0
    return x, it, dt, t_setup


def rel_err_mean_free(a, b, singular):
    """Relative L2 distance of a to b; for the singular fully periodic
    problem both are taken mean-free first (its solution is fixed up to a
    constant)."""
    import numpy as np
    if singular:
        a, b = a - a.mean(), b - b.mean()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def workload_name(cfg, solver):
    npts = cfg["nel"][0] * cfg["nel"][1] * cfg["nel"][2] * cfg["lx"] ** 3
    return (f"periodic deformed box {cfg['nel'][0]}^3 hex, lx={cfg['lx']} "
            f"({npts / 1e6:.1f}M points), {solver} to 1e-8 rel")


def run_reference(args, cfg, world, rank):
    """--impl reference: the reference's CPU algorithm (the oracle port; the
    Fortran reference does not build here) on the host, same metric,
    workload, preconditioner and tolerance.  Each timed step is one complete
    solve from x0 = 0 to 1e-8 relative; the --warmup steps are short solves
    (two iterations each) that warm the host threads and caches.  Rank 0
    only."""
    if rank != 0:
        return
    import numpy as np
    from neko_b200 import workloads
    O = oracle_problem(cfg)
    x, y, z, B = O.f64("x"), O.f64("y"), O.f64("z"), O.f64("B")
    b = O.gs_add(workloads.periodic_box_rhs(x, y, z, B, args.seed))
    mult = O.f64("mult")
    r0 = math.sqrt(float(np.sum(b * mult * b)) / O.volume)
    tol = cfg["rel_tol"] * r0
    for _ in range(args.warmup):
        oracle_solve(O, b, args.pc, 0.0, args.coarse_tol, 2)
    times, iters = [], []
    for _ in range(args.steps):
        _, it, dt, _ = oracle_solve(O, b, args.pc, tol, args.coarse_tol, cfg["max_iter"])
        times.append(dt)
        iters.append(it)
    O.close()
    total = sum(times)
    v = args.steps / total
    name = "hsmg-FCG" if args.pc == "hsmg" else "Jacobi-PCG"
    cores = host_threads()
    line = {"impl": "reference", "metric": "Poisson solves/s to 1e-8 rel", "value": v,
            "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(cfg, f"FP64 {name}"), "pc": args.pc,
                       "r0": r0, "iterations": iters[-1], "seed": args.seed},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} complete {name} solves to 1e-8 rel "
                                       f"({iters[-1]} iterations each) on {cores} host threads, "
                                       f"each timed from x0 = 0 (preconditioner set-up "
                                       f"untimed); warm-up: {args.warmup} two-iteration solves"},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def kernel_only(args, cfg):
    """A smaller case of one kernel for profilers: nel^3 elements of the
    periodic-box geometry, `--steps` launches after `--warmup`."""
    import torch
    import neko_b200 as nb
    cfg = dict(cfg, nel=(args.nel,) * 3, lx=args.lx)
    P = build_problem(nb, cfg)
    if args.kernel_only == "solve":
        # --warmup FP64 and mixed hsmg-FCG solves, then one of each inside a
        # profiler window (ncu --profile-from-start off captures only those)
        b = make_rhs(nb, P, args.seed)
        r0 = math.sqrt(float((b * P.field("mult") * b).sum()) / P.volume)
        x = P.zeros()
        solvers = [nb.FCG(max_iter=cfg["max_iter"], abs_tol=cfg["rel_tol"] * r0,
                          M=nb.Hsmg(mixed=m)) for m in (False, True)]
        for _ in range(args.warmup):
            for sv in solvers:
                sv.solve(nb.AxHelm(), x, b, P.n, P)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        mons = [sv.solve(nb.AxHelm(), x, b, P.n, P) for sv in solvers]
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"kernel": "solve", "n": P.n, "iterations": [m.iter for m in mons],
                          "launches": [m.launches for m in mons]}))
        return
    u = torch.rand(P.n, dtype=torch.float64, device="cuda")
    z = torch.rand(P.n, dtype=torch.float64, device="cuda")
    w = P.zeros()
    s = torch.cuda.Stream()

    if args.kernel_only == "stress":
        v3 = [torch.rand(P.n, dtype=torch.float64, device="cuda") for _ in range(3)]
        o3 = [P.zeros() for _ in range(3)]
    if args.kernel_only == "dropin_ax":  # separate dx, dy, dz arrays, as Neko passes them
        import ctypes
        lib = nb.load()
        mats = [P.field("dx").clone() for _ in range(3)] + [P.field("dxt").clone() for _ in range(3)]
        geo = [P.field(k) for k in ("h1", "g11", "g22", "g33", "g12", "g13", "g23")]
        ci = lambda v: ctypes.byref(ctypes.c_int(v))
        vp = lambda t: ctypes.c_void_p(t.data_ptr())
        dstream = ctypes.c_void_p(s.cuda_stream)
    if args.kernel_only in ("dropin_fdm", "dropin_tnsr3d"):
        import ctypes
        lib = nb.load()
        nel, nl = P.nelv, P.lx + 2
        ci = lambda v: ctypes.byref(ctypes.c_int(v))
        vp = lambda t: ctypes.c_void_p(t.data_ptr())
        if args.kernel_only == "dropin_fdm":
            fr = torch.rand(nel * nl ** 3, dtype=torch.float64, device="cuda")
            fe = torch.zeros_like(fr)
            fd = torch.rand_like(fr)
            fs = torch.rand(nel * 6 * nl * nl, dtype=torch.float64, device="cuda")
        else:
            tu = torch.rand(P.n, dtype=torch.float64, device="cuda")
            tv = torch.zeros(nel * 64, dtype=torch.float64, device="cuda")
            tJ = torch.rand(4 * P.lx, dtype=torch.float64, device="cuda")
            tJt = torch.rand(4 * P.lx, dtype=torch.float64, device="cuda")
        dstream = ctypes.c_void_p(s.cuda_stream)

    def launch():
        if args.kernel_only == "ax":
            nb.AxHelm().compute(w, u, P, stream=s)
        elif args.kernel_only == "fused":
            nb.AxHelm().update_p_compute(w, u, z, 0.5, P, stream=s)
        elif args.kernel_only == "stress":
            nb.AxHelmFull().compute_vector(*o3, *v3, P, stream=s)
        elif args.kernel_only == "dropin_ax":
            lib.nb_set_default_stream(dstream)
            lib.cuda_ax_helm(vp(w), vp(u), *(vp(m) for m in mats), *(vp(g) for g in geo),
                             ci(P.nelv), ci(P.lx))
        elif args.kernel_only == "dropin_fdm":
            lib.cuda_fdm_do_fast(vp(fe), vp(fr), vp(fs), vp(fd), ci(nl), ci(nel), dstream)
        elif args.kernel_only == "dropin_tnsr3d":
            with torch.cuda.stream(s):  # cuda_tnsr3d launches on the drop-in default stream
                lib.nb_set_default_stream(dstream)
                lib.cuda_tnsr3d(vp(tv), ci(4), vp(tu), ci(P.lx), vp(tJ), vp(tJt), vp(tJt),
                                ci(nel))
        else:
            P.gs.op(u, P.n, stream=s)
    for _ in range(args.warmup):
        launch()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(args.steps):
        launch()
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    nl = P.lx + 2
    nbytes = {"ax": 72 * P.n, "dropin_ax": 72 * P.n, "fused": 88 * P.n, "stress": 136 * P.n,
              "gs": GS_B_PER_ENTRY * P.nlocal,
              # r read and written, e written, d read, six nl x nl matrices read
              "dropin_fdm": P.nelv * (4 * nl ** 3 + 6 * nl * nl) * 8,
              # u read, v written (lx -> 4 points a side)
              "dropin_tnsr3d": (P.n + P.nelv * 64) * 8}[args.kernel_only]
    peaks, src = measured_peaks()
    gbs = nbytes / ms / 1e6
    print(json.dumps({"kernel": args.kernel_only, "n": P.n, "entries": P.nlocal,
                      "launches": args.warmup + args.steps, "ms_per_launch": ms,
                      "bytes_per_launch": nbytes, "achieved_gbs": gbs,
                      "frac": gbs / peaks["hbm_gbs"], "peak_source": src}))


def run_batch(args):
    """Batched uneven Helmholtz solves: `--batch-count` problems of
    workloads.uneven_specs (Jacobi for boxes of at most 3^3 elements, hsmg
    for the others), to 1e-8 relative, all present at once, served by one
    Batch: the Jacobi problems as slots of the persistent batched engine
    (one Ax launch over every such solve's elements per iteration, graph
    replay, per-lx autotuned k-split), the hsmg problems as per-problem
    flexible-CG solves advanced concurrently on a stream pool by the same run
    loop, in mixed precision (FP32 smoothing, FP64 outer iteration) and in
    FP64; timed against the same solves run one by one on the plain FP64
    path (nb_solve).  An untimed warm-up pass of each builds the problem
    instances, preconditioners, graphs and the autotuner's choice."""
    import torch
    import neko_b200 as nb
    from neko_b200 import serve, workloads
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    # replicas: each GPU serves its share of the independent problems
    specs = shard(workloads.uneven_specs(args.batch_count, seed=args.seed), rank, world)
    cache = serve.GeometryCache()
    pool = serve.RhsPool(cache)
    inst = serve.InstancePool(cache, variants=(False, True))
    for sp in specs:
        pool.get(sp)
    zeros = [0.0] * len(specs)
    stream = torch.cuda.Stream()
    B = nb.Batch()

    def timed_run(fn):
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(e0.elapsed_time(e1) / 1e3, world), time.perf_counter() - t0, out

    res = {}
    for mode in ("mixed", "fp64"):
        run = lambda: serve.serve_batched(specs, zeros, pool, 0, batch=B, mode=mode,
                                          instances=inst, max_solves=args.max_solves,
                                          stream=stream)
        run()  # warm-up: instances, preconditioners, graphs, autotune
        res[mode] = timed_run(run)
    # one by one on the plain FP64 path (preconditioners already built)
    seq = lambda: serve.serve_sequential(specs, zeros, pool, mode="fp64")
    seq()
    t_seq, wall_seq, (lat_s, it_s, conv_s, _) = timed_run(seq)
    xs_seq = None  # the one-by-one solutions of each request
    lat_s2, it_s2, conv_s2, _, xs_seq = serve.serve_batched(specs, zeros, pool, 0, batch=B,
                                                            mode="fp64", instances=inst,
                                                            max_solves=1, stream=stream)
    total = args.batch_count
    out = {}
    for mode, (t, wall, (lat, it, conv, span, xs)) in res.items():
        err = max(float(torch.linalg.norm(xs[i] - xs_seq[i]) / torch.linalg.norm(xs_seq[i]))
                  for i in range(len(specs)))
        out[mode] = {"value": total / t, "seconds": t, "wall_s": wall,
                     "converged": int(sum_over_ranks(sum(1 for c in conv if c), world)),
                     "iterations": {"min": min(it), "max": max(it), "mean": sum(it) / len(it)},
                     "max_iter_diff_vs_sequential": int(max_over_ranks(
                         max(abs(a - b) for a, b in zip(it, it_s)), world)),
                     "max_rel_diff_vs_sequential": max_over_ranks(err, world)}
    ndof = sum_over_ranks(sum(cache.get(sp).n for sp in specs), world)
    n_hsmg = int(sum_over_ranks(sum(1 for sp in specs if sp["pc"] == "hsmg"), world))
    line = {
        "metric": "batched uneven Helmholtz solves/s to 1e-8 rel", "value": out["mixed"]["value"],
        "unit": "solves/s", "n_gpus": world, "higher_is_better": True, "dtype": "f64+f32",
        "data": "synthetic", "vs_baseline": None, "scaling": "strong",
        "parallelism": "replicas x%d" % world,
        "config": {"workload": f"{total} Helmholtz solves, n^3 elements n~U{{2..16}}, "
                               f"N~{{5,7,9}}, h1~U[0.5,2], h2~U[0,100], 8 deformation seeds, "
                               f"zero Dirichlet, Fourier RHS ({ndof / 1e6:.0f}M DOF in total); "
                               f"{n_hsmg} hsmg flexible-CG (mixed precision), "
                               f"{total - n_hsmg} Jacobi-PCG in the persistent batched launch",
                   "max_concurrent_hsmg_solves": args.max_solves,
                   "instances": inst.instances(), "geometries": len(cache.problems),
                   "setup_s": cache.setup_s + inst.setup_s},
        "mixed": out["mixed"], "fp64_batched": out["fp64"],
        "sequential": {"value": total / t_seq, "seconds": t_seq, "wall_s": wall_seq,
                       "path": "nb_solve one by one on the plain FP64 path (hsmg flexible CG or "
                               "Jacobi-PCG per problem, constant coefficients set per solve)"},
        "speedup_vs_sequential": t_seq / res["mixed"][0],
        "fp64_speedup_vs_sequential": t_seq / res["fp64"][0],
        "autotune": {str(lx): {"ks": B.tuning(lx)[0], "candidate_ms": B.tuning(lx)[1]}
                     for lx in (6, 8, 10) if B.tuning(lx)[0]},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    B.close()
    inst.close()
    cache.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_velocity(args):
    """The velocity solve of a time step with variable viscosity on the
    periodic 32^3 box (periodic deformed box 32^3 hex, lx 8, three components of
    16.8 M points): coupled Jacobi-CG (cg_cpld) with the full-stress
    operator, h1 = 1 + 0.5 sin x sin y sin z (the viscosity field), h2 = 10
    (the BDF mass term), each component's right-hand side B f_c assembled,
    to 1e-8 relative; solves/s timed on the device, and the full-stress
    operator timed alone with events (152 algorithmic bytes a point: u, v,
    w, h1, 1/jac, nine cofactors, h2 and B read, three outputs written)."""
    import numpy as np
    import torch
    import neko_b200 as nb
    from neko_b200 import workloads
    torch.cuda.set_device(0)
    cfg = dict(workloads.PERIODIC_BOX_32)
    cfg["lx"] = args.lx
    P = build_problem(nb, cfg)
    x, y, z, B = (P.field(k) for k in ("x", "y", "z", "B"))
    h1 = 1.0 + 0.5 * torch.sin(x) * torch.sin(y) * torch.sin(z)
    P.set_coefficients(h1.contiguous(), torch.full_like(h1, 10.0))
    f = []
    for c in range(3):
        fc = (B * torch.sin(x + c) * torch.cos(2 * y - c) * torch.sin(3 * z + 0.5 * c)).contiguous()
        P.gs.op(fc, P.n)
        f.append(fc)
    mult = P.field("mult")
    r0 = math.sqrt(sum(float((fc * mult * fc).sum()) for fc in f) / P.volume)
    tol = cfg["rel_tol"] * r0
    xs = [P.zeros() for _ in range(3)]
    solver = nb.CoupledCG(max_iter=2000, abs_tol=tol, M=nb.Jacobi())
    Ax = nb.AxHelmFull()
    s = torch.cuda.Stream()
    mons = None
    for _ in range(args.warmup):
        mons = solver.solve_coupled(Ax, *xs, *f, P.n, P, stream=s)
    out = [P.zeros() for _ in range(3)]
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(args.steps):
            mons = solver.solve_coupled(Ax, *xs, *f, P.n, P, stream=s)
        e1.record(s)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        # the operator alone (its inputs, 15 arrays of 134 MB, exceed L2)
        for _ in range(5):
            Ax.compute_vector(*out, *xs, P, stream=s)
        reps = args.ax_reps
        torch.cuda.synchronize()
        e0.record(s)
        for _ in range(reps):
            Ax.compute_vector(*out, *xs, P, stream=s)
        e1.record(s)
        torch.cuda.synchronize()
    t_op = e0.elapsed_time(e1) / 1e3 / reps
    peaks, src = measured_peaks()
    nbytes = (136 + 16) * P.n  # + h2 and B: the h2 B term is folded into the same pass
    gbs = nbytes / t_op / 1e9
    line = {
        "metric": "velocity solves/s to 1e-8 rel (coupled CG, full-stress operator)",
        "value": args.steps / t, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic", "vs_baseline": None,
        "config": {"workload": workload_name(cfg, "coupled Jacobi-CG, full-stress operator, "
                                             "h1 = 1 + 0.5 sin x sin y sin z, h2 = 10")
                   + ", three components", "iterations": mons[0].iter,
                   "converged": mons[0].converged, "r0": r0},
        "roofline": {"bound": "hbm", "kernel": f"ax_stress_tma_kernel<{cfg['lx']}> "
                     "(nb_ax_stress, three components)", "achieved": gbs,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": gbs / peaks["hbm_gbs"],
                     "peak_source": src, "bytes_per_launch": nbytes, "launch_ms": t_op * 1e3,
                     "traffic": None},
        "gpu_launches": mons[0].launches * args.steps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    P.close()


def run_axgs(args):
    """Unit box 8^3, lx = 8, zero Dirichlet.  (a) ax_helm followed
    by gs add on a continuous u ~ U[-1,1] (h1 = 1, h2 = 0), 100 times,
    GDOF/s; (b) the Jacobi-PCG solve of the sin^3 + noise right-hand side to
    1e-10 relative, solves/s."""
    import torch
    import neko_b200 as nb
    from neko_b200 import workloads
    torch.cuda.set_device(0)
    c = workloads.UNIT_BOX_8
    P = nb.Problem(c["nel"], c["lx"], lo=c["lo"], hi=c["hi"], periodic=c["periodic"],
                   deform=c["deform"], dirichlet=c["dirichlet"])
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    u = torch.rand(P.n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    P.gs.op(u)
    u *= P.field("mult")
    w = P.zeros()
    Ax = nb.AxHelm()
    s = torch.cuda.Stream()
    reps = 100
    for _ in range(args.warmup):
        Ax.compute(w, u, P, stream=s)
        P.gs.op(w, stream=s)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        Ax.compute(w, u, P, stream=s)
        P.gs.op(w, stream=s)
    e1.record(s)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    x, y, z = (P.field(k) for k in ("x", "y", "z"))
    xi = torch.randn(P.n, dtype=torch.float64, device="cuda", generator=g) * 1e-3
    P.gs.op(xi)
    xi *= P.field("mult")
    f = workloads.unit_box_pointwise(x, y, z, xi) * P.field("B")
    P.gs.op(f)
    P.bclst.apply(f)
    r0 = math.sqrt(float((f * P.field("mult") * f).sum()) / P.volume)
    solver = nb.CG(max_iter=c["max_iter"], abs_tol=c["rel_tol"] * r0, M=nb.Jacobi())
    xs = P.zeros()
    for _ in range(args.warmup):
        mon = solver.solve(Ax, xs, f, P.n, P, stream=s)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(args.steps):
        mon = solver.solve(Ax, xs, f, P.n, P, stream=s)
    e1.record(s)
    torch.cuda.synchronize()
    ts = e0.elapsed_time(e1) / 1e3 / args.steps
    err = float((xs - torch.sin(math.pi * x) * torch.sin(math.pi * y) *
                 torch.sin(math.pi * z)).abs().max())
    print(json.dumps({
        "metric": "ax_helm + gs add GDOF/s (unit box 8^3, lx 8)", "value": P.n / t / 1e9, "unit": "GDOF/s",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "vs_baseline": None,
        "config": {"workload": "unit box 8^3 hex, lx=8 (262,144 points), zero Dirichlet, "
                               "ax_helm then gs add x100 (working set fits in L2)"},
        "ms_per_apply": t * 1e3,
        "solve": {"value": 1.0 / ts, "unit": "solves/s", "iterations": mon.iter,
                  "converged": mon.converged, "max_error_vs_sin3": err,
                  "workload": "Jacobi-PCG to 1e-10 rel, f = 3 pi^2 sin^3 + N(0,1e-3)"},
    }), flush=True)
    P.close()


def run_serve(args):
    """Served request stream: open-loop Poisson arrivals at each of
    --serve-rates (plus one rate at half the measured capacity when no
    given rate is below three quarters of it), --serve-requests requests per rate drawn as the
    batched workload, answered by the continuous-batching server under a
    --serve-budget-gb HBM budget in mixed precision and in FP64 (hsmg
    problems as per-problem solves, Jacobi ones in the persistent batched
    launch), and a bounded sample of each stream by the one-request-at-a-time
    server on the plain FP64 path; latency percentiles and solves/s."""
    import numpy as np
    import torch
    import neko_b200 as nb
    from neko_b200 import serve, workloads
    torch.cuda.set_device(0)
    cache = serve.GeometryCache()
    pool = serve.RhsPool(cache)
    inst = serve.InstancePool(cache, variants=(False, True))
    stream = torch.cuda.Stream()
    # capacity: the solves/s of a saturated mixed-precision stream
    cap_specs = workloads.uneven_specs(min(args.serve_requests, 512), seed=args.seed + 999)
    for sp in cap_specs:
        pool.get(sp)
    B = nb.Batch(hbm_budget=max(int(args.serve_budget_gb * 1e9) - cache.device_bytes(), 1))
    zeros = np.zeros(len(cap_specs))
    serve.serve_batched(cap_specs, zeros, pool, 0, batch=B, mode="mixed", instances=inst,
                        max_solves=args.max_solves, stream=stream, keep_solutions=False)
    _, _, _, span, _ = serve.serve_batched(cap_specs, zeros, pool, 0, batch=B, mode="mixed",
                                           instances=inst, max_solves=args.max_solves,
                                           stream=stream, keep_solutions=False)
    capacity = len(cap_specs) / span
    rates = [float(r) for r in args.serve_rates.split(",")]
    # a rate well below the capacity, so that one stream's latencies are
    # service time rather than queueing
    if min(rates) >= 0.75 * capacity:
        rates.insert(0, round(0.5 * capacity, 1))
    out = {}
    for q, rate in enumerate(rates):
        specs = workloads.uneven_specs(args.serve_requests, seed=args.seed + 17 * q)
        for sp in specs:
            pool.get(sp)
        t_arr = serve.arrivals(rate, len(specs), seed=args.seed + q)
        # untimed warm-up over the head of the stream with every request
        # present at once: the instances (and their preconditioners) that
        # the stream's concurrency needs exist before the timed run, as on a
        # server that has been running
        head = specs[:min(len(specs), 2000)]
        for mode in ("mixed", "fp64"):
            serve.serve_batched(head, np.zeros(len(head)), pool, 0, batch=B, mode=mode,
                                instances=inst, max_solves=args.max_solves, stream=stream,
                                keep_solutions=False)
        r = {}
        for mode in ("mixed", "fp64"):
            status = []
            lat, it, conv, span, _ = serve.serve_batched(
                specs, t_arr, pool, 0, batch=B, mode=mode, instances=inst,
                max_solves=args.max_solves, stream=stream, status=status,
                keep_solutions=False)
            r[mode] = dict(serve.percentiles(lat), solves_per_s=len(specs) / span,
                           requests=len(specs), converged=int(sum(conv)),
                           mean_iter=float(np.mean(it)), span_s=span)
        k = min(args.serve_seq_requests, len(specs))
        lat_s, it_s, conv_s, span_s = serve.serve_sequential(specs[:k], t_arr[:k], pool,
                                                             mode="fp64")
        r["one_by_one_fp64"] = dict(serve.percentiles(lat_s), solves_per_s=k / span_s,
                                    requests=k, converged=int(sum(conv_s)))
        r["arrival_span_s"] = float(t_arr[-1])
        out[str(rate)] = r
    first = str(rates[0])
    line = {
        "metric": "served Helmholtz solves: p50/p95/p99 latency (ms) and solves/s",
        "value": out[first]["mixed"]["p99_ms"],
        "unit": f"ms (p99, mixed precision, at {rates[0]:g} req/s)", "higher_is_better": False,
        "n_gpus": 1, "dtype": "f64+f32", "data": "synthetic", "vs_baseline": None,
        "config": {"workload": f"{args.serve_requests} requests per rate, open-loop Poisson "
                               f"arrivals, shapes/orders/coefficients as the batched workload, "
                               f"hsmg flexible CG (boxes above 3^3 elements) or Jacobi-PCG, "
                               f"to 1e-8 rel, HBM budget {args.serve_budget_gb:.0f} GB, "
                               f"geometry cached by (n, lx, deformation seed)",
                   "rates_per_s": rates, "capacity_solves_per_s": capacity,
                   "max_concurrent_hsmg_solves": args.max_solves,
                   "one_by_one_sample": f"first {args.serve_seq_requests} requests of each "
                                        f"stream",
                   "warm_server": "geometry, right-hand sides and problem instances with "
                                  "their preconditioners built before each timed stream "
                                  "(an untimed pass over its first 2000 requests)",
                   "geometries": len(cache.problems), "instances": inst.instances(),
                   "instances_evicted": inst.evicted, "instance_waits": inst.deferred,
                   "setup_s": cache.setup_s + inst.setup_s},
        "rates": out,
    }
    print(json.dumps(line), flush=True)
    B.close()
    inst.close()
    cache.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--pc", default="hsmg", choices=["jacobi", "hsmg", "phmg"])
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--ax-reps", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU oracle solve (cpu_baseline and the parity fields)")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision solve measured beside the FP64 one")
    ap.add_argument("--no-phmg", action="store_true",
                    help="skip the phmg-CG solve measured beside the hsmg-FCG one")
    ap.add_argument("--kernel-only", choices=["ax", "dropin_ax", "fused", "gs", "stress",
                                              "dropin_fdm",
                                              "dropin_tnsr3d", "solve"],
                    default=None,
                    help="run only this kernel (or one FP64 + one mixed solve inside a "
                         "profiler window) on an nel^3 box (profiling case)")
    ap.add_argument("--workload", choices=["solve", "axgs", "batch", "serve", "velocity"],
                    default="solve",
                    help="solve: the hsmg-FCG line on the periodic 32^3 box (default); batch: batched "
                         "uneven solves; serve: the served request stream; velocity: the "
                         "coupled full-stress velocity solve on the periodic 32^3 box")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--max-solves", type=int, default=64,
                    help="per-problem hsmg solves running at once in the batch / server")
    ap.add_argument("--coarse-tol", type=float, default=1e-9,
                    help="hsmg coarse CG absolute tolerance (reference KSP_ABS_TOL 1e-9; "
                         "1e-4 is the weaker variant)")
    ap.add_argument("--serve-rates", default="200,1000,5000")
    ap.add_argument("--serve-requests", type=int, default=20000)
    ap.add_argument("--serve-seq-requests", type=int, default=1000,
                    help="requests of each stream also answered one at a time")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--nel", type=int, default=16)
    ap.add_argument("--lx", type=int, default=8)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    from neko_b200 import workloads
    cfg = dict(workloads.PERIODIC_BOX_32)
    cfg["lx"] = args.lx
    if args.kernel_only:
        return kernel_only(args, cfg)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "axgs":
        return run_axgs(args)
    if args.workload == "velocity":
        return run_velocity(args)
    world, rank, local = dist_setup()

    if args.impl == "reference":
        run_reference(args, cfg, world, rank)
        barrier(world)
        return

    import torch
    import neko_b200 as nb
    torch.cuda.set_device(local)
    P = build_problem(nb, cfg)
    b = make_rhs(nb, P, args.seed + rank)
    mult = P.field("mult")
    r0 = math.sqrt(float((b * mult * b).sum()) / P.volume)
    tol = cfg["rel_tol"] * r0
    if args.pc == "jacobi":
        solver = nb.CG(max_iter=cfg["max_iter"], abs_tol=tol, M=nb.Jacobi())
    elif args.pc == "phmg":  # Chebyshev smoothing and an AMG V-cycle: symmetric, plain CG
        solver = nb.CG(max_iter=cfg["max_iter"], abs_tol=tol, M=nb.Phmg())
    else:  # hsmg is not symmetric: flexible CG (plain CG stalls with it)
        solver = nb.FCG(max_iter=cfg["max_iter"], abs_tol=tol,
                        M=nb.Hsmg(coarse_tol=args.coarse_tol))
    msolver = None
    if args.pc == "hsmg" and not args.no_mixed:
        msolver = nb.FCG(max_iter=cfg["max_iter"], abs_tol=tol,
                         M=nb.Hsmg(coarse_tol=args.coarse_tol, mixed=True))
    Ax = nb.AxHelm()
    x = P.zeros()
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            mon = solver.solve(Ax, x, b, P.n, P, stream=stream)
    torch.cuda.synchronize()
    if not mon.converged:
        raise RuntimeError(f"warm-up solve did not converge: {mon}")
    x64 = x.clone()
    xm = None
    if msolver is not None:
        for _ in range(args.warmup):
            mon_m = msolver.solve(Ax, x, b, P.n, P, stream=stream)
        torch.cuda.synchronize()
        if not mon_m.converged:
            raise RuntimeError(f"mixed warm-up solve did not converge: {mon_m}")
        xm = x.clone()

    def timed(fn, steps):
        """Device time of `steps` calls of fn on `stream`, max over ranks."""
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        out = [fn() for _ in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(e0.elapsed_time(e1) / 1e3, world), out

    hb = b.cpu().pin_memory()
    hx = [torch.empty(P.n, dtype=torch.float64).pin_memory() for _ in range(2)]
    fdev = torch.empty_like(b)
    with ClockSampler(local) as clk:
        # --- device-timed steps (inputs resident in HBM, > L2) -----------
        t_dev, mons = timed(lambda: solver.solve(Ax, x, b, P.n, P, stream=stream), args.steps)
        launches = sum(m.launches for m in mons)
        iters = [m.iter for m in mons]
        value = world * args.steps / t_dev

        # --- end to end through the public API with host buffers ---------
        # Every step uploads its right-hand side from pinned host memory and
        # downloads its solution.  Pipelined as a serving loop would run it:
        # the upload of step k+1 and the download of step k-1 run on a copy
        # stream while step k solves; device staging buffers keep the
        # solver's operands (and so its captured iteration graph) fixed.
        # The serial form (copy, solve, copy on one stream) is reported
        # beside it.
        f_st = [torch.empty_like(b) for _ in range(2)]
        x_st = [torch.empty_like(b) for _ in range(2)]
        cstream = torch.cuda.Stream()
        ev = lambda: torch.cuda.Event()
        ev_in, ev_used, ev_done, ev_out = ([ev(), ev()] for _ in range(4))
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cstream.wait_stream(stream)
        with torch.cuda.stream(cstream):
            f_st[0].copy_(hb, non_blocking=True)
            ev_in[0].record(cstream)
        for k in range(args.steps):
            bk = k % 2
            if k + 1 < args.steps:  # prefetch the next input while this step solves
                with torch.cuda.stream(cstream):
                    if k >= 1:
                        cstream.wait_event(ev_used[1 - bk])
                    f_st[1 - bk].copy_(hb, non_blocking=True)
                    ev_in[1 - bk].record(cstream)
            with torch.cuda.stream(stream):
                stream.wait_event(ev_in[bk])
                fdev.copy_(f_st[bk], non_blocking=True)
                ev_used[bk].record(stream)
                solver.solve(Ax, x, fdev, P.n, P, stream=stream)
                if k >= 2:
                    stream.wait_event(ev_out[bk])
                x_st[bk].copy_(x, non_blocking=True)
                ev_done[bk].record(stream)
            with torch.cuda.stream(cstream):
                cstream.wait_event(ev_done[bk])
                hx[bk].copy_(x_st[bk], non_blocking=True)
                ev_out[bk].record(cstream)
        stream.wait_stream(cstream)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
        e2e = world * args.steps / t_e2e
        if not torch.equal(hx[(args.steps - 1) % 2], x.cpu()):
            raise RuntimeError("end-to-end solution read back differs from the device solution")

        def serial_step():
            with torch.cuda.stream(stream):
                fdev.copy_(hb, non_blocking=True)
                solver.solve(Ax, x, fdev, P.n, P, stream=stream)
                hx[0].copy_(x, non_blocking=True)
        t_ser, _ = timed(serial_step, args.steps)
        e2e_serial = world * args.steps / t_ser

        # --- mixed precision beside it: FP32 smoothing levels, FP64 FCG --
        mixed = None
        if msolver is not None:
            t_m, mons_m = timed(lambda: msolver.solve(Ax, x, b, P.n, P, stream=stream),
                                args.steps)
            mon_m = mons_m[-1]
            v_m = world * args.steps / t_m
            singular = all(cfg["periodic"])
            err = rel_err_mean_free(x.cpu().numpy(), x64.cpu().numpy(), singular)
            mixed = {"value": v_m, "unit": "solves/s", "ms_per_step": t_m / args.steps * 1e3,
                     "iterations": mon_m.iter, "fp64_iterations": iters[-1],
                     "res_final": mon_m.res_final, "abs_tol": tol,
                     "err_vs_fp64": err,
                     "speedup_vs_fp64": v_m / value,
                     "gpu_launches": sum(m.launches for m in mons_m),
                     "precision": "FP32 Schwarz/FDM smoothing and restriction/prolongation; "
                                  "FP64 outer FCG, inner products, coarse CG, true residual "
                                  "every 50 iterations"}

        # --- phmg-CG beside it: the other multigrid of the reference --------
        phmg = None
        if args.pc == "hsmg" and not args.no_phmg:
            psolver = nb.CG(max_iter=cfg["max_iter"], abs_tol=tol, M=nb.Phmg())
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            psolver.M.init(P)  # levels, aggregation, 150-step eigenvalue estimates
            t_setup = time.perf_counter() - t0
            for _ in range(args.warmup):
                mon_p = psolver.solve(Ax, x, b, P.n, P, stream=stream)
            torch.cuda.synchronize()
            if not mon_p.converged:
                raise RuntimeError(f"phmg warm-up solve did not converge: {mon_p}")
            t_p, mons_p = timed(lambda: psolver.solve(Ax, x, b, P.n, P, stream=stream),
                                args.steps)
            v_p = world * args.steps / t_p
            phmg = {"value": v_p, "unit": "solves/s", "ms_per_step": t_p / args.steps * 1e3,
                    "iterations": mons_p[-1].iter, "res_final": mons_p[-1].res_final,
                    "abs_tol": tol, "speedup_vs_hsmg_fp64": v_p / value,
                    "err_vs_hsmg_fp64": rel_err_mean_free(x.cpu().numpy(), x64.cpu().numpy(),
                                                          all(cfg["periodic"])),
                    "setup_s": t_setup,
                    "gpu_launches": sum(m.launches for m in mons_p),
                    "settings": "levels lx 8 -> 4 -> 2, 3 Chebyshev-Jacobi steps a level, "
                                "tree AMG of 3 levels (Chebyshev degree 4, one V-cycle); "
                                "plain CG, FP64"}

        # --- the dominant kernel of the solve, timed with events ----------
        # The fused CG step (p = z + beta p, w = A p, sum p w: 88 B/point) is
        # the largest share of the solve's device time; it is timed on its
        # launching stream, three loops of --ax-reps launches, median loop.
        # The standalone operator (72 B/point) is timed the same way.
        w = P.zeros()
        pd = x64.clone()
        zd = b.clone()
        pap = torch.zeros(1, dtype=torch.float64, device="cuda")

        def loop_time(fn):
            for _ in range(5):
                fn()
            loops = []
            for _ in range(3):
                t, _ = timed(lambda: [fn() for _ in range(args.ax_reps)], 1)
                loops.append(t / args.ax_reps)
            return sorted(loops)[1]
        t_fused = loop_time(lambda: Ax.update_p_compute(w, pd, zd, 0.0, P, pap=pap, stream=stream))
        t_ax = loop_time(lambda: Ax.compute(w, x64, P, stream=stream))
        # the fine-level gather-scatter add, in place on a copy of x
        gu = x64.clone()
        t_gs = loop_time(lambda: P.gs.op(gu, P.n, stream=stream))
    peaks, peak_src = measured_peaks()
    fused_bytes = 88 * P.n  # z, p read; p, w written; h1, G11..G23 read
    ax_bytes = 72 * P.n     # u, w, h1, G11..G23
    gs_bytes = GS_B_PER_ENTRY * P.nlocal
    achieved = fused_bytes / t_fused / 1e9
    traffic_pp = FUSED_TRAFFIC_B_PER_POINT.get(cfg["lx"])
    singular = all(cfg["periodic"])

    line = {
        "metric": "Poisson solves/s to 1e-8 rel", "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(
                       cfg, "FP64 " + {"jacobi": "Jacobi-PCG", "hsmg": "hsmg-FCG",
                                       "phmg": "phmg-CG"}[args.pc])
                       + ", one solve per step per GPU",
                   "pc": args.pc, "iterations": iters[-1], "r0": r0, "seed": args.seed,
                   "coarse": f"10 Jacobi-CG iterations, abs tol {args.coarse_tol:g}",
                   "l2": f"inputs larger than L2 ({88 * P.n / 1e9:.1f} GB fused-step working set)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": P.n * 8,
                "d2h_bytes_per_step": P.n * 8,
                "form": "pipelined: step k+1's upload and step k-1's download overlap "
                        "step k's solve on a second stream",
                "serial_value": e2e_serial},
        "roofline": {"bound": "hbm",
                     "kernel": f"ax_cg_fused_kernel<{cfg['lx']}> (p = z + beta p, w = A p, "
                               f"sum p w; the solve's largest kernel)",
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"],
                     "traffic": traffic_pp * P.n if traffic_pp else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per "
                                       "point of a 24^3-element launch of the same kernel, "
                                       "times the points",
                     "peak_source": peak_src, "bytes_per_launch": fused_bytes,
                     "launch_ms": t_fused * 1e3, "gdof_s": P.n / t_fused / 1e9},
        "ax_helm": {"kernel": f"ax_helm_tma_kernel<double,{cfg['lx']}>",
                    "achieved": ax_bytes / t_ax / 1e9, "unit": "GB/s",
                    "frac": ax_bytes / t_ax / 1e9 / peaks["hbm_gbs"],
                    "bytes_per_launch": ax_bytes, "launch_ms": t_ax * 1e3,
                    "gdof_s": P.n / t_ax / 1e9},
        "gs": {"kernel": "gs_add_warp_kernel<double,4>",
               "achieved": gs_bytes / t_gs / 1e9, "unit": "GB/s",
               "frac": gs_bytes / t_gs / 1e9 / peaks["hbm_gbs"],
               "entries": P.nlocal, "bytes_per_launch": gs_bytes,
               "bytes_definition": f"{GS_B_PER_ENTRY} B per local entry (value read and "
                                   f"written, 4 B index)",
               "launch_ms": t_gs * 1e3},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if mixed is not None:
        line["mixed"] = mixed
    if phmg is not None:
        line["phmg"] = phmg
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # One complete FP64 solve of the CPU oracle on the same right-hand
        # side: the CPU baseline (whole solve, host threads), and the parity
        # of the GPU solves at full size (iterations within +-1, error).
        O = oracle_problem(cfg)
        xo, it_o, dt_o, _ = oracle_solve(O, b.cpu().numpy(), args.pc, tol, args.coarse_tol,
                                         cfg["max_iter"])
        O.close()
        cores = host_threads()
        name = {"hsmg": "hsmg-FCG", "phmg": "phmg-CG", "jacobi": "Jacobi-PCG"}[args.pc]
        line["cpu_baseline"] = {
            "value": 1.0 / dt_o, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"one complete FP64 {name} solve of the same problem and right-hand "
                      f"side to 1e-8 rel ({it_o} iterations, {dt_o:.1f} s) on {cores} host "
                      f"threads, preconditioner set-up untimed"}
        line["parity"] = {
            "iterations": iters[-1], "iterations_oracle": it_o,
            "err_vs_oracle": rel_err_mean_free(x64.cpu().numpy(), xo, singular),
            "err_definition": "relative L2 distance to the CPU oracle's FP64 solution"
                              + (" (both mean-free: the periodic problem is singular)"
                                 if singular else "")}
        if mixed is not None:
            mixed["err_vs_oracle"] = rel_err_mean_free(xm.cpu().numpy(), xo, singular)
    if rank == 0:
        print(json.dumps(line), flush=True)
    P.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
