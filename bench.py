"""SOL101 throughput benchmark (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed] [--workload wing_panel|plate|solid_block]

Workload (default): the stiffened wing-box panel -- 200x400 CQUAD4 skin plus 9
blade stiffeners of 20x400 CQUAD4 (152,781 GRIDs, 916,686 DOF, 914,400 free),
8 subcases.  One step = one SOL101 analysis of that model on the device:
element kernels + slot-map assembly + numeric Cholesky + forward/backward
solves of the 8 subcases with FP64 refinement to relative residual 1e-10.
The symbolic analysis and the CSC pattern are built once per mesh, before the
timed region (the device-resident model registry keeps them).

value  = SOL101 solves/s with the model and the load matrix resident in HBM.
e2e    = the same through the public C ABI with host buffers: every step
         copies the 8 load cases host->device and the 8 displacement fields
         device->host (jfg_solve with host arrays).
Multi-GPU: replicas only -- every rank solves its own copy; value is the sum
over ranks of solves divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SOL101 solves/s & p50/p99 latency, mixed+IR vs FP64 Cholesky, resid<=1e-10"


def make_workload(name: str):
    from jf_2026_05_25_b200 import model as M
    if name == "wing_panel":
        return M.wing_panel(), {"workload": "wing_panel_200x400_9blades_20x400", "grids": 152781,
                                "cquad4": 152000, "ndof": 916686, "free_dof": 914400, "subcases": 8}
    if name == "wing_panel_small":
        m = M.wing_panel(nx=100, ny=200, blade_nz=10)
        return m, {"workload": "wing_panel_100x200_9blades_10x200", "grids": m.n_nodes,
                   "cquad4": len(m.q4_nodes), "ndof": m.ndof, "subcases": len(m.load_cases)}
    if name == "plate":
        return M.flat_plate(), {"workload": "flat_plate_20x20", "grids": 441, "ndof": 2646, "subcases": 1}
    if name == "solid_block":
        return M.solid_block(), {"workload": "solid_block_40cube_ctetra10", "grids": 531441, "ctetra10": 384000,
                                 "ndof": 3188646, "subcases": 4}
    if name == "solid_block_small":   # profiling-sized case of the same kernels
        m = M.solid_block(n=16)
        return m, {"workload": "solid_block_16cube_ctetra10", "grids": m.n_nodes, "ctetra10": len(m.t10_nodes),
                   "ndof": m.ndof, "subcases": len(m.load_cases)}
    raise ValueError(name)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU arms
def cpu_sol101(mdl, nthreads, u_keep=False):
    """The CPU restatement of the reference path (oracle only; the device
    library is not loaded): element loop and sparse() CSC, the SPC1 +
    AUTOSPC partition, K_ff, the oracle's CHOLMOD-rule ordering (approximate
    minimum degree, nested dissection when that is poor), supernodal
    Cholesky with OpenBLAS, then one RHS at a time."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    asm = O.assemble(mdl)
    K = O.csc_matrix(asm)
    t1 = time.perf_counter()
    free, _, _ = O.partition(mdl, K)
    Kff = K[free][:, free].tocsc()
    perm, oinfo = O.order(Kff, free, mdl.xyz)
    t2 = time.perf_counter()
    F = O.load_matrix(mdl)
    U, info = O.chol_solve(len(free), Kff.indptr.astype(np.int64), Kff.indices, Kff.data, perm, F[free],
                           nthreads=nthreads)
    t3 = time.perf_counter()
    out = dict(assembly_s=t1 - t0, constraints_ordering_s=t2 - t1, factor_s=info["factor_s"],
               solve_s=info["solve_s"], total_s=t3 - t0, flops=info["flops"], nnz_L=info["nnz_L"],
               ordering=oinfo["method"])
    if u_keep:
        u = np.zeros((mdl.ndof, F.shape[1]))
        u[free] = U
        out["u"] = u
        out["free"] = free
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    os.environ.setdefault("JFEM_ORACLE_OPENBLAS", _openblas())
    mdl, cfg = make_workload(args.workload)
    nthreads = os.cpu_count() or 1
    times = []
    for k in range(args.warmup + args.steps):
        r = cpu_sol101(mdl, nthreads)
        if k >= args.warmup:
            times.append(r["total_s"])
    ms = 1000.0 * float(np.mean(times))
    value = 1000.0 / ms
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": dict(cfg, parallelism="cpu", precision="fp64",
                           note="CPU restatement of the reference SOL101 path (Julia/CHOLMOD unavailable on this box)"),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "port",
                             "sample": f"full {cfg['workload']} SOL101 per step (assembly, sparse(), K_ff, "
                                       f"supernodal Cholesky, {cfg['subcases']} single-RHS solves)"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "stages_s": r}
    print(json.dumps(line), flush=True)


def _openblas():
    import glob
    import scipy
    c = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "libscipy_openblas-*.so"))
    return os.path.abspath(c[0]) if c else ""


# ---------------------------------------------------------------- replicas
def slowest_rank(seconds: float, world: int, device: str) -> float:
    """Max over ranks of a per-rank time: with replicas the job ends when the
    slowest rank does (every rank takes this collective at the same point)."""
    if world <= 1:
        return seconds
    import torch
    import torch.distributed as dist
    tt = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def replica_throughput(steps: int, world: int, seconds: float) -> float:
    """Whole-job throughput of N independent replicas: every rank solved
    `steps` analyses, the job took the slowest rank's time."""
    return world * steps / seconds


# ---------------------------------------------------------------- device arm
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from jf_2026_05_25_b200 import backend as B
    from jf_2026_05_25_b200 import lib
    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local_rank))
    L = lib.load()
    prec = lib.PREC_MIXED if args.precision == "mixed" else lib.PREC_FP64
    mdl, cfg = make_workload(args.workload)
    be = B.JFEMGPUBackend(device=local_rank, precision=prec, tol=1e-10)
    st = B.prepare(be, mdl)
    dm = st["dm"]
    sym = dm.symbolic_info()
    F = mdl.load_matrix()
    nrhs = F.shape[1]
    dF = torch.from_numpy(np.asarray(F, order="F").T.copy()).to("cuda")   # [nrhs, ndof] == column-major ndof x nrhs
    dU = torch.zeros_like(dF)
    hF = torch.from_numpy(np.ascontiguousarray(np.asarray(F, order="F").T)).pin_memory()
    hU = torch.zeros_like(hF).pin_memory()
    stream = torch.cuda.current_stream()

    def step_device():
        dm.assemble()
        dm.factor(prec)
        return dm.solve_device(dF.data_ptr(), dU.data_ptr(), nrhs, 1e-10, 20, raise_on_stall=False)

    def step_e2e():
        dm.assemble()
        dm.factor(prec)
        rep = lib.SolveReport()
        st_ = L.jfg_solve(dm.h, nrhs, lib.P(hF.data_ptr()), lib.P(hU.data_ptr()), 1e-10, 20, lib._c.byref(rep))
        if st_ not in (0, 2):
            lib._check(st_)
        return rep.as_dict()

    for _ in range(args.warmup):
        rep = step_device()
    # ---- timed region (device-resident inputs)
    clocks = ClockSampler(local_rank)
    clocks.start()
    L.jfg_reset_kernel_stats()
    L.jfg_set_profiling(1)
    launches0 = L.jfg_launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t_wall0 = time.perf_counter()
    reps = []
    for _ in range(args.steps):
        reps.append(step_device())
    e1.record(stream)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    launches = L.jfg_launch_count() - launches0
    L.jfg_set_profiling(0)
    # The library runs on its own stream and synchronises before returning, so
    # the host interval between two device synchronisations brackets exactly
    # the device work of the K steps; the torch events on the current stream
    # give the same interval on the device clock.
    ms_dev = max(e0.elapsed_time(e1), 1000.0 * t_wall)
    ms_dev = slowest_rank(ms_dev, world, "cuda")
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    stats = {}
    for which, name in ((0, "schur_update"), (1, "q4_element"), (2, "assembly_gather"), (3, "solves"),
                        (4, "t10_element"), (5, "f_extend_add"), (6, "f_potrf"), (7, "f_trsm"), (8, "f_panel_update"),
                        (9, "s_vec_extend_add"), (10, "s_fwd_diag"), (11, "s_fwd_update"), (12, "s_bwd_partial"),
                        (13, "s_bwd_diag")):
        o = np.zeros(3)
        L.jfg_get_kernel_stats(which, o.ctypes.data_as(lib.P))
        if o[0] > 0:
            stats[name] = {"launches": int(o[0]), "ms": float(o[1]), "units": float(o[2])}
    ms_step = ms_dev / args.steps
    value = replica_throughput(args.steps, world, ms_dev / 1000.0)
    # ---- e2e through the public API with host buffers
    if not args.no_e2e:
        step_e2e()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(0 if args.no_e2e else args.steps):
        step_e2e()
    torch.cuda.synchronize()
    e2e_s = max(time.perf_counter() - t0, 1e-9)
    e2e_s = slowest_rank(e2e_s, world, "cuda")
    e2e_value = replica_throughput(args.steps, world, e2e_s)
    # ---- roofline of the dominant kernel
    peaks = _peaks()
    # the roofline reports the dominant single kernel among the coarse classes
    coarse = {k: v for k, v in stats.items() if k in ("schur_update", "q4_element", "assembly_gather", "solves",
                                                     "t10_element")}
    dom = max(coarse.items(), key=lambda kv: kv[1]["ms"]) if coarse else None
    roof = None
    if dom:
        name, s = dom
        if name == "schur_update":
            achieved = s["units"] / (s["ms"] / 1000.0) / 1e12
            if prec == lib.PREC_MIXED:
                peak, src = peaks["tf32x3_tflops"], peaks["src"] + " bf16/2/3 (3xTF32)"
            else:
                peak, src = peaks["fp64_tflops"], "nominal B200 FP64 40 TFLOP/s (no measured FP64 peak)"
            roof = {"kernel": name, "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None, "peak_source": src,
                    "launches": s["launches"], "ms_total": s["ms"]}
        else:
            achieved = s["units"] / (s["ms"] / 1000.0) / 1e9
            peak = peaks["hbm_gbs"]
            roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": None, "peak_source": peaks["src"] + " hbm_gbs",
                    "launches": s["launches"], "ms_total": s["ms"]}
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        os.environ.setdefault("JFEM_ORACLE_OPENBLAS", _openblas())
        nthreads = os.cpu_count() or 1
        r = cpu_sol101(mdl, nthreads, u_keep=True)
        u_ref = r.pop("u")
        free_ref = r.pop("free")
        U_dev = dU.double().cpu().numpy().T          # ndof x nrhs
        parity = {"max_rel_disp_err_vs_fp64_oracle": float(np.abs(U_dev - u_ref).max() / np.abs(u_ref).max()),
                  "same_free_set": bool(np.array_equal(free_ref, st["free"])),
                  "oracle": "CPU restatement: oracle partition and ordering, supernodal FP64 Cholesky (OpenBLAS)"}
        cpu = {"value": 1.0 / r["total_s"], "unit": "solves/s", "cores": nthreads, "kind": "port",
               "sample": f"one full {cfg['workload']} SOL101 (assembly, sparse(), partition, ordering, K_ff, "
                         f"supernodal Cholesky with OpenBLAS, {cfg['subcases']} single-RHS solves)",
               "stages_s": r}
    rep = reps[-1]
    tflops_factor = sym["flops"] / 1e12
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == lib.PREC_FP64 else "f32+f64",
            "data": "synthetic",
            "config": dict(cfg, parallelism=f"replicas{world}", precision=args.precision,
                           l2="inputs larger than L2 (factor %.1f GB)" % (sym["nnz_L"] * (8 if prec == 0 else 4) / 1e9)),
            "e2e": None if args.no_e2e else {"value": e2e_value, "unit": "solves/s",
                                             "h2d_bytes_per_step": int(F.nbytes), "d2h_bytes_per_step": int(F.nbytes)},
            "gpu_launches": int(launches),
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            "parity": parity,
            "detail": {"rel_residual": rep["rel_residual"], "ir_iters": rep["ir_iters"],
                       "fallback_used": rep["fallback_used"], "subcase_solves_per_s": value * nrhs,
                       "factor_tflop": tflops_factor, "factor_tflops_per_s": tflops_factor / (ms_step / 1000.0),
                       "dof_per_s_assembled": cfg["ndof"] * value, "symbolic": sym, "kernel_stats": stats,
                       "phase_s_last_step": dm.timings()}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    dm.close()
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------- batched and serving workloads
def _lat(xs):
    xs = np.asarray(xs, float)
    return {"p50_ms": float(np.percentile(xs, 50) * 1e3), "p99_ms": float(np.percentile(xs, 99) * 1e3)}


def run_batched(args):
    """1,024 independent stiffened panels (seeded generator; 0.5k-50k DOF,
    1-16 subcases each).  Untimed: pattern, partition and symbolic analysis
    of every pack.  One step: element kernels + assembly + numeric factor +
    all subcase solves of every model.  Packed arm: models packed into
    block-diagonal packs of <= --pack-dof DOF, packs spread over --slots
    device streams.  Per-model arm: every model alone on one stream, plain
    FP64.  Latency of a model = time from step start to its result."""
    import threading
    import torch
    from jf_2026_05_25_b200 import backend as B
    from jf_2026_05_25_b200 import lib
    from jf_2026_05_25_b200 import model as M
    from jf_2026_05_25_b200 import serving as S
    prec = lib.PREC_MIXED if args.precision == "mixed" else lib.PREC_FP64
    models = [M.stiffened_panel(sd) for sd in range(args.models)]
    n_sub = sum(len(m.load_cases) for m in models)
    packs, cur, dof = [], [], 0
    for m in models:
        if cur and (dof + m.ndof > args.pack_dof or len(cur) >= 128):
            packs.append(cur); cur, dof = [], 0
        cur.append(m); dof += m.ndof
    if cur:
        packs.append(cur)
    ctxs = [lib.Context(0) for _ in range(args.slots)]
    work = []
    for i, p in enumerate(packs):
        be = B.JFEMGPUBackend(precision=prec, tol=1e-10)
        be._ctx = ctxs[i % args.slots]
        pk = S.PackedModel(p)
        st = B.prepare(be, pk)
        F, sc = pk.load_columns()
        work.append((i % args.slots, pk, st, F, sc, 0.5e-10 / np.sqrt(len(p))))
    done = [0.0] * len(work)
    worst = [0.0]

    def slot_run(si, t0, check):
        for j, (sj, pk, st, F, sc, tol) in enumerate(work):
            if sj != si:
                continue
            dm = st["dm"]
            dm.assemble()
            dm.factor(prec)
            U, rep = dm.solve(F, tol, 30, raise_on_stall=False)
            done[j] = time.perf_counter() - t0
            if check:
                res = S.member_residuals(dm, pk, U, F, st["free"], [len(x) for x in sc])
                worst[0] = max(worst[0], max(float(r.max()) for r in res))

    def step(check=False):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        th = [threading.Thread(target=slot_run, args=(si, t0, check)) for si in range(args.slots)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    times, lats = [], []
    for k in range(args.steps):
        times.append(step(check=(k == args.steps - 1)))
        for j, (_, pk, *_r) in enumerate(work):
            lats += [done[j]] * len(pk.members)
    packed_s = float(np.mean(times))
    # per-model plain FP64 arm on a bounded sample (every model alone)
    sample = models[:args.baseline_models]
    alone = []
    for m in sample:
        be = B.JFEMGPUBackend(precision=lib.PREC_FP64, tol=1e-10)
        be._ctx = ctxs[0]
        st = B.prepare(be, m)
        alone.append((st["dm"], m.load_matrix()))
    for dm, F in alone[:4]:
        dm.assemble(); dm.factor(lib.PREC_FP64); dm.solve(F, 1e-10, 30, raise_on_stall=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    alone_lat = []
    for dm, F in alone:
        dm.assemble(); dm.factor(lib.PREC_FP64); dm.solve(F, 1e-10, 30, raise_on_stall=False)
        alone_lat.append(time.perf_counter() - t0)
    alone_s = time.perf_counter() - t0
    alone_sub = sum(F.shape[1] for _, F in alone)
    value = n_sub / packed_s
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": packed_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == lib.PREC_FP64 else "f32+f64", "data": "synthetic",
            "config": {"workload": f"batched_stiffened_panels_{args.models}", "models": args.models,
                       "dof_total": int(sum(m.ndof for m in models)), "subcases": n_sub, "packs": len(packs),
                       "pack_dof": args.pack_dof, "streams": args.slots, "precision": args.precision,
                       "timing": "host clock around device-synchronised steps (several device streams)"},
            "latency": _lat(lats), "max_member_rel_residual": worst[0],
            "per_model_fp64": {"models": len(sample), "subcase_solves_per_s": alone_sub / alone_s,
                               "latency": _lat(np.diff(np.concatenate([[0.0], alone_lat])))},
            "speedup_vs_per_model_fp64": value / (alone_sub / alone_s)}
    print(json.dumps(line), flush=True)


def run_serving(args):
    """Serving stream: Poisson arrivals at --rate requests/s, --requests in
    total; 70 % stiffened panels (configs[3] class), 25 % wing boxes, 5 %
    solid blocks (configs[1]/[2] classes at reduced sizes so the stream ends
    in minutes: wing nx U{50..200} x ny U{100..400} with 9 blades, solid n
    U{12..20}); 30 % of the requests re-solve a resident model with new
    loads or with CQUAD4 thicknesses scaled U[0.9, 1.1].  Admission against
    a 150 GB HBM budget.  Latency = arrival to result."""
    import torch
    from jf_2026_05_25_b200 import lib
    from jf_2026_05_25_b200 import model as M
    from jf_2026_05_25_b200 import serving as S
    prec = lib.PREC_MIXED if args.precision == "mixed" else lib.PREC_FP64
    rng = np.random.default_rng(7)
    kinds = rng.choice(3, size=args.requests, p=[0.7, 0.25, 0.05])
    resolve = rng.random(args.requests) < 0.3
    pool = []
    for i, k in enumerate(kinds):
        if k == 0:
            pool.append(M.stiffened_panel(1000 + i))
        elif k == 1:
            pool.append(M.wing_panel(nx=int(rng.integers(50, 201)), ny=int(rng.integers(100, 401)),
                                     blade_nz=10, n_cases=int(rng.integers(1, 9)), seed=i))
        else:
            pool.append(M.solid_block(n=int(rng.integers(12, 21)), n_cases=int(rng.integers(1, 5)), seed=i))
    gaps = rng.exponential(1.0 / args.rate, size=args.requests)
    srv = S.SolveServer(slots=args.slots, hbm_budget_bytes=150e9, precision=prec, tol=1e-10)
    # warm-up: compile paths and allocator state on a few panels
    for f in [srv.solve(M.stiffened_panel(s)) for s in range(args.warmup)]:
        f.result()
    srv.latencies.clear()
    srv.subcase_solves = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    futs, keys = [], []
    for i in range(args.requests):
        target = t0 + float(np.sum(gaps[:i + 1]))
        now = time.perf_counter()
        if target > now:
            time.sleep(target - now)
        done_keys = [f.result()["key"] for f in futs if f.done() and f.exception() is None and "key" in f.result()]
        if resolve[i] and done_keys:
            key = done_keys[int(rng.integers(len(done_keys)))]
            res = srv.registry.get(key)
            if res is not None and len(res.model.q4_nodes) and rng.random() < 0.5:
                sect = res.model.q4_sections().copy()
                f = rng.uniform(0.9, 1.1)        # thickness scale: Cm, Cs, h ~ t; Cb ~ t^3
                sect[:, 0:9] *= f
                sect[:, 9:18] *= f ** 3
                sect[:, 18:23] *= f
                futs.append(srv.update(key, np.arange(len(sect)), sect))
                continue
            if res is not None:
                futs.append(srv.resolve(key, rng.uniform(0.5, 2.0) * res.model.load_matrix()))
                continue
        futs.append(srv.solve(pool[i]))
    results = []
    for f in futs:
        try:
            results.append(f.result())
        except KeyError:
            pass    # re-solve of a model evicted meanwhile
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    st = srv.stats()
    worst = max(float(np.max(r["rel_residual"])) for r in results)
    srv.close()
    line = {"metric": METRIC, "value": st["subcase_solves"] / wall, "unit": "solves/s", "n_gpus": 1,
            "steps": args.requests, "warmup": args.warmup, "ms_per_step": wall * 1e3 / max(1, args.requests),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == lib.PREC_FP64 else "f32+f64", "data": "synthetic",
            "config": {"workload": "serving_stream", "requests": args.requests, "rate_per_s": args.rate,
                       "mix": "70% panels / 25% wing boxes / 5% solid blocks, 30% re-solves",
                       "streams": args.slots, "precision": args.precision, "hbm_budget_gb": 150},
            "latency": {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"]},
            "completed": len(results), "subcase_solves": st["subcase_solves"], "max_rel_residual": worst}
    print(json.dumps(line), flush=True)


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "tf32x3_tflops": d["bf16_tflops"] / 2 / 3, "fp64_tflops": 40.0,
                "src": "MEASURED_PEAKS.json (measured)"}
    return {"hbm_gbs": 6650.0, "tf32x3_tflops": 1590.0 / 2 / 3, "fp64_tflops": 40.0, "src": "fallback"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--workload", default="wing_panel",
                    choices=["wing_panel", "wing_panel_small", "plate", "solid_block", "solid_block_small", "batched",
                             "serving"])
    ap.add_argument("--models", type=int, default=1024, help="batched: number of panels")
    ap.add_argument("--pack-dof", type=int, default=400000, help="batched: DOF per pack")
    ap.add_argument("--slots", type=int, default=4, help="batched/serving: device streams")
    ap.add_argument("--baseline-models", type=int, default=128, help="batched: per-model FP64 sample")
    ap.add_argument("--requests", type=int, default=160, help="serving: requests in the stream")
    ap.add_argument("--rate", type=float, default=5.0, help="serving: Poisson arrival rate (requests/s)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if "RANK" in os.environ else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batched":
        run_batched(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
