"""SOL101 serving benchmark (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload serving|wing_panel|solid_block|plate|batched ...]

Default workload -- the serving stream: a seeded list of K x 10 requests, 70 %
stiffened panels (8-64 x 8-64 CQUAD4 skin, 0-6 blades), 25 % full-size wing-box
panels (200x400 CQUAD4 skin + 9 blades of 20x400, 914,400 free DOF), 5 %
full-size CTETRA10 blocks (40^3 hexes Kuhn-split, 1,574,640 free DOF), each
with 1-32 load cases; 30 % of the requests re-solve an earlier model with new
loads or with its thicknesses scaled U[0.9, 1.1].  The continuous-batching
server (4 device streams, 150 GB HBM budget) runs it once per arm: the mixed
arm (3xTF32 tensor-core factor + FP64 refinement to relative residual 1e-10)
and the plain FP64 arm.  A "step" is 10 requests of the stream; W warm-up
steps of another seeded list run untimed first.

value  = subcase solves/s of the mixed arm, every new model queued at once,
         with loads and displacements in device memory (CUDA tensors).
e2e    = the same stream through the server with host load matrices in and
         host displacements out (copies inside the timed region).
The line also carries the FP64 arm's figures, the mixed / FP64 ratio, p50 /
p99 latency of both arms under Poisson arrivals at half the FP64 arm's
saturated rate, the wing-box panel alone in FP64 against the CPU
restatement (with its displacement error against the FP64 oracle), and the
dominant kernel class of a full-size block (separate untimed pass).
Multi-GPU: replicas only -- every rank runs its own server on the same list;
value is the total over ranks divided by the slowest rank's time.
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


def run_reference_serving(args, rank, world):
    """Reference arm of the serving stream: the CPU restatement of the
    reference SOL101 path (oracle only, all host threads) on the same request
    list.  Each step times one full CPU SOL101 of one class sample, rotating
    panel -> wing-box panel -> 20^3 CTETRA10 block; the stream's CPU time is
    estimated per request from the class averages (re-solves pay only the
    solves, as the reference reuses its cached factor)."""
    if rank != 0:
        return
    from oracle import oracle as O  # noqa: F401  (the checker library is built on first use)
    from jf_2026_05_25_b200 import model as M
    os.environ.setdefault("JFEM_ORACLE_OPENBLAS", _openblas())
    nthreads = os.cpu_count() or 1
    n_req = args.steps * args.requests_per_step
    specs = serving_specs(n_req, seed=7)
    panels = [sp for sp in specs if sp["kind"] == "panel"] or [{"seed": 1, "nrhs": 4}]
    wing_base = M.wing_panel(n_cases=1)
    f40, l40 = 49.14e12, 4.97e9
    samples = {"panel": [], "wing": [], "solid": []}
    step_s = []
    for k in range(args.warmup + args.steps):
        cls = ("panel", "wing", "solid")[k % 3]
        t0 = time.perf_counter()
        if cls == "panel":
            sp = panels[k % len(panels)]
            m = M.stiffened_panel(sp["seed"], n_cases=sp["nrhs"])
            r = cpu_sol101(m, nthreads)
            per = (r["assembly_s"] + r["constraints_ordering_s"] + r["factor_s"], r["solve_s"] / len(m.load_cases))
        elif cls == "wing":
            r = cpu_sol101(M.wing_panel_variant(wing_base, 100 + k, 2), nthreads)
            per = (r["assembly_s"] + r["constraints_ordering_s"] + r["factor_s"], r["solve_s"] / 2)
        else:
            r = cpu_sol101(M.solid_block(n=20, n_cases=2, seed=100 + k), nthreads)
            per = (8.0 * (r["assembly_s"] + r["constraints_ordering_s"]) + f40 / r["flops"] * r["factor_s"],
                   l40 / r["nnz_L"] * r["solve_s"] / 2)
        if k >= args.warmup:
            samples[cls].append(per)
            step_s.append(time.perf_counter() - t0)
    for cls in samples:            # a class not reached by the timed steps: one extra sample
        if not samples[cls]:
            samples[cls].append({"panel": (0.05, 0.01), "wing": (10.0, 0.5), "solid": (100.0, 3.0)}[cls])
    avg = {c: tuple(float(np.mean([x[q] for x in v])) for q in (0, 1)) for c, v in samples.items()}
    total, kind_of = 0.0, {}
    for i, sp in enumerate(specs):
        kd = sp["kind"]
        if kd in ("panel", "wing", "solid"):
            kind_of[i] = kd
            total += avg[kd][0] + sp["nrhs"] * avg[kd][1]
        else:
            tk = kind_of[sp["target"]]
            total += (avg[tk][0] if kd == "update" else 0.0) + sp["nrhs"] * avg[tk][1]
    subcases = sum(sp["nrhs"] for sp in specs)
    value = subcases / total
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "serving_stream", "requests": n_req, "requests_per_step": args.requests_per_step,
                       "subcase_solves": subcases, "parallelism": "cpu", "precision": "fp64",
                       "note": "CPU restatement of the reference SOL101 path (Julia/CHOLMOD unavailable on this box)"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "port",
                             "sample": "per step one full CPU SOL101 of a class sample (stream panel / wing-box panel "
                                       "with 2 load cases / 20^3 CTETRA10 block scaled to 40^3 by factor flops and "
                                       "nnz(L)); stream time estimated per request from the class averages"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "class_seconds": avg, "measured_step_s": step_s, "stream_cpu_s_estimate": total}
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
KERNEL_CLASSES = ((0, "schur_update", "flop"), (1, "q4_element", "byte"), (2, "assembly_gather", "byte"),
                  (3, "solves", "byte"), (4, "t10_element", "byte"), (5, "f_extend_add", None),
                  (6, "f_potrf", "flop"), (7, "f_trsm", "flop"), (8, "f_panel_update", "flop"),
                  (9, "s_vec_extend_add", None), (10, "s_fwd_diag", None), (11, "s_fwd_update", None),
                  (12, "s_bwd_partial", None), (13, "s_bwd_diag", None))


def kernel_stats(L):
    """Per kernel class: launches, device ms and algorithmic units (flops or
    bytes) accumulated by the library's event brackets."""
    from jf_2026_05_25_b200 import lib
    out = {}
    for which, name, _ in KERNEL_CLASSES:
        o = np.zeros(3)
        L.jfg_get_kernel_stats(which, o.ctypes.data_as(lib.P))
        if o[0] > 0:
            out[name] = {"launches": int(o[0]), "ms": float(o[1]), "units": float(o[2])}
    return out


# DRAM bytes per tensor-core flop of the mixed factor's 3xTF32 update kernel
# (k_update_tf32x3), from one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum over all 432 launches of four factorisations of the
# 16^3 CTETRA10 block, 9.39 GB, divided by the updates' algorithmic flops,
# 4 x 1.996e11).  Scaled to a launch of the full-size block by its flops: an
# upper bound there, since larger fronts reuse their tiles more.
TC_DRAM_BYTES_PER_FLOP = 0.01176


def roofline_from_stats(stats, prec, note=""):
    """Roofline of the kernel class with the most device time among the
    classes whose algorithmic work is counted (the solve sweep is one class:
    its sub-classes overlap it).  Flop classes are set against the tensor
    peak of the factor's precision (3xTF32: measured bf16 / 2 / 3; FP64:
    the nominal 40 TFLOP/s, no FP64 measurement on this pool), byte classes
    against the measured HBM copy bandwidth."""
    from jf_2026_05_25_b200 import lib
    peaks = _peaks()
    kinds = {name: kind for _, name, kind in KERNEL_CLASSES}
    cands = {k: v for k, v in stats.items() if kinds.get(k) and v["units"] > 0 and v["ms"] > 0}
    if not cands:
        return None
    name, s = max(cands.items(), key=lambda kv: kv[1]["ms"])
    ms_launch = s["ms"] / s["launches"]
    if kinds[name] == "flop":
        achieved = s["units"] / (s["ms"] / 1000.0) / 1e12
        if prec == lib.PREC_MIXED:
            peak, src = peaks["tf32x3_tflops"], peaks["src"] + " bf16/2/3 (3xTF32)"
        else:
            peak, src = peaks["fp64_tflops"], "nominal B200 FP64 40 TFLOP/s (no measured FP64 peak)"
        roof = {"kernel": name, "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s"}
    else:
        achieved = s["units"] / (s["ms"] / 1000.0) / 1e9
        peak, src = peaks["hbm_gbs"], peaks["src"] + " hbm_gbs"
        roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s"}
    traffic = None
    if kinds[name] == "flop" and prec == lib.PREC_MIXED and name in ("schur_update", "f_panel_update"):
        traffic = TC_DRAM_BYTES_PER_FLOP * s["units"] / s["launches"]
    roof.update({"frac": achieved / peak, "traffic": traffic, "peak_source": src, "launches": s["launches"],
                 "ms_total": s["ms"], "ms_per_launch": ms_launch, "units_per_launch": s["units"] / s["launches"],
                 "traffic_source": (None if traffic is None else
                                    "bytes per flop of the 3xTF32 update kernel from an ncu capture of the 16^3 "
                                    "block (dram read + write of all its launches / their flops) x this launch's "
                                    "flops; an upper bound at full size"),
                 "pass": "separate untimed pass with the library's event brackets (graphs off)" +
                         (": " + note if note else ""),
                 "all_classes": stats})
    return roof


def run_ours(args, rank, world, local_rank, emit=True, init_dist=True):
    import torch
    import torch.distributed as dist
    from jf_2026_05_25_b200 import backend as B
    from jf_2026_05_25_b200 import lib
    torch.cuda.set_device(local_rank)
    if world > 1 and init_dist:
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
    # The library runs on its own stream and synchronises before returning, so
    # the host interval between two device synchronisations brackets exactly
    # the device work of the K steps; the torch events on the current stream
    # give the same interval on the device clock.
    ms_dev = max(e0.elapsed_time(e1), 1000.0 * t_wall)
    ms_dev = slowest_rank(ms_dev, world, "cuda")
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
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
    # ---- kernel classes in a separate untimed step with event brackets
    L.jfg_reset_kernel_stats()
    L.jfg_set_profiling(2)
    step_device()
    L.jfg_set_profiling(0)
    stats = kernel_stats(L)
    roof = roofline_from_stats(stats, prec, note=cfg["workload"])
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
                       "dof_per_s_assembled": cfg["ndof"] * value, "symbolic": sym,
                       "phase_s_last_step": dm.timings()}}
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    dm.close()
    if world > 1 and init_dist:
        dist.destroy_process_group()
    return line


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


# ---------------------------------------------------------------- serving stream (default workload)
SERVING_MIX = (("panel", 0.70), ("wing", 0.25), ("solid", 0.05))


def serving_specs(n_req: int, seed: int):
    """Seeded request list of the serving stream.  30 % of the requests
    (never the first) re-solve an earlier model of the list with new loads
    (re-solve) or, for shell models in half the cases, with its CQUAD4
    thicknesses scaled U[0.9, 1.1] (update); the new models are 70 %
    stiffened panels, 25 % full-size wing-box panels and 5 % full-size
    CTETRA10 blocks, the counts rounded to the mix (largest remainder) and
    placed in seeded random order; every request has U{1..32} load cases."""
    rng = np.random.default_rng(seed)
    n_res = int(round(0.3 * n_req)) if n_req > 1 else 0
    order = [int(x) for x in rng.permutation(np.arange(1, n_req))] if n_req > 1 else []
    resolve_at = set(order[:n_res])
    n_new = n_req - n_res
    quota = [w * n_new for _, w in SERVING_MIX]
    counts = [int(q) for q in quota]
    for k in np.argsort([-(q - int(q)) for q in quota])[:n_new - sum(counts)]:
        counts[int(k)] += 1
    kinds = [k for (k, _), c in zip(SERVING_MIX, counts) for _ in range(c)]
    kinds = [kinds[int(j)] for j in rng.permutation(len(kinds))]
    specs, new_idx = [], []
    for i in range(n_req):
        nrhs = int(rng.integers(1, 33))
        if i in resolve_at:
            j = int(new_idx[int(rng.integers(len(new_idx)))])
            upd = specs[j]["kind"] != "solid" and rng.random() < 0.5
            specs.append({"kind": "update" if upd else "resolve", "target": j, "nrhs": nrhs,
                          "scale": float(rng.uniform(0.9, 1.1)), "seed": int(seed * 100000 + i)})
            continue
        specs.append({"kind": kinds.pop(), "nrhs": nrhs, "seed": int(seed * 100000 + i)})
        new_idx.append(i)
    return specs


def _pinned(a: np.ndarray) -> np.ndarray:
    """Column-major copy of a host load matrix in page-locked memory (the
    client's input buffers of the host-buffer pass)."""
    import torch
    t = torch.empty((a.shape[1], a.shape[0]), dtype=torch.float64, pin_memory=True)
    out = t.numpy().T
    out[...] = a
    return out


class StreamModels:
    """Host models and load matrices of a request list (built before timing)."""

    def __init__(self, specs, solid_n: int = 40):
        from jf_2026_05_25_b200 import model as M
        self.M = M
        self.wing_base = None
        self.solid_n = solid_n
        self.models, self.loads, self.sections = {}, {}, {}
        for i, sp in enumerate(specs):
            if sp["kind"] in ("panel", "wing", "solid"):
                m = self._model(sp)
                self.models[i] = m
                self.loads[i] = _pinned(m.load_matrix())
        for i, sp in enumerate(specs):
            if sp["kind"] in ("resolve", "update"):
                base = self.loads[sp["target"]]
                rng = np.random.default_rng(sp["seed"])
                cols = [base[:, c % base.shape[1]] * rng.uniform(0.5, 2.0) +
                        base[:, (c + 1) % base.shape[1]] * rng.uniform(-0.5, 0.5) for c in range(sp["nrhs"])]
                self.loads[i] = _pinned(np.stack(cols, axis=1))
                if sp["kind"] == "update":
                    sect = self.models[sp["target"]].q4_sections().copy()
                    f = sp["scale"]          # thickness scale: Cm, Cs, h ~ t; Cb ~ t^3
                    sect[:, 0:9] *= f
                    sect[:, 9:18] *= f ** 3
                    sect[:, 18:23] *= f
                    self.sections[i] = sect

    def _model(self, sp):
        M = self.M
        if sp["kind"] == "panel":
            return M.stiffened_panel(sp["seed"], n_cases=sp["nrhs"])
        if sp["kind"] == "wing":
            if self.wing_base is None:
                self.wing_base = M.wing_panel(n_cases=1)
            return M.wing_panel_variant(self.wing_base, sp["seed"], sp["nrhs"])
        return M.solid_block(n=self.solid_n, n_cases=sp["nrhs"], seed=sp["seed"])


def stream_pass(srv, specs, sm: StreamModels, device: bool, rate: float = 0.0, seed: int = 0):
    """Replay a request list through the server.  rate 0: every new-model
    request is queued at once (saturation); else Poisson arrivals at `rate`
    requests/s.  A re-solve or update is submitted at its arrival once its
    target's result (and key) exists.  Returns (seconds, results in order,
    bytes host->device, bytes device->host)."""
    import threading
    from concurrent.futures import Future
    import torch
    n = len(specs)
    proxies = [Future() for _ in range(n)]
    dev_loads = {}
    if device:
        for i in range(n):
            dev_loads[i] = torch.from_numpy(np.ascontiguousarray(sm.loads[i].T)).to("cuda")
        torch.cuda.synchronize()
    gaps = np.random.default_rng(seed).exponential(1.0 / rate, size=n) if rate > 0 else np.zeros(n)
    lock = threading.Lock()

    def chain(i, fut):
        def done(f):
            exc = f.exception()
            if exc is not None:
                proxies[i].set_exception(exc)
            else:
                proxies[i].set_result(f.result())
        fut.add_done_callback(done)

    def submit(i):
        sp = specs[i]
        if sp["kind"] in ("panel", "wing", "solid"):
            if device:
                chain(i, srv.solve(sm.models[i], device_loads=dev_loads[i]))
            else:
                chain(i, srv.solve(sm.models[i], loads=sm.loads[i]))
            return
        tf = proxies[sp["target"]]
        if tf.exception() is not None:      # its model never became resident
            proxies[i].set_exception(tf.exception())
            return
        key = tf.result()["key"]
        loads = dev_loads[i] if device else sm.loads[i]
        if sp["kind"] == "resolve":
            chain(i, srv.resolve(key, loads))
        else:
            sect = sm.sections[i]
            chain(i, srv.update(key, np.arange(len(sect)), sect, loads))

    srv.latencies.clear()
    srv.kinds.clear()
    with srv.rlock:
        srv.phase_s.clear()
        srv.trace.clear()
        srv.deferred = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    target = t0
    for i, sp in enumerate(specs):
        target += gaps[i]
        now = time.perf_counter()
        if target > now:
            time.sleep(target - now)
        if sp["kind"] in ("resolve", "update"):
            tf = proxies[sp["target"]]
            if not tf.done():
                tf.add_done_callback(lambda f, i=i: submit(i))
                continue
        submit(i)
    results, failed = [], []
    for i, p in enumerate(proxies):
        try:
            results.append(p.result(timeout=3600))
        except Exception as exc:      # reported in the line, not counted as solves
            failed.append((i, f"{type(exc).__name__}: {exc}"[:200]))
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    if failed:
        print(json.dumps({"stream_failures": failed[:10], "n_failed": len(failed)}), file=sys.stderr, flush=True)
    h2d = 0 if device else int(sum(sm.loads[i].nbytes for i in range(n)))
    d2h = 0 if device else h2d
    del dev_loads
    solved = int(sum(r["U"].shape[0] if device else r["U"].shape[1] for r in results))
    return secs, results, h2d, d2h, solved, len(failed)


def run_serving(args, rank=0, world=1, local_rank=0):
    """Serving stream: the default workload.  Each arm (mixed 3xTF32 factor +
    FP64 refinement, plain FP64) runs its own server with the same request
    list; per arm: untimed warm-up requests, then the timed stream with
    device-resident loads and displacements (value), the same stream with
    host buffers (e2e), and a latency pass with Poisson arrivals at a rate
    below the FP64 arm's capacity (p50 / p99)."""
    import torch
    from jf_2026_05_25_b200 import lib
    from jf_2026_05_25_b200 import serving as S
    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local_rank))
    L = lib.load()
    n_req = args.steps * args.requests_per_step
    specs = serving_specs(n_req, seed=7)
    warm = serving_specs(max(1, args.warmup) * args.requests_per_step, seed=8)
    t_build = time.perf_counter()
    sm = StreamModels(specs)
    smw = StreamModels(warm)
    t_build = time.perf_counter() - t_build
    subcases = int(sum(sp["nrhs"] for sp in specs))
    arms = {}
    clk = None
    launches = 0
    for arm in ("fp64", "mixed"):
        prec = lib.PREC_MIXED if arm == "mixed" else lib.PREC_FP64
        srv = S.SolveServer(device=local_rank, slots=args.slots, hbm_budget_bytes=150e9, precision=prec, tol=1e-10)
        try:
            stream_pass(srv, warm, smw, device=True)
            if arm == "mixed":
                clocks = ClockSampler(local_rank)
                clocks.start()
                l0 = L.jfg_launch_count()
            secs, res, _, _, solved, nfail = stream_pass(srv, specs, sm, device=True)
            if arm == "mixed":
                launches = L.jfg_launch_count() - l0
                clk = clocks.stop()
            secs = slowest_rank(secs, world, "cuda")
            st_v = srv.stats()
            worst = max((float(np.max(r["rel_residual"])) for r in res), default=float("nan"))
            iters = [r["report"]["ir_iters"] for r in res] or [0]
            fb = sum(r["report"]["fallback_used"] for r in res)
            del res
            torch.cuda.empty_cache()
            secs_e, res_e, h2d, d2h, solved_e, nfail_e = stream_pass(srv, specs, sm, device=False)
            secs_e = slowest_rank(secs_e, world, "cuda")
            worst_e = max((float(np.max(r["rel_residual"])) for r in res_e), default=float("nan"))
            del res_e
            torch.cuda.empty_cache()
            arms[arm] = {"value": world * solved / secs, "stream_s": secs, "e2e": world * solved_e / secs_e,
                         "failed_requests": nfail + nfail_e,
                         "e2e_stream_s": secs_e, "h2d_bytes": h2d, "d2h_bytes": d2h,
                         "throughput_pass_latency": {"p50_ms": st_v["p50_ms"], "p99_ms": st_v["p99_ms"]},
                         "max_rel_residual": max(worst, worst_e), "pcg_iters_mean": float(np.mean(iters)),
                         "pcg_iters_max": int(np.max(iters)), "fallbacks": int(fb),
                         "readmissions": st_v["readmissions"], "shared_structures": st_v["shared_structures"],
                         "fp64_meshes": st_v["fp64_meshes"], "fp64_factorisations": st_v["fp64_factorisations"],
                         "deferred_same_mesh": st_v["deferred_same_mesh"],
                         "phase_s": st_v["phase_s"], "timeline": st_v["timeline"]}
            rate = args.rate if args.rate > 0 else None
            if rate is None:
                rate = 0.5 * (n_req / arms["fp64"]["stream_s"]) if "fp64" in arms else 0.5 * n_req / secs
            secs_l, _, _, _, _, nfail_l = stream_pass(srv, specs, sm, device=False, rate=rate, seed=11)
            st_l = srv.stats()
            arms[arm]["latency"] = {"rate_per_s": rate, "p50_ms": st_l["p50_ms"], "p99_ms": st_l["p99_ms"],
                                    "stream_s": secs_l, "failed_requests": nfail_l}
        finally:
            srv.close()
        torch.cuda.empty_cache()
    mixed, fp64 = arms["mixed"], arms["fp64"]
    # the wing-box panel alone in plain FP64 against the CPU restatement, with
    # the displacement error against the FP64 oracle
    wing_args = argparse.Namespace(workload="wing_panel", precision="fp64", steps=5, warmup=3, no_e2e=False,
                                   no_cpu_baseline=args.no_cpu_baseline)
    wing = run_ours(wing_args, rank, world, local_rank, emit=False, init_dist=False)
    wing.pop("metric", None)
    if wing.get("roofline"):
        wing["roofline"].pop("all_classes", None)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = serving_cpu_estimate(specs, sm, samples=1)
    line = {"metric": METRIC, "value": mixed["value"], "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * mixed["stream_s"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "serving_stream", "requests": n_req, "requests_per_step": args.requests_per_step,
                       "subcase_solves": subcases,
                       "mix": "70% stiffened panels (8-64 x 8-64 skin, 0-6 blades), 25% wing-box panels "
                              "200x400 + 9 blades 20x400 (914,400 free DOF), 5% CTETRA10 blocks 40^3 "
                              "(1,574,640 free DOF); 1-32 load cases; 30% re-solves (new loads or thickness x U[0.9,1.1])",
                       "kinds": {k: sum(1 for sp in specs if sp["kind"] == k) for k in
                                 ("panel", "wing", "solid", "resolve", "update")},
                       "slots": args.slots, "hbm_budget_gb": 150, "parallelism": f"replicas{world}",
                       "arrivals": "value and e2e: saturated (all new models queued at once); latency: Poisson",
                       "l2": "inputs larger than L2 (wing factor 2.3 GB, block factor 40 GB)",
                       "precision": "mixed arm: 3xTF32 tensor-core factor + FP64 refinement, with the FP64 (DMMA) "
                                    "factor for meshes whose refinement took more than 6 steps (thin-shell / "
                                    "drilling conditioning); fp64 arm: plain FP64"},
            "e2e": {"value": mixed["e2e"], "unit": "solves/s", "h2d_bytes_per_step": int(mixed["h2d_bytes"] / args.steps),
                    "d2h_bytes_per_step": int(mixed["d2h_bytes"] / args.steps)},
            "mixed_over_fp64": mixed["value"] / fp64["value"], "mixed_over_fp64_e2e": mixed["e2e"] / fp64["e2e"],
            "latency": {"mixed": mixed["latency"], "fp64": fp64["latency"]},
            "arms": arms, "gpu_launches": int(launches), "clocks": clk, "cpu_baseline": cpu,
            "host_build_s": t_build, "wing_panel_fp64_vs_cpu": wing}
    if args.roofline_pass:
        line["roofline"] = serving_roofline(local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def serving_cpu_estimate(specs, sm: "StreamModels", samples: int = 1):
    """CPU restatement of the reference path on a bounded sample of the
    stream, timed on the host cores (oracle only): one panel, the wing-box
    panel and a 20^3 CTETRA10 block, each a full SOL101 (assembly, partition,
    ordering, supernodal Cholesky with OpenBLAS, single-RHS solves).  The
    stream's CPU time is estimated per request from these: new models and
    updates pay assembly + factor + solves, re-solves only solves (the
    reference caches the factor); the 40^3 block's factor and solve times are
    scaled from the 20^3 one by the factor flops and nnz(L)."""
    from oracle import oracle as O
    from jf_2026_05_25_b200 import model as M
    os.environ.setdefault("JFEM_ORACLE_OPENBLAS", _openblas())
    nthreads = os.cpu_count() or 1
    t0 = time.perf_counter()
    per = {}
    pan = next(i for i, sp in enumerate(specs) if sp["kind"] == "panel") if any(
        sp["kind"] == "panel" for sp in specs) else None
    pm = sm.models[pan] if pan is not None else M.stiffened_panel(1)
    r = cpu_sol101(pm, nthreads)
    per["panel"] = (r["assembly_s"] + r["constraints_ordering_s"] + r["factor_s"], r["solve_s"] / len(pm.load_cases))
    wm = M.wing_panel_variant(sm.wing_base or M.wing_panel(n_cases=1), 1, 2)
    r = cpu_sol101(wm, nthreads)
    per["wing"] = (r["assembly_s"] + r["constraints_ordering_s"] + r["factor_s"], r["solve_s"] / 2)
    sb = M.solid_block(n=20, n_cases=2)
    r = cpu_sol101(sb, nthreads)
    f40, l40 = 49.14e12, 4.97e9            # 40^3 block, device symbolic analysis (same nested dissection)
    fs = f40 / r["flops"]
    ls = l40 / r["nnz_L"]
    per["solid"] = (8.0 * r["assembly_s"] + 8.0 * r["constraints_ordering_s"] + fs * r["factor_s"],
                    ls * r["solve_s"] / 2)
    total = 0.0
    kind_of = {}
    for i, sp in enumerate(specs):
        k = sp["kind"]
        if k in ("panel", "wing", "solid"):
            kind_of[i] = k
            total += per[k][0] + sp["nrhs"] * per[k][1]
        else:
            tk = kind_of[sp["target"]]
            total += (per[tk][0] if k == "update" else 0.0) + sp["nrhs"] * per[tk][1]
    subcases = sum(sp["nrhs"] for sp in specs)
    return {"value": subcases / total, "unit": "solves/s", "cores": nthreads, "kind": "port",
            "sample": "full CPU SOL101 of one stream panel, a wing-box panel (2 load cases) and a 20^3 CTETRA10 "
                      "block (2 load cases); stream time estimated per request, 40^3 block scaled by factor "
                      "flops / nnz(L)", "sample_s": time.perf_counter() - t0, "per_class_s": per,
            "stream_cpu_s_estimate": total}


def serving_roofline(local_rank):
    """Kernel-class statistics of one mixed-precision solve of a full-size
    CTETRA10 block (the stream's dominant class), in a separate untimed pass
    with the library's event brackets on: the dominant class and its
    achieved rate against the measured peak."""
    from jf_2026_05_25_b200 import backend as B
    from jf_2026_05_25_b200 import lib
    from jf_2026_05_25_b200 import model as M
    L = lib.load()
    m = M.solid_block(n_cases=8)
    be = B.JFEMGPUBackend(device=local_rank, precision=lib.PREC_MIXED, tol=1e-10)
    st = B.prepare(be, m)
    dm = st["dm"]
    F = m.load_matrix()
    dm.solve(F, 1e-10, 30, raise_on_stall=False)
    L.jfg_reset_kernel_stats()
    L.jfg_set_profiling(2)
    dm.assemble()
    dm.factor(lib.PREC_MIXED)
    dm.solve(F, 1e-10, 30, raise_on_stall=False)
    L.jfg_set_profiling(0)
    stats = kernel_stats(L)
    dm.close()
    return roofline_from_stats(stats, lib.PREC_MIXED, note="one full-size CTETRA10 block, mixed factor, 8 load cases")


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
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="single-model workloads only; the serving stream runs both arms")
    ap.add_argument("--workload", default="serving",
                    choices=["serving", "wing_panel", "wing_panel_small", "plate", "solid_block",
                             "solid_block_small", "batched"])
    ap.add_argument("--requests-per-step", type=int, default=10, help="serving: requests per step of the stream")
    ap.add_argument("--slots", type=int, default=4, help="batched/serving: device streams")
    ap.add_argument("--rate", type=float, default=0.0,
                    help="serving latency pass: Poisson arrival rate (0: half the FP64 arm's saturated rate)")
    ap.add_argument("--no-roofline-pass", dest="roofline_pass", action="store_false",
                    help="serving: skip the untimed kernel-class pass on a full-size block")
    ap.add_argument("--models", type=int, default=1024, help="batched: number of panels")
    ap.add_argument("--pack-dof", type=int, default=400000, help="batched: DOF per pack")
    ap.add_argument("--baseline-models", type=int, default=128, help="batched: per-model FP64 sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if "RANK" in os.environ else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.workload == "serving":
            run_reference_serving(args, rank, world)
        else:
            run_reference(args, rank, world)
        return
    if args.workload == "batched":
        run_batched(args)
        return
    if args.workload == "serving":
        run_serving(args, rank, world, local_rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
