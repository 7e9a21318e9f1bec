"""SOL101 on the device behind OpenJFEM's backend plugin seam.

Mirrors ``src/backend/BackendInterface.jl`` (``AbstractJFEMBackend``,
``normalize_backend_name``, ``backend_from_model``) and the parity path
``_solve_model_parity`` -> ``_solve_sol101`` -> ``solve_case`` ->
``apply_bc_and_solve`` (src/JFEMSolver.jl:2246-2335, 2494-2587;
src/solver/boundary_conditions.jl:1324-1975; src/solver/solve_case.jl:182-303).

The host keeps the reference's host-side work -- SPC1 + AUTOSPC partition,
the post-factor pivot check and the results dictionary -- and calls the
device library for assembly, factorisation, solves and residuals.  There is
no CPU fallback: a missing library or a device error raises.
"""
from __future__ import annotations

import os
import time
from typing import Dict, Optional

import numpy as np

from . import lib
from .lib import PREC_FP64, PREC_MIXED, JfgError

BACKEND_NAMES = ("reference_parity", "tacs_formulation", "jfem_gpu")
_ALIASES = {"reference": "reference_parity", "parity": "reference_parity", "default": "reference_parity",
            "tacs": "tacs_formulation", "gpu": "jfem_gpu", "b200": "jfem_gpu", "cuda": "jfem_gpu"}


def normalize_backend_name(name) -> str:
    """BackendInterface.jl:13-37, extended with the device backend name."""
    s = str(name).strip().lower().replace("-", "_")
    s = _ALIASES.get(s, s)
    if s not in BACKEND_NAMES:
        raise ValueError(f"unknown JFEM backend {name!r}; expected one of {BACKEND_NAMES}")
    return s


def backend_from_model(model_meta: Optional[dict] = None, env=os.environ) -> str:
    """model["backend"] wins over ENV["JFEM_BACKEND"] (BackendInterface.jl:42-45)."""
    if model_meta and "backend" in model_meta:
        return normalize_backend_name(model_meta["backend"])
    return normalize_backend_name(env.get("JFEM_BACKEND", "reference_parity"))


class JFEMGPUBackend:
    """The device backend (``solve_model(::JFEMGPUBackend, model)``)."""

    name = "jfem_gpu"

    def __init__(self, device: int = 0, precision: int = PREC_FP64, tol: float = 1e-10, max_ir: int = 10,
                 hbm_budget_bytes: int = 0, post_factor_pivot_threshold: float = 1e-7, eps_zero: float = 1e-8):
        self.device = device
        self.precision = precision
        self.tol = tol
        self.max_ir = max_ir
        self.hbm_budget_bytes = hbm_budget_bytes
        self.pivot_threshold = post_factor_pivot_threshold
        self.eps_zero = eps_zero
        self._ctx = None

    @property
    def ctx(self) -> lib.Context:
        if self._ctx is None:
            self._ctx = lib.Context(self.device, self.hbm_budget_bytes)
        return self._ctx


# ----------------------------------------------------------------------------
# partition (boundary_conditions.jl:1028-1138, :745-845, :538-549)
# ----------------------------------------------------------------------------

def compute_free_dofs(model, diag: np.ndarray, node_blocks: np.ndarray, eps_zero: float = 1e-8):
    """Fixed = SPC1 u zero-diagonal AUTOSPC u grid-point singularities (GPST).

    ``node_blocks``: (n_nodes, 18) translational and rotational 3x3 blocks.
    With GPST enabled (the reference default) the diagonal pass fixes exact
    zeros only; GPST eigen-decomposes each node's free 3x3 block and fixes,
    for each eigenvalue below eps_zero * lambda_max, the free DOF the
    eigenvector lies closest to (ties to the lowest DOF).
    Returns (free ascending int32, fixed ascending int64, diagnostics).
    """
    n = model.ndof
    fixed = np.zeros(n, bool)
    spc = model.spc_dofs()
    fixed[spc] = True
    zero = (~fixed) & (diag == 0.0)
    fixed |= zero
    nn = model.n_nodes
    B = node_blocks.reshape(nn, 2, 3, 3, order="C").transpose(0, 1, 3, 2)  # [node, off, row, col]
    n_gpst = 0
    fx = fixed.reshape(nn, 2, 3)
    for off in (0, 1):
        freeblk = ~fx[:, off, :]
        full = freeblk.all(axis=1)
        idx = np.where(full)[0]
        if len(idx):
            S = 0.5 * (B[idx, off] + B[idx, off].transpose(0, 2, 1))
            # screen before the eigen-decomposition: with |l_1| >= |l_2| >=
            # |l_3| and |l_1| <= ||S||_F, |l_3| / |l_1| >= |det S| / ||S||_F^3,
            # so a block with |det S| > 10 eps ||S||_F^3 has no eigenvalue
            # below eps |l_1| and fixes nothing; only the others are decomposed
            a, b, c = S[:, 0, 0], S[:, 0, 1], S[:, 0, 2]
            d, e, f = S[:, 1, 0], S[:, 1, 1], S[:, 1, 2]
            g, h, k = S[:, 2, 0], S[:, 2, 1], S[:, 2, 2]
            det = a * (e * k - f * h) - b * (d * k - f * g) + c * (d * h - e * g)
            fro = np.sqrt(np.einsum("nij,nij->n", S, S))
            keep = ~(np.abs(det) > 10.0 * eps_zero * fro ** 3)
            idx, S = idx[keep], S[keep]
        if len(idx):
            vals, vecs = np.linalg.eigh(S)
            lam = np.abs(vals).max(axis=1)
            ratio = np.abs(vals) / np.where(lam > 0, lam, 1.0)[:, None]
            sing = (ratio < eps_zero) & (lam > 0)[:, None]
            for r in np.where(sing.any(axis=1))[0]:
                node = idx[r]
                claimed = set()
                for k in range(3):
                    if not sing[r, k]:
                        continue
                    w = np.abs(vecs[r][:, k])
                    best_a, best_w = -1, -1.0
                    for a in range(3):
                        if a in claimed:
                            continue
                        if w[a] > best_w + 1e-12:
                            best_w, best_a = w[a], a
                    if best_a < 0:
                        continue
                    claimed.add(best_a)
                    fixed[6 * node + 3 * off + best_a] = True
                    n_gpst += 1
        part = np.where(freeblk.any(axis=1) & ~full)[0]
        for node in part:
            loc = [a for a in range(3) if freeblk[node, a]]
            blk = B[node, off][np.ix_(loc, loc)]
            S = 0.5 * (blk + blk.T)
            vals, vecs = np.linalg.eigh(S)
            lam = np.abs(vals).max()
            if not lam > 0:
                continue
            claimed = set()
            for k in range(len(loc)):
                if not abs(vals[k]) / lam < eps_zero:
                    continue
                best_a, best_w = -1, -1.0
                for ii, a in enumerate(loc):
                    if a in claimed:
                        continue
                    if abs(vecs[ii, k]) > best_w + 1e-12:
                        best_w, best_a = abs(vecs[ii, k]), a
                if best_a < 0 or fixed[6 * node + 3 * off + best_a]:
                    continue
                claimed.add(best_a)
                fixed[6 * node + 3 * off + best_a] = True
                n_gpst += 1
    free = np.where(~fixed)[0].astype(np.int32)
    diagnostics = {"explicit_spc_dofs": int(len(spc)), "autospc_diagonal_zero_dofs": int(zero.sum()),
                   "autospc_gpst_dofs": int(n_gpst), "fixed_dofs": int(fixed.sum()), "free_dofs": int(len(free)),
                   "autospc_gpst_eps_zero": eps_zero}
    return free, np.where(fixed)[0], diagnostics


# ----------------------------------------------------------------------------
# solve_model
# ----------------------------------------------------------------------------

def prepare(backend: JFEMGPUBackend, model, donor: Optional["lib.DeviceModel"] = None,
            before_factor=None, dm: Optional["lib.DeviceModel"] = None, precision: Optional[int] = None) -> Dict:
    """Upload, assemble, partition, analyse and factor: the per-model state
    that the reference caches in LinearSolveCacheEntry (boundary_conditions.jl:62-75).

    ``donor``: a resident model of the same mesh whose pattern and symbolic
    analysis the new model takes over (jfg_model_share_structure).
    ``before_factor(dm)``: called once the symbolic analysis exists and before
    the factor is allocated (the serving loop admits the model's bytes there).
    ``dm``: the model already uploaded (and possibly given a donor's structure).
    ``precision``: the factor's precision when it differs from the backend's.
    """
    prec = backend.precision if precision is None else precision
    timings = {}
    t0 = time.perf_counter()
    if dm is None:
        dm = lib.DeviceModel(backend.ctx, model)
        if donor is not None:
            dm.share_structure(donor)
    dm.assemble()
    timings["assembly"] = time.perf_counter() - t0
    t1 = time.perf_counter()
    diag, max_elem = dm.diag()
    blocks = dm.node_blocks()
    free, fixed, bc = compute_free_dofs(model, diag, blocks, backend.eps_zero)
    t_sym = time.perf_counter()
    dm.set_free_dofs(free)
    timings["constraints"] = time.perf_counter() - t1
    timings["symbolic"] = time.perf_counter() - t_sym
    if before_factor is not None:
        before_factor(dm)
    t2 = time.perf_counter()
    dm.factor(prec)
    # post-factor pivot check L_ii^2 / K_ii < threshold (boundary_conditions.jl:1662-1710)
    Ld = np.abs(dm.factor_diag())
    perm = dm.perm()
    Kd = np.abs(diag[free[perm]])
    ratios = np.where(Kd > 1e-30, Ld * Ld / np.where(Kd > 1e-30, Kd, 1.0), 1.0)
    sing = np.where(ratios < backend.pivot_threshold)[0]
    bc["post_factorization_singular_dofs"] = int(len(sing))
    if len(sing):
        extra = free[perm[sing]]
        keep = np.setdiff1d(free, extra).astype(np.int32)
        dm.set_free_dofs(keep)
        free = keep
        fixed = np.union1d(fixed, extra)
        dm.factor(prec)
    timings["factorization"] = time.perf_counter() - t2
    return dict(dm=dm, free=free, fixed=fixed, bc=bc, max_elem_stiff=max_elem, timings=timings, precision=prec)


def solve_model(backend: JFEMGPUBackend, model, state: Optional[Dict] = None) -> Dict:
    """SOL101 for every subcase of ``model`` on the device; the results
    dictionary follows _solve_sol101 / _build_results_from_state."""
    if state is None:
        state = prepare(backend, model)
    dm = state["dm"]
    timings = dict(state["timings"])
    t0 = time.perf_counter()
    F = model.load_matrix()
    U, rep = dm.solve(F, backend.tol, backend.max_ir)
    timings["constraints_linear_solve"] = time.perf_counter() - t0
    t1 = time.perf_counter()
    R = dm.residual(U, F)          # K u - F  (solve_case.jl:1200)
    fixed = state["fixed"]
    spc_mask = np.zeros(model.ndof, bool)
    spc_mask[fixed] = True
    subcases = []
    for k, case in enumerate(model.load_cases):
        u = U[:, k]
        r = np.where(spc_mask, R[:, k], 0.0)
        rn = r.reshape(-1, 6)
        keep = np.linalg.norm(rn, axis=1) > 1e-20
        subcases.append({
            "sid": case.sid,
            "displacements": u.reshape(-1, 6),
            "raw_displacement": u,
            "spc_forces": {int(model.grid_ids[i]): rn[i] for i in np.where(keep)[0]},
            "fixed_dofs": fixed,
            "solver_diagnostics": {"backend": "jfem_gpu", "bc_partition": state["bc"],
                                   "linear_solver": dict(rep, strategy="direct")},
        })
    timings["static_case"] = time.perf_counter() - t1
    timings["device"] = dm.timings()
    return {"subcases": subcases, "ndof": model.ndof, "timings": timings, "state": state}
