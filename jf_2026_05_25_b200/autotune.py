"""Autotuner for the factor/solve schedule of a model class.

The knobs are the host symbolic-analysis options the library reads at every
analysis (csrc/symbolic.cpp SymbolicOptions::from_env):

* ``JFG_ND_LEAF``: nested-dissection leaf size in nodes;
* ``JFG_RELAX_COLS`` / ``JFG_RELAX_ZEROS``: relaxed supernode amalgamation
  thresholds, which set front widths and so the tile shapes the factor and
  strip-solve kernels see;

the FP64 update-kernel choice (``JFG_DMMA``: tensor-core DMMA tiles or
SIMT tiles) and, for the mixed factor, the FP32 update-kernel choice
(``JFG_TENSOR_CORES``: tcgen05 3xTF32 tiles or SIMT FP32 tiles; the time
includes the refinement iterations each choice needs).  ``tune`` times symbolic analysis + numeric factor + solve of a
representative model for every candidate and returns the fastest; the
choice is cached per size class (element kind, DOF bucket) so that a serving
process tunes once per class.  The options are process-wide environment
settings, so tune before starting the serving threads.
"""
from __future__ import annotations

import itertools
import math
import os
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import backend as B
from . import lib

KNOBS = ("JFG_ND_LEAF", "JFG_RELAX_COLS", "JFG_RELAX_ZEROS", "JFG_DMMA", "JFG_TENSOR_CORES")

DEFAULT_CANDIDATES: List[Dict[str, str]] = [
    {"JFG_ND_LEAF": leaf, "JFG_RELAX_COLS": cols, "JFG_RELAX_ZEROS": zeros, "JFG_DMMA": dmma}
    for leaf, (cols, zeros), dmma in itertools.product(
        ("16", "24", "48"),
        (("24,64,192", "0.6,0.15,0.05"), ("16,48,128", "0.5,0.1,0.03"), ("32,96,256", "0.7,0.2,0.08")),
        ("1", "0"))
]

_cache: Dict[tuple, Dict[str, str]] = {}


def size_class(model) -> tuple:
    kind = "q4" if len(model.q4_nodes) else ("t10" if len(model.t10_nodes) else "q8")
    return kind, int(math.log2(max(model.ndof, 2)))


def apply(options: Dict[str, str]):
    """Set the knobs for the analyses and factorisations that follow."""
    for k in KNOBS:
        if k in options:
            os.environ[k] = str(options[k])
        else:
            os.environ.pop(k, None)


def candidate_list(precision: int, candidates: Optional[Sequence[Dict[str, str]]] = None) -> List[Dict[str, str]]:
    """The schedules `tune` times: the given ones, or the default grid; for the
    mixed factor the default grid is doubled with the FP32 update choice
    (tensor cores on / off)."""
    cands = [dict(c) for c in (candidates or DEFAULT_CANDIDATES)]
    if candidates is None and precision == lib.PREC_MIXED:
        cands = [dict(c, JFG_TENSOR_CORES=t) for c in cands for t in ("1", "0")]
    return cands


def tune(model, candidates: Optional[Sequence[Dict[str, str]]] = None, repeats: int = 2,
         ctx: Optional[lib.Context] = None, precision: int = lib.PREC_FP64) -> Dict:
    """Time every candidate on `model`; returns dict(best, timings) and caches
    the best options for the model's size class."""
    cands = candidate_list(precision, candidates)
    saved = {k: os.environ.get(k) for k in KNOBS}
    own_ctx = ctx is None
    ctx = ctx or lib.Context(0)
    timings = []
    try:
        be = B.JFEMGPUBackend(precision=precision)
        be._ctx = ctx
        dm = lib.DeviceModel(ctx, model)
        dm.assemble()
        diag, _ = dm.diag()
        free, _, _ = B.compute_free_dofs(model, diag, dm.node_blocks(), be.eps_zero)
        F = model.load_matrix()
        for opt in cands:
            apply(opt)
            best = math.inf
            for _ in range(repeats):
                t0 = time.perf_counter()
                dm.set_free_dofs(free)
                dm.factor(precision)
                dm.solve(F, 1e-10, 30, raise_on_stall=False)
                best = min(best, time.perf_counter() - t0)
            timings.append((best, opt))
        dm.close()
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        if own_ctx:
            ctx.close()
    timings.sort(key=lambda x: x[0])
    best = dict(timings[0][1])
    _cache[size_class(model)] = best
    return {"best": best, "seconds": timings[0][0],
            "timings": [{"seconds": t, **o} for t, o in timings]}


def tuned_options(model) -> Optional[Dict[str, str]]:
    """Cached best options for the model's size class, if tuned."""
    return _cache.get(size_class(model))
