"""The CPU oracle's own orderings and the independence of the CPU arm (CPU).

The CPU checker and the timed CPU baseline order K_ff with the oracle's
approximate-minimum-degree and nested-dissection restatements (CHOLMOD's
default rule), never with the device library's symbolic analysis.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from jf_2026_05_25_b200 import model as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _kff(oracle_mod, m):
    K = oracle_mod.csc_matrix(oracle_mod.assemble(m))
    free, _, _ = oracle_mod.partition(m, K)
    return K, free, K[free][:, free].tocsc()


@pytest.mark.parametrize("method", ["amd", "nd", "cholmod"])
@pytest.mark.parametrize("mk", [lambda: M.flat_plate(), lambda: M.stiffened_panel(3),
                                lambda: M.solid_block(n=4, n_cases=1)], ids=["plate", "panel", "solid"])
def test_orderings_are_grid_blocked_permutations(oracle_mod, mk, method):
    m = mk()
    K, free, Kff = _kff(oracle_mod, m)
    perm, info = oracle_mod.order(Kff, free, m.xyz, method)
    n = len(free)
    assert np.array_equal(np.sort(perm), np.arange(n))
    # a grid's free DOFs are eliminated consecutively, in ascending order
    g = free[perm] // 6
    starts = np.r_[True, g[1:] != g[:-1]]
    assert len(np.unique(g)) == starts.sum()
    d = free[perm]
    assert np.all(np.diff(d)[~starts[1:]] > 0)
    # far less fill than the natural order of the unknowns
    nat = oracle_mod.chol_counts(Kff, np.arange(n, dtype=np.int32))
    assert info["nnz_L"] < nat["nnz_L"]


def test_minimum_degree_on_a_path_has_no_fill(oracle_mod):
    """On a tree (here a path of grids) minimum degree eliminates leaves first:
    no fill, nnz(L) = nnz of the lower triangle."""
    n = 50
    adj = []
    for i in range(n):
        adj += [j for j in (i - 1, i + 1) if 0 <= j < n]
    ptr = np.zeros(n + 1, np.int64)
    for i in range(n):
        ptr[i + 1] = ptr[i] + (1 if i in (0, n - 1) else 2)
    adj = np.asarray(adj, np.int32)
    order = np.empty(n, np.int32)
    lib = oracle_mod.lib()
    wt = np.ones(n, np.int32)
    assert lib.or_amd_order(n, oracle_mod._p(ptr), oracle_mod._p(adj), oracle_mod._p(wt), oracle_mod._p(order)) == 0
    import scipy.sparse as sp
    A = sp.diags([np.full(n - 1, -1.0), np.full(n, 2.0), np.full(n - 1, -1.0)], [-1, 0, 1], format="csc")
    info = oracle_mod.chol_counts(A, order)
    assert info["nnz_L"] == info["nnz_A_lower"] == 2 * n - 1


def test_oracle_cholesky_with_its_own_ordering_solves(oracle_mod):
    m = M.stiffened_panel(11)
    K, free, Kff = _kff(oracle_mod, m)
    perm, _ = oracle_mod.order(Kff, free, m.xyz)
    F = oracle_mod.load_matrix(m)[free]
    U, info = oracle_mod.chol_solve(len(free), Kff.indptr.astype(np.int64), Kff.indices, Kff.data, perm, F)
    rel = np.linalg.norm(Kff @ U - F, axis=0) / np.linalg.norm(F, axis=0)
    assert rel.max() < 1e-9


def test_cpu_arm_does_not_load_the_device_library():
    """bench.py's CPU leg (the reference arm and cpu_baseline) runs the oracle
    only: after a full CPU SOL101 of the plate the process has mapped
    liboracle.so and not libjfemgpu.so."""
    code = ("import json, sys; sys.path.insert(0, %r); import bench; "
            "from jf_2026_05_25_b200 import model as M; "
            "r = bench.cpu_sol101(M.flat_plate(), 1); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'gpu': 'libjfemgpu' in maps, 'oracle': 'liboracle' in maps, 't': r['total_s']}))"
            % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["oracle"] and not res["gpu"]
