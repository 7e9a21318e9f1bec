"""Python side of the CPU oracle (test infrastructure, not product code).

Restates OpenJFEM's SOL101 host-side partition (SPC1 + AUTOSPC) in numpy and
wraps the C++ element/assembly restatement in ``oracle_fem.cpp``.  Only the
tests, the smoke check and the CPU-baseline leg of ``bench.py`` use this
module, always as the checker of the CUDA library, never as a product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile oracle_fem.cpp + oracle_chol.cpp into _build/liboracle.so."""
    srcs = [os.path.join(HERE, f) for f in ("oracle_fem.cpp", "oracle_chol.cpp", "oracle_order.cpp")]
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    if not force and os.path.exists(LIB_PATH):
        lib_m = os.path.getmtime(LIB_PATH)
        if all(os.path.getmtime(s) <= lib_m for s in srcs):
            return LIB_PATH
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-o", LIB_PATH] + srcs + ["-ldl"]
    subprocess.check_call(cmd)
    return LIB_PATH


def _default_openblas():
    """SciPy's bundled OpenBLAS (the checker's dense kernels), if present."""
    import glob
    try:
        import scipy
    except ImportError:
        return None
    c = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "libscipy_openblas-*.so"))
    return os.path.abspath(c[0]) if c else None


def lib():
    global _lib
    if _lib is None:
        if "JFEM_ORACLE_OPENBLAS" not in os.environ and _default_openblas():
            os.environ["JFEM_ORACLE_OPENBLAS"] = _default_openblas()
        build()
        L = ctypes.CDLL(LIB_PATH)
        d, i32, i64 = ctypes.c_double, ctypes.c_int32, ctypes.c_int64
        P = ctypes.c_void_p
        L.or_q4_local.argtypes = [P, P, P, P, d, d, d, P]
        L.or_q4_element.argtypes = [P, P, P, P]
        L.or_q8_element.argtypes = [P, P, P, P]
        L.or_q8_parallelogram.argtypes = [P]
        L.or_t10_element.argtypes = [P, P, d, d, P]
        L.or_assemble_triplets.argtypes = [i64, P, P, i64, P, P, i64, P, P, i64, P, P, i64, P, P, i64, P, P,
                                           P, P]
        L.or_tria3_guard.argtypes = [P, d, d, d, d, d]
        L.or_tria3_guard.restype = i32
        L.or_tria3_local.argtypes = [P, P, P, P, d, P]
        L.or_t3_element.argtypes = [P, P, P, P]
        L.or_assemble_triplets.restype = i64
        L.or_build_csc.argtypes = [i64, i64, P, P, P, P, P, P, P]
        L.or_build_csc.restype = i64
        L.or_csc_matvec.argtypes = [i64, P, P, P, i32, P, P]
        for name in ("or_q4_local", "or_q4_element", "or_q8_element", "or_q8_parallelogram", "or_t10_element",
                     "or_tria3_local", "or_t3_element"):
            getattr(L, name).restype = ctypes.c_int
        L.or_chol_factor_solve.argtypes = [i64, P, P, P, P, i32, P, P, i32, P]
        L.or_chol_factor_solve.restype = ctypes.c_int
        L.or_chol_factor.argtypes = [i64, P, P, P, P, i32, ctypes.POINTER(P)]
        L.or_chol_factor.restype = ctypes.c_int
        L.or_chol_solve.argtypes = [P, i32, P, P]
        L.or_chol_solve.restype = ctypes.c_int
        L.or_chol_free.argtypes = [P]
        L.or_chol_free.restype = None
        L.or_t10_stress.argtypes = [P, P, d, d, P, P]
        L.or_t10_stress.restype = ctypes.c_int
        L.or_q4_stress.argtypes = [P, P, d, d, d, d, P, P, P]
        L.or_q4_stress.restype = ctypes.c_int
        L.or_csc_residual_dd.argtypes = [i64, i64, P, P, P, i32, P, P, P]
        L.or_csc_residual_dd.restype = None
        L.or_chol_counts.argtypes = [i64, P, P, P, P]
        L.or_chol_counts.restype = ctypes.c_int
        L.or_amd_order.argtypes = [i32, P, P, P, P]
        L.or_amd_order.restype = ctypes.c_int
        L.or_nd_order.argtypes = [i32, P, P, P, P, i32, P]
        L.or_nd_order.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def q4_local(lc, Cm, Cb, Cs, h, k6rot, drill_scale=1.0):
    lc = np.asfortranarray(lc, dtype=np.float64)
    Ke = np.zeros((24, 24), order="F")
    st = lib().or_q4_local(_p(lc), _p(np.asfortranarray(Cm, float)), _p(np.asfortranarray(Cb, float)),
                           _p(np.asfortranarray(Cs, float)), float(h), float(k6rot), float(drill_scale), _p(Ke))
    if st:
        raise ValueError(f"or_q4_local status {st}")
    return Ke


def _ident_R(n):
    R = np.zeros((n, 9)); R[:, 0] = R[:, 4] = R[:, 8] = 1.0
    return R


def q4_element(xyz, sect, nodeR=None):
    xyz = np.ascontiguousarray(xyz, float)
    R = np.ascontiguousarray(_ident_R(4) if nodeR is None else nodeR, float)
    Ke = np.zeros((24, 24), order="F")
    st = lib().or_q4_element(_p(xyz), _p(R), _p(np.ascontiguousarray(sect, float)), _p(Ke))
    if st:
        raise ValueError(f"or_q4_element status {st}")
    return Ke


def q8_element(xyz, sect, nodeR=None):
    xyz = np.ascontiguousarray(xyz, float)
    R = np.ascontiguousarray(_ident_R(8) if nodeR is None else nodeR, float)
    Ke = np.zeros((48, 48), order="F")
    st = lib().or_q8_element(_p(xyz), _p(R), _p(np.ascontiguousarray(sect, float)), _p(Ke))
    if st:
        raise ValueError(f"or_q8_element status {st}")
    return Ke


def tria3_guard(Zb, La, Lb, c, s, Dnormal):
    """FEMKernels.jl:9281-9313 on a copy of Zb: (changed, Zb).  Raises where
    the reference raises (non-positive residual normal flexibility)."""
    Z = np.asfortranarray(np.array(Zb, float))
    st = lib().or_tria3_guard(_p(Z), float(La), float(Lb), float(c), float(s), float(Dnormal))
    if st < 0:
        raise ValueError("Triangle residual normal flexibility must be positive")
    return bool(st), Z


def tria3_local(coords, Dm, Db, Ds, k6rot=100.0):
    """18 x 18 local CTRIA3 stiffness (FEMKernels.jl:9375-9809, default path)."""
    X = np.asfortranarray(np.asarray(coords, float).reshape(3, 2))
    Ke = np.zeros((18, 18), order="F")
    st = lib().or_tria3_local(_p(X), _p(np.asfortranarray(Dm, float)), _p(np.asfortranarray(Db, float)),
                              _p(np.asfortranarray(Ds, float)), float(k6rot), _p(Ke))
    if st:
        raise ValueError(f"or_tria3_local status {st}")
    return Ke


def t3_element(xyz, sect, nodeR=None):
    xyz = np.ascontiguousarray(xyz, float)
    R = np.ascontiguousarray(_ident_R(3) if nodeR is None else nodeR, float)
    Ke = np.zeros((18, 18), order="F")
    st = lib().or_t3_element(_p(xyz), _p(R), _p(np.ascontiguousarray(sect, float)), _p(Ke))
    if st:
        raise ValueError(f"or_t3_element status {st}")
    return Ke


# the six CTRIA3 that replace a CQUAD8 without the native eight-node section
# (assembly.jl:3176-3196): [1,5,8] [5,2,6] [6,3,7] [7,4,8] [5,6,8] [6,7,8]
_Q8_SPLIT = ((0, 4, 7), (4, 1, 5), (5, 2, 6), (6, 3, 7), (4, 5, 7), (5, 6, 7))


def shells_as_assembled(model):
    """(native CQUAD8 nodes, their sections, CTRIA3 nodes, their sections): a
    CQUAD8 keeps the native stiffness when quad8_shell_parallelogram holds
    (quad8_shell.jl:34-46, or_q8_parallelogram), else it becomes six CTRIA3
    with its PSHELL section, appended after the model's own triangles."""
    L = lib()
    X = np.asarray(model.xyz, float)
    q8n = np.asarray(model.q8_nodes, np.int32).reshape(-1, 8)
    q8s = np.asarray(model.q8_sections(), float).reshape(-1, 22)
    keep = np.array([L.or_q8_parallelogram(_p(np.ascontiguousarray(X[nd]))) != 0 for nd in q8n], bool)
    split = np.where(~keep)[0]
    nodes = [np.asarray(getattr(model, "t3_nodes", np.zeros((0, 3))), np.int32).reshape(-1, 3)]
    pids = [np.asarray(getattr(model, "t3_pid", np.zeros(0)), np.int64)]
    if len(split):
        nodes.append(np.array([[q8n[e][k] for k in tri] for e in split for tri in _Q8_SPLIT], np.int32))
        pids.append(np.repeat(np.asarray(model.q8_pid, np.int64)[split], 6))
    pid = np.concatenate(pids)
    recs = np.zeros((len(pid), 26))
    for q in np.unique(pid):
        recs[pid == q] = _t3_record(model, int(q))
    return (np.ascontiguousarray(q8n[keep]), np.ascontiguousarray(q8s[keep]),
            np.ascontiguousarray(np.vstack(nodes)), recs)


def _t3_record(model, pid: int) -> np.ndarray:
    """CTRIA3 section record of an isotropic PSHELL (assembly.jl:3375-3461 with
    n = 3): Cm = E h / (1 - nu^2) [1 nu 0; nu 1 0; 0 0 (1-nu)/2] of MID1; Cb
    the same law of MID2 (MID1 when blank) times 12I/T^3 h^3 / 12; Cs =
    TS/T h G I2 of MID3 (MID1 when blank), G derived as E / 2(1 + nu) when
    blank; Cb = Cs = 0 and K6ROT 0 for a membrane-only shell (12I/T^3 <= 1e-12);
    Eref = that G; flags 0."""
    p = model.pshells[pid]
    h, br, tst = float(p.T), float(p.BEND_RATIO), float(p.TS_T)

    def law(mat):
        E, nu = float(mat.E), float(mat.NU)
        return E / (1 - nu * nu) * np.array([[1.0, nu, 0.0], [nu, 1.0, 0.0], [0.0, 0.0, (1 - nu) / 2]])
    m1 = model.mats[p.MID1]
    Cm = h * law(m1)
    Cb = np.zeros((3, 3))
    Cs = np.zeros((2, 2))
    sm = model.mats[p.MID3] if p.MID3 != 0 else m1
    G = float(sm.G) if float(sm.G) > 0 else (float(sm.E) / (2 * (1 + float(sm.NU))) if float(sm.E) > 0 else 0.0)
    if br > 1e-12:
        Cb = (br * h ** 3 / 12.0) * law(model.mats[p.MID2] if p.MID2 != 0 else m1)
        Cs = tst * h * G * np.eye(2)
    rec = np.zeros(26)
    rec[0:9] = Cm.ravel(order="F")
    rec[9:18] = Cb.ravel(order="F")
    rec[18:22] = Cs.ravel(order="F")
    rec[22] = h
    rec[23] = G
    rec[24] = 0.0 if br <= 1e-12 else float(model.k6rot)
    return rec


def t10_element(xyz, E, nu, nodeR=None):
    xyz = np.ascontiguousarray(xyz, float)
    R = np.ascontiguousarray(_ident_R(10) if nodeR is None else nodeR, float)
    Ke = np.zeros((30, 30), order="F")
    st = lib().or_t10_element(_p(xyz), _p(R), float(E), float(nu), _p(Ke))
    if st:
        raise ValueError(f"or_t10_element status {st}")
    return Ke


def t10_stresses(model, U) -> np.ndarray:
    """Centroid stress / strain / von Mises of every CTETRA10 for every column
    of U (ndof x nrhs): array (nrhs, n_t10, 13) = sxx syy szz txy tyz tzx,
    exx eyy ezz gxy gyz gzx, von Mises (stress_recovery.jl:1823-1960)."""
    U = np.asarray(U, float)
    if U.ndim == 1:
        U = U[:, None]
    L = lib()
    nodes = np.asarray(model.t10_nodes)
    mat = model.t10_materials()
    R = np.asarray(model.node_R, float)
    X = np.asarray(model.xyz, float)
    out = np.zeros((U.shape[1], len(nodes), 13))
    rec = np.zeros(13)
    for k in range(U.shape[1]):
        un = U[:, k].reshape(-1, 6)[:, :3]
        for e in range(len(nodes)):
            nd = nodes[e]
            st = L.or_t10_stress(_p(np.ascontiguousarray(X[nd])), _p(np.ascontiguousarray(R[nd])),
                                 float(mat[e, 0]), float(mat[e, 1]), _p(np.ascontiguousarray(un[nd])), _p(rec))
            if st:
                raise ValueError(f"element {e}: or_t10_stress status {st}")
            out[k, e] = rec
    return out


Q4_STRESS_REC = 31


def q4_stresses(model, U) -> np.ndarray:
    """CQUAD4 centre forces, fibre stresses and strains of every element for
    every column of U (ndof x nrhs): array (nrhs, n_q4, 31) in the layout of
    or_q4_stress (recover_shell_stresses!, stress_recovery.jl:505-1237, the
    default isotropic PSHELL path)."""
    U = np.asarray(U, float)
    if U.ndim == 1:
        U = U[:, None]
    L = lib()
    nodes = np.asarray(model.q4_nodes)
    sect = model.q4_sections()
    R = np.asarray(model.node_R, float)
    X = np.asarray(model.xyz, float)
    out = np.zeros((U.shape[1], len(nodes), Q4_STRESS_REC))
    rec = np.zeros(Q4_STRESS_REC)
    for e in range(len(nodes)):
        p = model.pshells[int(model.q4_pid[e])]
        mat = model.mats[p.MID1]
        nd = nodes[e]
        Xe, Re = np.ascontiguousarray(X[nd]), np.ascontiguousarray(R[nd])
        se = np.ascontiguousarray(sect[e])
        for k in range(U.shape[1]):
            ue = np.ascontiguousarray(U[:, k].reshape(-1, 6)[nd].ravel())
            st = L.or_q4_stress(_p(Xe), _p(Re), float(mat.E), float(mat.NU), float(p.T), float(p.BEND_RATIO),
                                _p(se), _p(ue), _p(rec))
            if st:
                raise ValueError(f"element {e}: or_q4_stress status {st}")
            out[k, e] = rec
    return out


def assemble(model):
    """Triplets in reference order and Julia's sparse() CSC + slot map."""
    L = lib()
    xyz = np.ascontiguousarray(model.xyz, float)
    R = np.ascontiguousarray(model.node_R, float)
    q4n = np.ascontiguousarray(model.q4_nodes, np.int32)
    q4s = np.ascontiguousarray(model.q4_sections())
    q8n, q8s, t3n, t3s = shells_as_assembled(model)
    t10n = np.ascontiguousarray(model.t10_nodes, np.int32)
    t10m = np.ascontiguousarray(model.t10_materials())
    cap = 576 * len(q4n) + 324 * len(t3n) + 900 * len(t10n) + 2304 * len(q8n)
    I = np.empty(cap, np.int64); J = np.empty(cap, np.int64); V = np.empty(cap)
    err = np.full(1, -1, np.int32)
    nt = L.or_assemble_triplets(model.n_nodes, _p(xyz), _p(R), len(q4n), _p(q4n), _p(q4s),
                                len(t3n), _p(t3n), _p(t3s),
                                len(q8n), _p(q8n), _p(q8s), len(t10n), _p(t10n), _p(t10m),
                                cap, _p(I), _p(J), _p(V), _p(err))
    if nt < 0:
        raise ValueError(f"element {err[0]} failed with status {-nt}")
    I, J, V = I[:nt], J[:nt], V[:nt]
    n = model.ndof
    colptr = np.empty(n + 1, np.int64)
    rowval = np.empty(nt, np.int32)
    nzval = np.empty(nt)
    slot = np.empty(nt, np.int64)
    nnz = L.or_build_csc(n, nt, _p(I), _p(J), _p(V), _p(colptr), _p(rowval), _p(nzval), _p(slot))
    return dict(colptr=colptr, rowval=rowval[:nnz].copy(), nzval=nzval[:nnz].copy(), slot=slot,
                I=I, J=J, V=V, ndof=n)


def csc_matrix(asm):
    import scipy.sparse as sp
    n = asm["ndof"]
    return sp.csc_matrix((asm["nzval"], asm["rowval"], asm["colptr"]), shape=(n, n))


# ----------------------------------------------------------------------------
# Partition (boundary_conditions.jl:1028-1138 diagonal AUTOSPC, :745-845 GPST)
# ----------------------------------------------------------------------------

def node_blocks(K, n_nodes: int) -> np.ndarray:
    """(n_nodes, 2, 3, 3): every grid's translational and rotational 3x3
    diagonal blocks of K (row, column)."""
    Kc = K.tocsc()
    out = np.zeros((n_nodes, 2, 3, 3))
    base = 6 * np.arange(n_nodes)
    for off in (0, 1):
        for a in range(3):
            for b in range(3):
                out[:, off, a, b] = np.asarray(Kc[base + 3 * off + a, base + 3 * off + b]).ravel()
    return out


def _gpst_claim(vals, vecs, loc, eps_zero):
    """The DOFs (positions in loc) that the singular eigenvalues of one block
    fix: each eigenvalue below eps_zero * max|eigenvalue| claims the unclaimed
    DOF its eigenvector lies closest to (ties to the lowest DOF)."""
    lam = np.max(np.abs(vals))
    if not lam > 0:
        return []
    claimed = []
    for k in range(len(loc)):
        if not abs(vals[k]) / lam < eps_zero:
            continue
        best_a, best_w = -1, -1.0
        for ii in range(len(loc)):
            if ii in claimed:
                continue
            w = abs(vecs[ii, k])
            if w > best_w + 1e-12:
                best_w, best_a = w, ii
        if best_a >= 0:
            claimed.append(best_a)
    return claimed


def partition(model, K, eps_zero: float = 1e-8) -> Tuple[np.ndarray, np.ndarray, dict]:
    """Fixed set = SPC1 u zero-diagonal AUTOSPC u grid-point singularities.

    With grid-point-singularity processing on (the reference default) the
    diagonal pass fixes exact zeros only (boundary_conditions.jl:1028-1138);
    GPST then eigen-decomposes every grid's free 3x3 translational /
    rotational block and fixes the DOF the eigenvector of each eigenvalue
    below eps_zero * lambda_max lies closest to (:745-845).  Full blocks are
    decomposed in one batched call, partly fixed ones one by one.
    Returns (free_dofs ascending, fixed_dofs ascending, diagnostics).
    """
    n = model.ndof
    nn = n // 6
    fixed = np.zeros(n, bool)
    fixed[model.spc_dofs()] = True
    diag = np.asarray(K.diagonal()).copy()
    zero = (~fixed) & (diag == 0.0)
    fixed |= zero
    blocks = node_blocks(K, nn)
    fx = fixed.reshape(nn, 2, 3).copy()
    n_gpst = 0
    for off in (0, 1):
        free_blk = ~fx[:, off, :]
        full = np.where(free_blk.all(axis=1))[0]
        if len(full):
            S = blocks[full, off]
            vals, vecs = np.linalg.eigh(0.5 * (S + S.transpose(0, 2, 1)))
            lam = np.abs(vals).max(axis=1)
            sing = ((np.abs(vals) / np.where(lam > 0, lam, 1.0)[:, None]) < eps_zero) & (lam > 0)[:, None]
            for r in np.where(sing.any(axis=1))[0]:
                for a in _gpst_claim(vals[r], vecs[r], [0, 1, 2], eps_zero):
                    fixed[6 * full[r] + 3 * off + a] = True
                    n_gpst += 1
        for node in np.where(free_blk.any(axis=1) & ~free_blk.all(axis=1))[0]:
            loc = [a for a in range(3) if free_blk[node, a]]
            blk = blocks[node, off][np.ix_(loc, loc)]
            vals, vecs = np.linalg.eigh(0.5 * (blk + blk.T))
            for ii in _gpst_claim(vals, vecs, loc, eps_zero):
                g = 6 * node + 3 * off + loc[ii]
                if not fixed[g]:
                    fixed[g] = True
                    n_gpst += 1
    free = np.where(~fixed)[0].astype(np.int32)
    return free, np.where(fixed)[0], {"autospc_zero": int(zero.sum()), "autospc_gpst": n_gpst}


# ----------------------------------------------------------------------------
# Fill-reducing ordering of K_ff (what CHOLMOD chooses inside cholesky())
# ----------------------------------------------------------------------------

def grid_graph(Kff, free: np.ndarray):
    """Grid-point graph of K_ff: one vertex per grid with free DOFs (weight =
    its free DOFs), an edge where two grids share a nonzero block.
    Returns (ptr, adj, weights, grid of each vertex, vertex of each free DOF)."""
    free = np.asarray(free, np.int64)
    grid = free // 6
    ugrid, vert_of = np.unique(grid, return_inverse=True)
    Kc = Kff.tocsc()
    cols = np.repeat(np.arange(Kc.shape[1]), np.diff(Kc.indptr))
    a = vert_of[Kc.indices].astype(np.int64)
    b = vert_of[cols].astype(np.int64)
    keep = a != b
    nv = len(ugrid)
    code = np.unique(a[keep] * nv + b[keep])
    src, dst = code // nv, code % nv
    both = np.unique(np.concatenate([src * nv + dst, dst * nv + src]))
    src, dst = both // nv, both % nv
    ptr = np.zeros(nv + 1, np.int64)
    np.add.at(ptr, src + 1, 1)
    ptr = np.cumsum(ptr)
    wt = np.bincount(vert_of, minlength=nv).astype(np.int32)
    return ptr, dst.astype(np.int32), wt, ugrid, vert_of


def chol_counts(Kff, perm) -> dict:
    """nnz(L) and flops (sum of squared column counts) of Symmetric(K_ff) in order perm."""
    Kc = Kff.tocsc()
    info = np.zeros(3)
    st = lib().or_chol_counts(Kc.shape[0], _p(np.ascontiguousarray(Kc.indptr, np.int64)),
                              _p(np.ascontiguousarray(Kc.indices, np.int32)),
                              _p(np.ascontiguousarray(perm, np.int32)), _p(info))
    if st != 0:
        raise ValueError("bad permutation")
    return {"nnz_L": float(info[0]), "flops": float(info[1]), "nnz_A_lower": float(info[2])}


def order(Kff, free, xyz, method: str = "cholmod", leaf: int = 64):
    """Elimination order of K_ff's unknowns: perm[k] = position in `free` of
    the k-th eliminated unknown (a grid's DOFs stay together, ascending).

    method "amd": approximate minimum degree; "nd": nested dissection by
    coordinate bisection; "cholmod": CHOLMOD's default rule -- take AMD, and
    when its factor is poor (nnz(L) >= 5 nnz(A) and flops >= 500 nnz(L)) also
    try nested dissection and keep the ordering with the fewer nonzeros in L.
    Returns (perm, info dict with the method used, nnz_L and flops).
    """
    L = lib()
    ptr, adj, wt, ugrid, vert_of = grid_graph(Kff, free)
    nv = len(ugrid)

    def expand(vorder):
        rank = np.empty(nv, np.int64)
        rank[vorder] = np.arange(nv)
        # DOFs by their grid's rank, ascending DOF within a grid
        return np.lexsort((np.arange(len(free)), rank[vert_of])).astype(np.int32)

    def run(m):
        vo = np.empty(nv, np.int32)
        if m == "amd":
            st = L.or_amd_order(nv, _p(ptr), _p(adj), _p(wt), _p(vo))
        else:
            X = np.ascontiguousarray(np.asarray(xyz, float)[ugrid])
            st = L.or_nd_order(nv, _p(ptr), _p(adj), _p(wt), _p(X), int(leaf), _p(vo))
        if st != 0:
            raise RuntimeError(f"oracle ordering {m} failed")
        perm = expand(vo)
        info = chol_counts(Kff, perm)
        info["method"] = m
        return perm, info

    if method in ("amd", "nd"):
        return run(method)
    perm, info = run("amd")
    if info["nnz_L"] >= 5 * info["nnz_A_lower"] and info["flops"] >= 500 * info["nnz_L"]:
        perm2, info2 = run("nd")
        if info2["nnz_L"] < info["nnz_L"]:
            return perm2, info2
    return perm, info


# ----------------------------------------------------------------------------
# Applied loads (loads.jl:497-586 resolve_loads, solve_case.jl:57-91)
# ----------------------------------------------------------------------------

def load_vector(model, case) -> np.ndarray:
    """Global force vector of one subcase, restated from the reference.

    PLOAD4 on a 4-node shell (loads.jl:546-585): the face normal is
    (x3 - x1) x (x4 - x2), area = |normal| / 2, and each of the 4 nodes gets
    area * p / 4 along the unit normal (no nodal moments); on a 3-node shell
    the normal is (x2 - x1) x (x3 - x1) and each node gets area * p / 3.  FORCE and the
    consistent C3D10 face loads (delivered as nodal forces, abaqus_input.jl:
    347-405) add their vectors to the translational DOFs.  The accumulated
    global vector is then expressed in each node's displacement frame,
    F_node = node_R' * F_global, per 3-block (solve_case.jl:78-82).
    """
    n_nodes = model.n_nodes
    acc = np.zeros((n_nodes, 6))
    X = np.asarray(model.xyz, float)
    if case.pload4 is not None:
        eidx, pres = case.pload4
        q4 = np.asarray(model.q4_nodes)[np.asarray(eidx)]
        a = X[q4[:, 2]] - X[q4[:, 0]]
        b = X[q4[:, 3]] - X[q4[:, 1]]
        nx = a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1]
        ny = a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2]
        nz = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
        nrm = np.sqrt(nx * nx + ny * ny + nz * nz)
        ok = 0.5 * nrm > 1e-30
        share = np.where(ok, 0.5 * nrm * np.asarray(pres, float) / 4.0, 0.0)
        unit = np.stack([nx, ny, nz], axis=1) / np.where(nrm > 0, nrm, 1.0)[:, None]
        fnode = unit * share[:, None]
        for k in range(4):
            for c in range(3):
                acc[:, c] += np.bincount(q4[:, k], weights=fnode[:, c], minlength=n_nodes)
    if getattr(case, "pload4_t3", None) is not None:
        # PLOAD4 on a 3-node shell: normal (x2 - x1) x (x3 - x1), p A / 3 per node
        eidx, pres = case.pload4_t3
        t3 = np.asarray(model.t3_nodes)[np.asarray(eidx)]
        a = X[t3[:, 1]] - X[t3[:, 0]]
        b = X[t3[:, 2]] - X[t3[:, 0]]
        nv = np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                       a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)
        nrm = np.sqrt((nv * nv).sum(axis=1))
        share = np.where(0.5 * nrm > 1e-30, 0.5 * nrm * np.asarray(pres, float) / 3.0, 0.0)
        fnode = nv / np.where(nrm > 0, nrm, 1.0)[:, None] * share[:, None]
        for k in range(3):
            for c in range(3):
                acc[:, c] += np.bincount(t3[:, k], weights=fnode[:, c], minlength=n_nodes)
    for item in (case.forces, case.cload):
        if item is None:
            continue
        nidx, vec = item
        for c in range(3):
            acc[:, c] += np.bincount(np.asarray(nidx), weights=np.asarray(vec, float)[:, c], minlength=n_nodes)
    R = np.asarray(model.node_R, float).reshape(n_nodes, 3, 3, order="C")   # R[n, col, row]
    out = np.empty_like(acc)
    for blk in (0, 3):
        g = acc[:, blk:blk + 3]
        # (node_R' g)_j = sum_i node_R[i, j] g_i, node_R column-major: R[n, j, i] = node_R[i, j]
        out[:, blk:blk + 3] = np.einsum("nji,ni->nj", R, g)
    return out.reshape(-1)


def load_matrix(model) -> np.ndarray:
    """ndof x nsubcases (column-major) of every subcase's force vector."""
    return np.asfortranarray(np.stack([load_vector(model, c) for c in model.load_cases], axis=1))


def solve_reference(model, asm=None, free=None):
    """FP64 SOL101 on the CPU with SciPy's SuperLU (independent small-case checker).

    Returns dict(u (ndof x nrhs), F, R = K u - F, free, rel_residual).
    """
    import scipy.sparse.linalg as spla
    if asm is None:
        asm = assemble(model)
    K = csc_matrix(asm)
    if free is None:
        free, _, _ = partition(model, K)
    F = load_matrix(model)
    Kff = K[free][:, free].tocsc()
    # Symmetric(K_ff) (upper triangle) is what the reference factorises
    import scipy.sparse as sp
    U = sp.triu(Kff, format="csc")
    A = (U + sp.triu(U, k=1, format="csc").T).tocsc()
    lu = spla.splu(A, permc_spec="MMD_AT_PLUS_A")
    Fff = np.asfortranarray(F[free])
    u_ff = lu.solve(Fff)
    # FP64 iterative refinement on the assembled K_ff: makes the checker
    # accurate to rounding even for ill-conditioned shell models
    for _ in range(6):
        r = Fff - Kff @ u_ff
        if np.all(np.linalg.norm(r, axis=0) <= 1e-15 * np.maximum(np.linalg.norm(Fff, axis=0), 1e-300)):
            break
        u_ff = u_ff + lu.solve(np.asfortranarray(r))
    u = np.zeros_like(F)
    u[free] = u_ff
    R = K @ u - F
    rel = np.linalg.norm(Kff @ u_ff - F[free], axis=0) / np.maximum(np.linalg.norm(F[free], axis=0), 1e-300)
    return dict(u=u, F=F, R=R, free=free, rel_residual=rel, asm=asm)


def residual_dd(A, x, f) -> np.ndarray:
    """f - A x, accumulated per row in double-double (compensated) arithmetic."""
    A = A.tocsc()
    x = np.asfortranarray(x, np.float64)
    f = np.asfortranarray(f, np.float64)
    if x.ndim == 1:
        x, f = x[:, None], f[:, None]
    r = np.zeros_like(f, order="F")
    lib().or_csc_residual_dd(A.shape[0], A.shape[1], _p(np.ascontiguousarray(A.indptr, np.int64)),
                             _p(np.ascontiguousarray(A.indices, np.int32)),
                             _p(np.ascontiguousarray(A.data, np.float64)), x.shape[1], _p(x), _p(f), _p(r))
    return r


class CholFactor:
    """The oracle's supernodal FP64 Cholesky of Symmetric(K_ff), factored once."""

    def __init__(self, Kff, perm, nthreads: int = 0):
        Kc = Kff.tocsc()
        self.n = Kc.shape[0]
        self.h = ctypes.c_void_p()
        st = lib().or_chol_factor(self.n, _p(np.ascontiguousarray(Kc.indptr, np.int64)),
                                  _p(np.ascontiguousarray(Kc.indices, np.int32)),
                                  _p(np.ascontiguousarray(Kc.data, np.float64)),
                                  _p(np.ascontiguousarray(perm, np.int32)), int(nthreads), ctypes.byref(self.h))
        if st != 0:
            raise RuntimeError(f"oracle cholesky failed: status {st}")

    def solve(self, F):
        F = np.asfortranarray(F, np.float64)
        one = F.ndim == 1
        if one:
            F = F[:, None]
        U = np.zeros_like(F, order="F")
        lib().or_chol_solve(self.h, F.shape[1], _p(F), _p(U))
        return U[:, 0] if one else U

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_chol_free(self.h)
            self.h = None


def solve_reference_chol(model, nthreads: int = 0, refine: int = 6):
    """FP64 SOL101 on the CPU for large checks: the oracle's partition and
    ordering, its supernodal Cholesky (OpenBLAS), and refinement on the
    assembled K_ff with compensated residuals, so that the checker's
    displacements are accurate to about the conditioning of the FP64 data.
    Returns dict(u (ndof x nrhs), F, R = K u - F, free, rel_residual)."""
    asm = assemble(model)
    K = csc_matrix(asm)
    free, _, _ = partition(model, K)
    Kff = K[free][:, free].tocsc()
    perm, _ = order(Kff, free, model.xyz)
    F = load_matrix(model)
    Fff = np.asfortranarray(F[free])
    C = CholFactor(Kff, perm, nthreads)
    u_ff = C.solve(Fff)
    fn = np.maximum(np.linalg.norm(Fff, axis=0), 1e-300)
    for _ in range(refine):
        r = residual_dd(Kff, u_ff, Fff)
        if np.all(np.linalg.norm(r, axis=0) <= 1e-16 * fn):
            break
        u_ff = u_ff + C.solve(r)
    u = np.zeros_like(F)
    u[free] = u_ff
    rel = np.linalg.norm(residual_dd(Kff, u_ff, Fff), axis=0) / fn
    return dict(u=u, F=F, R=K @ u - F, free=free, rel_residual=rel)


def chol_solve(n, colptr, rowval, nzval, perm, F, nthreads=0):
    """Oracle supernodal multifrontal FP64 Cholesky (OpenBLAS dense kernels).

    (colptr,rowval,nzval): CSC of K_ff; only the upper triangle (row <= col)
    is read, as Symmetric(K_ff) does.  perm: elimination order (perm[k] =
    unknown eliminated k-th).  F: n x nrhs.  Returns U (n x nrhs).
    """
    L = lib()
    F = np.asfortranarray(F, dtype=np.float64)
    if F.ndim == 1:
        F = F[:, None]
    U = np.zeros_like(F, order="F")
    info = np.zeros(4)
    st = L.or_chol_factor_solve(int(n), _p(np.ascontiguousarray(colptr, np.int64)),
                                _p(np.ascontiguousarray(rowval, np.int32)),
                                _p(np.ascontiguousarray(nzval, np.float64)),
                                _p(np.ascontiguousarray(perm, np.int32)), int(F.shape[1]),
                                _p(F), _p(U), int(nthreads), _p(info))
    if st != 0:
        raise RuntimeError(f"oracle cholesky failed: status {st}, info {info}")
    return U, dict(factor_s=info[0], solve_s=info[1], nnz_L=info[2], flops=info[3])
