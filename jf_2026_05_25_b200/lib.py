"""ctypes binding of libjfemgpu.so (the C ABI declared in include/jfemgpu.h).

The binding is the Python counterpart of the Julia ``ccall`` shim: it passes
plain host arrays and sizes and never exposes device pointers except through
``solve_device`` (torch/cupy tensors' ``data_ptr()``).  Importing this module
fails loudly when the shared library has not been built.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

from .build import LIB

JFG_OK = 0
STATUS = {0: "OK", 1: "NOT_SPD", 2: "IR_STALLED", 3: "OOM_BUDGET", 4: "TIMEOUT", 5: "UNSUPPORTED",
          6: "BAD_INPUT", 7: "CUDA_ERROR", 8: "NOT_READY"}
PREC_FP64 = 0
PREC_MIXED = 1

_c = ctypes
P = _c.c_void_p
I32 = _c.c_int32
I64 = _c.c_int64
D = _c.c_double


class JfgConfig(_c.Structure):
    _fields_ = [("device", I32), ("flags", I32), ("hbm_budget_bytes", I64)]


class SolveReport(_c.Structure):
    _fields_ = [("rel_residual", D), ("max_rel_update", D), ("ir_iters", I32), ("fallback_used", I32),
                ("precision", I32), ("reserved", I32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class SymbolicInfo(_c.Structure):
    _fields_ = [("n_supernodes", I64), ("n_levels", I64), ("nnz_L", I64), ("flops", D), ("factor_bytes", I64),
                ("max_front", I64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class JfgError(RuntimeError):
    def __init__(self, status: int, msg: str, detail: int):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status
        self.status_name = STATUS.get(status, str(status))
        self.detail = detail


_lib = None


def load():
    """Load libjfemgpu.so; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        raise ImportError(f"{LIB} is not built; run `python -m jf_2026_05_25_b200.build`")
    L = _c.CDLL(LIB)
    sig = {
        "jfg_create": [P, P],
        "jfg_destroy": [P],
        "jfg_model_upload": [P, I64, P, P, I64, P, P, I64, P, P, I64, P, P, P],
        "jfg_model_add_tria3": [P, I64, P, P],
        "jfg_model_free": [P],
        "jfg_assemble": [P],
        "jfg_get_sizes": [P, P, P, P],
        "jfg_get_pattern": [P, P, P],
        "jfg_get_values": [P, P],
        "jfg_get_slot_map": [P, P],
        "jfg_get_diag": [P, P, P],
        "jfg_get_node_blocks": [P, P],
        "jfg_get_element_matrix": [P, I32, I64, P],
        "jfg_set_free_dofs": [P, I64, P],
        "jfg_get_symbolic_info": [P, P],
        "jfg_get_perm": [P, P],
        "jfg_factor": [P, I32],
        "jfg_get_factor_diag": [P, P],
        "jfg_solve": [P, I32, P, P, D, I32, P],
        "jfg_solve_device": [P, I32, P, P, D, I32, P],
        "jfg_residual": [P, I32, P, P, P],
        "jfg_update_q4_sections": [P, I64, P, P],
        "jfg_get_timings": [P, P],
        "jfg_symbolic_dry_run": [I64, P, P, I64, P, P, P, P],
        "jfg_assemble_values_noalloc": [P, P],
        "jfg_recover_stresses": [P, I32, I32, P, P],
        "jfg_model_share_structure": [P, P],
        "jfg_factor_async": [P, I32, P],
        "jfg_apply_factor_async": [P, I32, P, P, P],
        "jfg_wait": [P],
        "jfg_get_memory": [P, I32, I32, P, P],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = _c.c_int
    L.jfg_launch_count.restype = I64
    L.jfg_launch_count.argtypes = []
    L.jfg_set_profiling.argtypes = [I32]
    L.jfg_set_profiling.restype = _c.c_int
    L.jfg_get_kernel_stats.argtypes = [I32, P]
    L.jfg_get_kernel_stats.restype = _c.c_int
    L.jfg_reset_kernel_stats.argtypes = []
    L.jfg_reset_kernel_stats.restype = _c.c_int
    L.jfg_last_error.restype = _c.c_char_p
    L.jfg_last_error.argtypes = []
    L.jfg_last_error_detail.restype = I64
    L.jfg_last_error_detail.argtypes = []
    _lib = L
    return L


def exported_symbols():
    """Names declared in include/jfemgpu.h (parsed from the header)."""
    import re
    hdr = os.path.join(os.path.dirname(LIB), "..", "include", "jfemgpu.h")
    return sorted(set(re.findall(r"\b(jfg_[a-z0-9_]+)\s*\(", open(hdr).read())))


def _check(st: int):
    if st != JFG_OK:
        L = load()
        raise JfgError(st, L.jfg_last_error().decode(errors="replace"), L.jfg_last_error_detail())


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(P)


class Context:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        L = load()
        self.h = P()
        cfg = JfgConfig(device, 0, hbm_budget_bytes)
        _check(L.jfg_create(_c.byref(self.h), _c.byref(cfg)))

    def close(self):
        if self.h:
            load().jfg_destroy(self.h)
            self.h = P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceModel:
    """A model resident on the device: CSC K, symbolic analysis and factor."""

    def __init__(self, ctx: Context, model):
        L = load()
        self.ctx = ctx
        self.model = model
        self.h = P()
        # shells as assembled: native CQUAD8 only; the model's CTRIA3 plus
        # the six triangles of every other CQUAD8
        q8n, q8s = model.device_q8()
        t3n, t3s = model.device_t3()
        self._keep = dict(
            xyz=np.ascontiguousarray(model.xyz, np.float64),
            R=np.ascontiguousarray(model.node_R, np.float64),
            q4n=np.ascontiguousarray(model.q4_nodes, np.int32),
            q4s=np.ascontiguousarray(model.q4_sections(), np.float64),
            q8n=np.ascontiguousarray(q8n, np.int32),
            q8s=np.ascontiguousarray(q8s, np.float64),
            t3n=np.ascontiguousarray(t3n, np.int32),
            t3s=np.ascontiguousarray(t3s, np.float64),
            t10n=np.ascontiguousarray(model.t10_nodes, np.int32),
            t10m=np.ascontiguousarray(model.t10_materials(), np.float64),
        )
        k = self._keep
        _check(L.jfg_model_upload(ctx.h, model.n_nodes, _p(k["xyz"]), _p(k["R"]), len(k["q4n"]), _p(k["q4n"]),
                                  _p(k["q4s"]), len(k["q8n"]), _p(k["q8n"]), _p(k["q8s"]), len(k["t10n"]),
                                  _p(k["t10n"]), _p(k["t10m"]), _c.byref(self.h)))
        if len(k["t3n"]):
            st = L.jfg_model_add_tria3(self.h, len(k["t3n"]), _p(k["t3n"]), _p(k["t3s"]))
            if st != 0:
                L.jfg_model_free(self.h)
                self.h = P()
                _check(st)
        self.ndof = model.ndof
        self.n_free = None

    def close(self):
        if self.h:
            load().jfg_model_free(self.h)
            self.h = P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def share_structure(self, src: "DeviceModel"):
        """Take over the pattern and the symbolic analysis of a resident model
        of the same mesh (see jfg_model_share_structure)."""
        _check(load().jfg_model_share_structure(self.h, src.h))

    # ---- assembly
    def assemble(self):
        _check(load().jfg_assemble(self.h))

    def sizes(self) -> Tuple[int, int, int]:
        a, b, c = I64(), I64(), I64()
        _check(load().jfg_get_sizes(self.h, _c.byref(a), _c.byref(b), _c.byref(c)))
        return a.value, b.value, c.value

    def pattern(self):
        ndof, nnz, _ = self.sizes()
        colptr = np.empty(ndof + 1, np.int64)
        rowval = np.empty(nnz, np.int32)
        _check(load().jfg_get_pattern(self.h, _p(colptr), _p(rowval)))
        return colptr, rowval

    def values(self) -> np.ndarray:
        _, nnz, _ = self.sizes()
        v = np.empty(nnz)
        _check(load().jfg_get_values(self.h, _p(v)))
        return v

    def slot_map(self) -> np.ndarray:
        _, _, nt = self.sizes()
        s = np.empty(nt, np.int64)
        _check(load().jfg_get_slot_map(self.h, _p(s)))
        return s

    def diag(self):
        d = np.empty(self.ndof)
        mx = D()
        _check(load().jfg_get_diag(self.h, _p(d), _c.byref(mx)))
        return d, mx.value

    def node_blocks(self) -> np.ndarray:
        b = np.empty((self.model.n_nodes, 18))
        _check(load().jfg_get_node_blocks(self.h, _p(b)))
        return b

    def element_matrix(self, kind: int, elem: int) -> np.ndarray:
        n = {0: 24, 1: 48, 2: 30, 3: 18}[kind]
        K = np.empty((n, n), order="F")
        _check(load().jfg_get_element_matrix(self.h, kind, elem, _p(K)))
        return K

    def csc(self):
        import scipy.sparse as sp
        colptr, rowval = self.pattern()
        return sp.csc_matrix((self.values(), rowval, colptr), shape=(self.ndof, self.ndof))

    # ---- symbolic / numeric
    def set_free_dofs(self, free: np.ndarray):
        free = np.ascontiguousarray(free, np.int32)
        _check(load().jfg_set_free_dofs(self.h, len(free), _p(free)))
        self.n_free = len(free)
        self.free = free

    def symbolic_info(self) -> dict:
        info = SymbolicInfo()
        _check(load().jfg_get_symbolic_info(self.h, _c.byref(info)))
        return info.as_dict()

    def perm(self) -> np.ndarray:
        p = np.empty(self.n_free, np.int32)
        _check(load().jfg_get_perm(self.h, _p(p)))
        return p

    def factor(self, precision: int = PREC_FP64):
        _check(load().jfg_factor(self.h, precision))

    def factor_async(self, precision: int, stream_ptr: int):
        """Enqueue the factorisation on a CUDA stream (cudaStream_t as int)."""
        _check(load().jfg_factor_async(self.h, precision, P(stream_ptr)))

    def apply_factor_async(self, F_ptr: int, U_ptr: int, nrhs: int, stream_ptr: int):
        """Enqueue U = K_ff^-1 F (one factor application, device arrays)."""
        _check(load().jfg_apply_factor_async(self.h, nrhs, P(F_ptr), P(U_ptr), P(stream_ptr)))

    def memory(self, precision: int, nrhs: int):
        """(bytes held now, bytes after factoring at `precision` and solving nrhs columns)."""
        a, b = I64(), I64()
        _check(load().jfg_get_memory(self.h, precision, nrhs, _c.byref(a), _c.byref(b)))
        return a.value, b.value

    def wait(self):
        _check(load().jfg_wait(self.h))

    def factor_diag(self) -> np.ndarray:
        d = np.empty(self.n_free)
        _check(load().jfg_get_factor_diag(self.h, _p(d)))
        return d

    def solve(self, F: np.ndarray, tol: float = 1e-10, max_ir: int = 10, raise_on_stall: bool = True):
        F = np.asfortranarray(F, np.float64)
        if F.ndim == 1:
            F = F[:, None]
        U = np.zeros_like(F, order="F")
        rep = SolveReport()
        st = load().jfg_solve(self.h, F.shape[1], _p(F), _p(U), tol, max_ir, _c.byref(rep))
        if st != JFG_OK and not (st == 2 and not raise_on_stall):
            _check(st)
        return U, rep.as_dict()

    def solve_device(self, F_ptr: int, U_ptr: int, nrhs: int, tol: float = 1e-10, max_ir: int = 10,
                     raise_on_stall: bool = True):
        rep = SolveReport()
        st = load().jfg_solve_device(self.h, nrhs, P(F_ptr), P(U_ptr), tol, max_ir, _c.byref(rep))
        if st != JFG_OK and not (st == 2 and not raise_on_stall):
            _check(st)
        return rep.as_dict()

    def residual(self, U: np.ndarray, F: np.ndarray) -> np.ndarray:
        U = np.asfortranarray(U, np.float64)
        F = np.asfortranarray(F, np.float64)
        R = np.empty_like(U, order="F")
        nr = 1 if U.ndim == 1 else U.shape[1]
        _check(load().jfg_residual(self.h, nr, _p(U), _p(F), _p(R)))
        return R

    def t10_stresses(self, U: np.ndarray) -> np.ndarray:
        """Centroid stress, strain and von Mises of every CTETRA10 for every
        column of U: array (nrhs, n_t10, 13)."""
        U = np.asfortranarray(U, np.float64)
        if U.ndim == 1:
            U = U[:, None]
        out = np.empty((U.shape[1], len(self.model.t10_nodes), 13))
        _check(load().jfg_recover_stresses(self.h, 2, U.shape[1], _p(U), _p(out)))
        return out

    def q4_stresses(self, U: np.ndarray) -> np.ndarray:
        """Centre forces, fibre stresses and strains of every CQUAD4 for every
        column of U: array (nrhs, n_q4, 31) in the layout of jfg_recover_stresses
        kind 0.  Elements whose PSHELL the reference leaves unrecovered (MID2 or
        MID3 a different material law, _pshell_local_constitutive_gap,
        stress_recovery.jl:193-215) are NaN, as the reference omits them."""
        U = np.asfortranarray(U, np.float64)
        if U.ndim == 1:
            U = U[:, None]
        out = np.empty((U.shape[1], len(self.model.q4_nodes), 31))
        _check(load().jfg_recover_stresses(self.h, 0, U.shape[1], _p(U), _p(out)))
        out[:, ~self.model.q4_recovery_mask()] = np.nan
        return out

    def update_q4_sections(self, elems: np.ndarray, sect: np.ndarray):
        elems = np.ascontiguousarray(elems, np.int32)
        sect = np.ascontiguousarray(sect, np.float64)
        _check(load().jfg_update_q4_sections(self.h, len(elems), _p(elems), _p(sect)))

    def assemble_values_noalloc(self, nzval_dev_ptr: int):
        """K's values into a caller-owned device buffer (nnz doubles) with no
        device allocation inside the library; see jfg_assemble_values_noalloc."""
        _check(load().jfg_assemble_values_noalloc(self.h, P(nzval_dev_ptr)))

    def timings(self) -> dict:
        t = np.zeros(4)
        _check(load().jfg_get_timings(self.h, _p(t)))
        return dict(elements=t[0], assembly=t[1], factor=t[2], solve=t[3])


def symbolic_dry_run(colptr, rowval, free, xyz):
    """Host-only symbolic analysis (no device): returns (info dict, perm)."""
    L = load()
    colptr = np.ascontiguousarray(colptr, np.int64)
    rowval = np.ascontiguousarray(rowval, np.int32)
    free = np.ascontiguousarray(free, np.int32)
    xyz = np.ascontiguousarray(xyz, np.float64)
    info = SymbolicInfo()
    perm = np.empty(len(free), np.int32)
    _check(L.jfg_symbolic_dry_run(len(colptr) - 1, _p(colptr), _p(rowval), len(free), _p(free), _p(xyz),
                                  _c.byref(info), _p(perm)))
    return info.as_dict(), perm
