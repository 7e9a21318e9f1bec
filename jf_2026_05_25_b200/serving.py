"""Device-resident SOL101 serving: packed batches, a resident-model registry
and continuous batching over several device streams.

The reference keeps one warm model per worker process and re-solves it
(utils/julia_tools/warm_model_session.jl:5-99, jfem_worker_jsonl.jl:77-100,
boundary_conditions.jl:62-75).  Here:

* ``PackedModel`` packs independent small models into one block-diagonal
  model (disjoint node sets, coordinates shifted apart).  Its element
  kernels, assembly, level-scheduled factor and strip solves then run as one
  set of launches for the whole batch: every level launch carries the fronts
  of all models.  Load case c of every member goes to column c, scaled to unit
  norm, and the refinement tolerance is divided by sqrt(members), so every
  member meets the requested relative residual on its own; the split undoes
  the scaling.
* ``SolveServer`` keeps models (or packs) resident on the device: their
  pattern, symbolic analysis and factor stay in HBM for re-solves with new
  loads or thickness updates.  Resident bytes are charged against an HBM
  budget and the least recently used models are freed to admit new ones.
* Continuous batching: ``slots`` worker threads each own a library context
  (its own CUDA stream); a free slot takes the next request, or every queued
  new small model up to a DOF limit as one pack, while the other slots'
  work is still on the device, so their kernels overlap.  Each request's
  latency runs from submission to its result; ``stats()`` gives p50/p99.
"""
from __future__ import annotations

import hashlib
import math
import os
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import backend as B
from . import lib


def _is_tensor(x) -> bool:
    return x is not None and type(x).__module__.startswith("torch")


class PackedModel:
    """Block-diagonal union of independent models (the batch unit)."""

    def __init__(self, models: Sequence, gap: float = 1.0):
        self.members = list(models)
        xyz, R, q4n, q4s, q8n, q8s, t10n, t10m, spc = [], [], [], [], [], [], [], [], []
        t3n, t3s = [], []
        self.node_off, self.q4_off = [], []
        n_off = 0
        q4_off = 0
        x0 = 0.0
        for m in self.members:
            p = np.asarray(m.xyz, float)
            lo, hi = p.min(axis=0), p.max(axis=0)
            shift = np.array([x0 - lo[0], -lo[1], -lo[2]])
            xyz.append(p + shift)
            x0 += (hi[0] - lo[0]) + gap
            R.append(np.asarray(m.node_R, float))
            q4n.append(np.asarray(m.q4_nodes, np.int32) + n_off)
            q4s.append(m.q4_sections())
            n8, s8 = m.device_q8()
            q8n.append(np.asarray(n8, np.int32) + n_off)
            q8s.append(s8)
            n3, s3 = m.device_t3()
            t3n.append(np.asarray(n3, np.int32) + n_off)
            t3s.append(s3)
            t10n.append(np.asarray(m.t10_nodes, np.int32) + n_off)
            t10m.append(m.t10_materials())
            spc.append(np.asarray(m.spc_dofs(), np.int64) + 6 * n_off)
            self.node_off.append(n_off)
            self.q4_off.append(q4_off)
            n_off += m.n_nodes
            q4_off += len(m.q4_nodes)
        self.node_off.append(n_off)
        self.q4_off.append(q4_off)
        self.xyz = np.vstack(xyz)
        self.node_R = np.vstack(R)
        self.q4_nodes = np.vstack(q4n).reshape(-1, 4)
        self._q4s = np.vstack(q4s).reshape(-1, 26)
        self.q8_nodes = np.vstack(q8n).reshape(-1, 8)
        self._q8s = np.vstack(q8s).reshape(-1, 22)
        self._t3n = np.vstack(t3n).reshape(-1, 3)
        self._t3s = np.vstack(t3s).reshape(-1, 26)
        self.t10_nodes = np.vstack(t10n).reshape(-1, 10)
        self._t10m = np.vstack(t10m).reshape(-1, 2)
        self._spc = np.unique(np.concatenate(spc))
        self.name = f"pack_{len(self.members)}"

    # attributes the device binding and the partition read
    @property
    def n_nodes(self) -> int:
        return int(self.node_off[-1])

    @property
    def ndof(self) -> int:
        return 6 * self.n_nodes

    def q4_sections(self):
        return self._q4s

    def q8_sections(self):
        return self._q8s

    def device_q8(self):
        return self.q8_nodes, self._q8s

    def device_t3(self):
        return self._t3n, self._t3s

    def t10_materials(self):
        return self._t10m

    def spc_dofs(self):
        return self._spc

    def dof_slice(self, k: int) -> slice:
        return slice(6 * self.node_off[k], 6 * self.node_off[k + 1])

    def load_columns(self, loads: Optional[Sequence[np.ndarray]] = None):
        """Packed load matrix: column c holds case c of every member, each
        scaled to unit norm.  Returns (F, scales[member][case])."""
        loads = [m.load_matrix() if loads is None or loads[k] is None else np.asarray(loads[k])
                 for k, m in enumerate(self.members)]
        ncol = max(L.shape[1] for L in loads)
        F = np.zeros((self.ndof, ncol), order="F")
        scales = []
        for k, L in enumerate(loads):
            sl = self.dof_slice(k)
            sc = []
            for c in range(L.shape[1]):
                nrm = float(np.linalg.norm(L[:, c]))
                s = 1.0 / nrm if nrm > 0 else 1.0
                F[sl, c] = L[:, c] * s
                sc.append(s)
            scales.append(sc)
        return F, scales

    def split(self, U: np.ndarray, scales) -> List[np.ndarray]:
        out = []
        for k, sc in enumerate(scales):
            sl = self.dof_slice(k)
            out.append(np.asfortranarray(U[sl, :len(sc)] / np.asarray(sc)[None, :]))
        return out


def member_residuals(dm, pack: PackedModel, U: np.ndarray, F: np.ndarray, free: np.ndarray,
                     ncases: Sequence[int]) -> List[np.ndarray]:
    """Relative residual |K u - f| / |f| of every member and case, on the
    member's own free DOFs (the reference's measure, boundary_conditions.jl:1858-1866)."""
    R = dm.residual(U, F)
    mask = np.zeros(pack.ndof, bool)
    mask[free] = True
    out = []
    for k, nc in enumerate(ncases):
        sl = pack.dof_slice(k)
        mk = mask[sl]
        r = np.linalg.norm(R[sl][mk, :nc], axis=0)
        f = np.linalg.norm(F[sl][mk, :nc], axis=0)
        out.append(r / np.where(f > 0, f, 1.0))
    return out


def solve_pack(be: B.JFEMGPUBackend, models: Sequence, tol: float = 1e-10) -> Dict:
    """Prepare and solve a pack of independent models in one set of launches.
    Returns dict(state, pack, U (list per member), residuals (list per member))."""
    pack = PackedModel(models)
    st = B.prepare(be, pack)
    F, scales = pack.load_columns()
    # each column mixes the members' unit-norm loads: tol / sqrt(members)
    # bounds every member's own relative residual by tol; the factor 0.5
    # covers the difference between the device's compensated residual and
    # the member-wise check
    tol_c = 0.5 * tol / math.sqrt(max(1, len(models)))
    U, rep = st["dm"].solve(F, tol_c, max(be.max_ir, 30), raise_on_stall=False)
    res = member_residuals(st["dm"], pack, U, F, st["free"], [len(sc) for sc in scales])
    return dict(state=st, pack=pack, U=pack.split(U, scales), residuals=res, report=rep, F=F, scales=scales)


# ----------------------------------------------------------------------------
# server
# ----------------------------------------------------------------------------

@dataclass
class Request:
    kind: str                          # "solve" (new model), "resolve" (new loads), "update" (thickness)
    model: object = None               # Sol101Model for "solve"
    key: Optional[str] = None          # registry key (returned by "solve", used by the others)
    loads: Optional[np.ndarray] = None # ndof x nrhs for "resolve"/"update" (None: the model's own cases)
    elems: Optional[np.ndarray] = None # CQUAD4 indices for "update"
    sections: Optional[np.ndarray] = None
    # device-resident input and output: `loads` is a CUDA tensor (nrhs x ndof,
    # i.e. the ndof x nrhs column-major load matrix) and the result's "U" is
    # one too; for "solve" it replaces the model's own load cases
    device: bool = False
    t_submit: float = 0.0
    t_start: float = 0.0               # when a slot took it
    mesh: Optional[bytes] = None       # mesh key of a single new model (set by the dispatcher)
    mesh_done: bool = False            # mesh key computed (it may be None: no key)
    was_deferred: bool = False         # skipped at least once by the dispatcher
    future: Future = field(default_factory=Future)


@dataclass
class Resident:
    dm: object
    state: Dict
    pack: Optional[PackedModel]
    index: int                         # member index inside the pack (0 for a single model)
    model: object
    nbytes: int
    lock: threading.Lock
    last_used: float = 0.0
    evicted: bool = False              # set under `lock` when the group is freed
    mesh: Optional[bytes] = None       # mesh key of a single model (structure sharing)
    # held while a new model copies this one's device pattern (short); a
    # running solve does not block that copy, eviction waits for it
    pin: threading.Lock = field(default_factory=threading.Lock)


def _model_class(model, pack) -> str:
    """Class of a unit of work in the phase accounting: a pack of small
    models, a solid model (CTETRA10) or a shell model."""
    if pack is not None:
        return "pack"
    return "solid" if len(getattr(model, "t10_nodes", ())) else "shell"


def mesh_key(model) -> Optional[bytes]:
    """Key of a model's mesh for structure sharing: grid count and CQUAD4 /
    CTRIA3 / CTETRA10 connectivity (CQUAD8 patterns depend on values: no key)."""
    if len(getattr(model, "q8_nodes", ())):
        return None
    h = hashlib.blake2b(digest_size=16)
    h.update(np.int64(model.n_nodes).tobytes())
    h.update(np.ascontiguousarray(model.q4_nodes, np.int32).tobytes())
    h.update(b"|")
    h.update(np.ascontiguousarray(getattr(model, "t3_nodes", np.zeros((0, 3))), np.int32).tobytes())
    h.update(b"|")
    h.update(np.ascontiguousarray(model.t10_nodes, np.int32).tobytes())
    return h.digest()


class SolveServer:
    """Continuous-batching SOL101 server on one device (see module docstring).

    Memory: a new model's bytes are admitted once its symbolic analysis is
    known and before its factor is allocated; least-recently-used idle
    residents are freed to make room (a pack as a unit), and when every
    resident is busy the admission waits up to ``wait_s`` for one to finish.
    A re-solve or update of a model freed meanwhile re-admits it from its
    host description.  New models of a resident mesh take over its pattern
    and symbolic analysis (``share_meshes``).
    """

    def __init__(self, device: int = 0, slots: int = 4, hbm_budget_bytes: float = 150e9,
                 precision: int = lib.PREC_FP64, tol: float = 1e-10, small_dof: int = 60000,
                 pack_dof: int = 400000, pack_models: int = 64, share_meshes: bool = True,
                 wait_s: float = 300.0, slow_refinement_steps: int = 6):
        self.device, self.precision, self.tol = device, precision, tol
        self.small_dof, self.pack_dof, self.pack_models = small_dof, pack_dof, pack_models
        self.share_meshes, self.wait_s = share_meshes, wait_s
        # mixed precision: a mesh whose refinement needed more than this many
        # steps (thin-shell / drilling conditioning) takes the FP64 factor
        # for its later models, updates and re-admissions
        self.slow_refinement_steps = slow_refinement_steps
        self.fp64_meshes = set()
        self.fp64_factorisations = 0
        self.budget = float(hbm_budget_bytes)
        self.q: "queue.Queue[Request]" = queue.Queue()
        self.pending: List[Request] = []
        self.plock = threading.Condition()
        self.registry: Dict[str, Resident] = {}
        self.groups: Dict[int, List[str]] = {}      # pack id -> member keys (freed together)
        self.meshes: Dict[bytes, str] = {}          # mesh key -> key of a resident single model of that mesh
        self.evicted: Dict[str, object] = {}        # key -> host model of a freed model (re-admitted on demand)
        self.rlock = threading.Lock()
        self.mem_cv = threading.Condition(self.rlock)
        self.resident_bytes = 0
        self.reserved = 0.0                          # bytes admitted for models still being prepared
        self.latencies: List[float] = []
        self.kinds: List[str] = []
        self.subcase_solves = 0
        self.readmissions = 0
        self.shared_structures = 0
        self.phase_s: Dict[str, Dict[str, float]] = {}   # class -> phase -> seconds (wall, summed over slots)
        # per finished request: (class, submitted, taken by a slot, finished), perf_counter seconds
        self.trace: List[tuple] = []
        # meshes whose first model is being prepared by a slot: a new model of
        # the same mesh waits in the queue (other work goes first) and then
        # takes over that model's pattern and analysis instead of repeating them
        self.preparing: Dict[bytes, int] = {}
        self.defer_same_mesh = share_meshes and os.environ.get("JFG_SERVE_DEFER", "1") != "0"
        self.deferred = 0
        self.waiting_reserved = 0.0   # reservations of requests waiting in _admit
        self._next_key = 0
        self._stop = False
        self.backends = []
        for _ in range(slots):
            be = B.JFEMGPUBackend(device=device, precision=precision, tol=tol)
            be._ctx = lib.Context(device)
            self.backends.append(be)
        self.threads = [threading.Thread(target=self._worker, args=(i,), daemon=True) for i in range(slots)]
        for t in self.threads:
            t.start()

    # ---------------------------------------------------------------- client API
    def submit(self, req: Request) -> Future:
        req.t_submit = time.perf_counter()
        with self.plock:
            self.pending.append(req)
            self.plock.notify()
        return req.future

    def solve(self, model, device_loads=None, loads=None) -> Future:
        """New model; ``device_loads`` (CUDA tensor, nrhs x ndof) keeps the
        loads and the displacements in device memory; ``loads`` (host array,
        ndof x nrhs) replaces the model's own load cases on the host path."""
        if device_loads is not None:
            return self.submit(Request("solve", model=model, loads=device_loads, device=True))
        return self.submit(Request("solve", model=model, loads=loads, device=False))

    def resolve(self, key: str, loads=None) -> Future:
        return self.submit(Request("resolve", key=key, loads=loads, device=_is_tensor(loads)))

    def update(self, key: str, elems: np.ndarray, sections: np.ndarray, loads=None) -> Future:
        return self.submit(Request("update", key=key, elems=elems, sections=sections, loads=loads,
                                   device=_is_tensor(loads)))

    def close(self):
        with self.plock:
            self._stop = True
            self.plock.notify_all()
        for t in self.threads:
            t.join(timeout=30)
        with self.rlock:
            for r in list(self.registry.values()):
                r.dm.close()
            self.registry.clear()
        for be in self.backends:
            be._ctx.close()

    def stats(self) -> Dict:
        lat = np.asarray(self.latencies)
        if lat.size == 0:
            return {"requests": 0}
        return {"requests": int(lat.size), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                "subcase_solves": int(self.subcase_solves), "resident_bytes": int(self.resident_bytes),
                "readmissions": int(self.readmissions), "shared_structures": int(self.shared_structures),
                "fp64_meshes": len(self.fp64_meshes), "fp64_factorisations": int(self.fp64_factorisations),
                "deferred_same_mesh": int(self.deferred),
                "phase_s": {c: {k: round(v, 4) for k, v in d.items()} for c, d in self.phase_s.items()},
                "timeline": self.timeline()}

    def timeline(self) -> Dict:
        """Per class of request: count, first taken and last finished (seconds
        from the earliest submission), summed slot seconds, and the request
        that finished last (the critical one of a saturated pass)."""
        with self.rlock:
            tr = list(self.trace)
        if not tr:
            return {}
        t0 = min(t[1] for t in tr)
        out: Dict[str, Dict] = {}
        for cls, ts, tt, te in tr:
            d = out.setdefault(cls, {"n": 0, "first_start_s": 1e30, "last_end_s": 0.0, "busy_s": 0.0,
                                     "max_wait_s": 0.0})
            d["n"] += 1
            d["first_start_s"] = min(d["first_start_s"], tt - t0)
            d["last_end_s"] = max(d["last_end_s"], te - t0)
            d["busy_s"] += te - tt
            d["max_wait_s"] = max(d["max_wait_s"], tt - ts)
        for d in out.values():
            for k in ("first_start_s", "last_end_s", "busy_s", "max_wait_s"):
                d[k] = round(d[k], 3)
        last = max(tr, key=lambda t: t[3])
        out["last_request"] = {"class": last[0], "submitted_s": round(last[1] - t0, 3),
                               "start_s": round(last[2] - t0, 3), "end_s": round(last[3] - t0, 3)}
        return out

    # ---------------------------------------------------------------- scheduling
    def _req_mesh(self, r: Request) -> Optional[bytes]:
        """Mesh key of a single new model (computed once per request; packs
        of small models have none)."""
        if not r.mesh_done:
            r.mesh = (mesh_key(r.model) if (self.share_meshes and r.kind == "solve"
                                            and r.model.ndof > self.small_dof) else None)
            r.mesh_done = True
        return r.mesh

    def _deferred(self, r: Request) -> bool:
        """A new model whose mesh another slot is preparing right now, with
        no resident model of that mesh yet: taking it now would repeat the
        pattern build and the symbolic analysis that the other slot is about
        to make resident, so it stays queued until that model is registered."""
        mk = self._req_mesh(r)
        if mk is None or not self.defer_same_mesh or mk not in self.preparing:
            return False
        with self.rlock:
            return mk not in self.meshes

    def _take(self) -> Optional[List[Request]]:
        """Next unit of work: the first queued request that is not deferred
        (see _deferred), or every queued new small model up to the pack
        limits (continuous batching: whatever arrived meanwhile)."""
        with self.plock:
            while True:
                while not self.pending and not self._stop:
                    self.plock.wait(timeout=0.5)
                if self._stop and not self.pending:
                    return None
                idx = None
                for i, r in enumerate(self.pending):
                    if not self._deferred(r):
                        idx = i
                        break
                    if not r.was_deferred:
                        r.was_deferred = True
                        self.deferred += 1
                if idx is not None:
                    break
                self.plock.wait(timeout=0.5)
            first = self.pending.pop(idx)
            first.t_start = time.perf_counter()
            mk = self._req_mesh(first)
            if mk is not None:
                self.preparing[mk] = self.preparing.get(mk, 0) + 1
            if first.kind != "solve" or first.model.ndof > self.small_dof:
                return [first]
            batch, dof = [first], first.model.ndof
            rest = []
            for r in self.pending:
                if (r.kind == "solve" and r.device == first.device and r.model.ndof <= self.small_dof
                        and len(batch) < self.pack_models and dof + r.model.ndof <= self.pack_dof):
                    batch.append(r)
                    dof += r.model.ndof
                else:
                    rest.append(r)
            self.pending = rest
            return batch

    def _worker(self, slot: int):
        be = self.backends[slot]
        be._tstream = None      # this slot's torch stream for device-resident loads
        while True:
            work = self._take()
            if work is None:
                return
            try:
                if work[0].kind == "solve":
                    self._do_solve(be, work)
                elif work[0].kind == "resolve":
                    self._do_resolve(be, work[0])
                else:
                    self._do_update(be, work[0])
            except Exception as exc:   # report to every waiting client
                for r in work:
                    if not r.future.done():
                        r.future.set_exception(exc)
            finally:
                mk = work[0].mesh
                if mk is not None:
                    with self.plock:     # deferred models of this mesh may go now
                        n = self.preparing.get(mk, 0) - 1
                        if n > 0:
                            self.preparing[mk] = n
                        else:
                            self.preparing.pop(mk, None)
                        self.plock.notify_all()

    def _finish(self, req: Request, result: Dict, cls: Optional[str] = None):
        t_end = time.perf_counter()
        dt = t_end - req.t_submit
        with self.rlock:
            self.latencies.append(dt)
            self.kinds.append(req.kind)
            self.trace.append((cls or req.kind, req.t_submit, req.t_start or req.t_submit, t_end))
            self.subcase_solves += int(result["U"].shape[0] if req.device else result["U"].shape[1])
        result["latency_s"] = dt
        req.future.set_result(result)

    # ---------------------------------------------------------------- memory
    @staticmethod
    def _bytes_of(dm) -> int:
        info = dm.symbolic_info()
        _, nnz, ntrip = dm.sizes()
        # factor and its workspaces, K, and the solve vectors of up to 32 right-hand sides
        return int(info["factor_bytes"] * 1.6 + 24 * nnz + 8 * ntrip + 2600 * dm.ndof)

    def _evict_group(self, r: Resident, key: str):
        """Free one group (caller holds rlock and r.lock)."""
        gid = id(r.dm)
        keys = self.groups.pop(gid, [key])
        for k in keys:
            member = self.registry.pop(k, None)
            if member is not None:
                member.evicted = True
                self.evicted[k] = member.model
                if member.mesh is not None and self.meshes.get(member.mesh) == k:
                    del self.meshes[member.mesh]
        r.evicted = True
        self.resident_bytes -= r.nbytes
        r.dm.close()
        self.mem_cv.notify_all()

    def _admit(self, need: float, wait: bool = False, own: float = 0.0, keep: Optional[int] = None):
        """Free least-recently-used residents until `need` more bytes fit, and
        reserve them for the model being prepared (released by _register).

        A pack is freed as a unit.  A group whose lock is held (a re-solve or
        an update is running on it) is skipped, so in-flight work is never
        freed under it.  When every remaining group is busy the request waits
        (``wait``) up to ``wait_s`` for memory to be released, then is
        admitted over budget rather than blocking the server.  The group's
        bytes are released once, and its registry entries go only after its
        lock is held.  ``own``: bytes this request reserved already (its
        upload estimate); with nothing resident and every reservation held by
        requests that are themselves waiting here, nothing can be released,
        so the request is admitted at once.  ``keep``: id of a group's device
        model that this request has pinned (its structure donor); it is not
        freed, and when nothing but it is left the request is admitted over
        budget instead of waiting.
        """
        with self.rlock:
            deadline = time.perf_counter() + self.wait_s
            busy = set()
            waiting = False
            try:
                while self.resident_bytes + self.reserved + need > self.budget:
                    cands = [k for k in self.registry if id(self.registry[k].dm) not in busy
                             and id(self.registry[k].dm) != keep]
                    if not cands and keep is not None and not busy:
                        break          # only the pinned donor is left
                    if not cands:
                        if not waiting:
                            waiting = True
                            self.waiting_reserved += own
                        stuck = not self.registry and self.reserved <= self.waiting_reserved
                        if not wait or time.perf_counter() >= deadline or stuck:
                            break
                        busy.clear()
                        self.mem_cv.wait(timeout=0.5)
                        continue
                    key = min(cands, key=lambda k: self.registry[k].last_used)
                    r = self.registry[key]
                    if not r.lock.acquire(blocking=False):
                        busy.add(id(r.dm))
                        continue
                    if not r.pin.acquire(blocking=False):
                        r.lock.release()
                        busy.add(id(r.dm))
                        continue
                    try:
                        self._evict_group(r, key)
                    finally:
                        r.pin.release()
                        r.lock.release()
            finally:
                if waiting:
                    self.waiting_reserved -= own
                    self.mem_cv.notify_all()
            self.reserved += need

    def _release(self, reserved: float):
        with self.rlock:
            self.reserved -= reserved
            self.mem_cv.notify_all()

    def _register(self, dm, state, pack, models, reserved: float = 0.0, keys: Optional[List[str]] = None,
                  mesh: Optional[bytes] = None) -> List[str]:
        # resident bytes: what was admitted for it, or an estimate from its sizes
        nbytes = reserved if reserved > 0 else self._bytes_of(dm)
        lock = threading.Lock()
        out = []
        with self.rlock:
            for i, m in enumerate(models):
                if keys is not None:
                    key = keys[i]
                else:
                    key = f"m{self._next_key}"
                    self._next_key += 1
                self.registry[key] = Resident(dm, state, pack, i, m, nbytes, lock, time.perf_counter(),
                                              mesh=mesh if len(models) == 1 else None)
                self.evicted.pop(key, None)
                out.append(key)
            self.groups[id(dm)] = out
            self.resident_bytes += nbytes
            self.reserved -= reserved
            if mesh is not None and len(models) == 1:
                self.meshes[mesh] = out[0]
            self.mem_cv.notify_all()
        return out

    # ---------------------------------------------------------------- work
    @staticmethod
    def _upload_estimate(target) -> float:
        """Device bytes of a model before its analysis (inputs, element
        values, CSC pattern), from its sizes: 9 node pairs of 36 entries per
        shell grid, 30 pairs of 9 per solid grid."""
        n_q4 = len(getattr(target, "q4_nodes", ()))
        n_q8 = len(getattr(target, "q8_nodes", ()))
        n_t10 = len(getattr(target, "t10_nodes", ()))
        n_t3 = len(target.device_t3()[0]) if hasattr(target, "device_t3") else 0
        n_ev = 576 * n_q4 + 2304 * n_q8 + 900 * n_t10 + 324 * n_t3
        nnz = (324 if n_t10 == 0 else 270) * target.n_nodes
        return float(8 * n_ev + 8 * 210 * n_q4 + 4 * n_ev + 28 * nnz + 150 * target.n_nodes)

    def _prepare(self, be, model, pack: Optional[PackedModel], nrhs: int = 8, mk: Optional[bytes] = None):
        """Upload (sharing a resident mesh's structure when there is one),
        analyse, admit the exact bytes, factor.  Device bytes are admitted
        twice: an estimate before the upload, and the library's own figure
        (jfg_get_memory: factor, its work arrays and the solve work space for
        `nrhs`) once the analysis exists.  Returns (state, reserved, mesh)."""
        target = pack if pack is not None else model
        if mk is None:
            mk = mesh_key(model) if (pack is None and self.share_meshes) else None
        prec = self.precision
        if prec == lib.PREC_MIXED and mk is not None and mk in self.fp64_meshes:
            prec = lib.PREC_FP64
            with self.rlock:
                self.fp64_factorisations += 1
        # the resident model of this mesh is pinned before the admission, so
        # that making room for the new model never frees the structure it is
        # about to take over (eviction skips pinned groups)
        donor = None
        if mk is not None:
            with self.rlock:
                dk = self.meshes.get(mk)
                donor = self.registry.get(dk) if dk is not None else None
            if donor is not None and not donor.pin.acquire(timeout=60.0):
                donor = None
        try:
            pre = self._upload_estimate(target)
            self._admit(pre, wait=True, keep=id(donor.dm) if donor is not None else None)
            admitted = [pre]
            t_up = time.perf_counter()
            try:
                dm = lib.DeviceModel(be.ctx, target)
            except Exception:
                self._release(pre)
                raise
            if donor is not None and not donor.evicted:
                dm.share_structure(donor.dm)
                with self.rlock:
                    self.shared_structures += 1
        finally:
            if donor is not None:
                donor.pin.release()

        def admit(d):
            need = float(d.memory(prec, nrhs)[1])
            if need > admitted[0]:
                self._admit(need - admitted[0], wait=True, own=admitted[0])
                admitted[0] = need

        t_prep = time.perf_counter()
        try:
            st = B.prepare(be, target, dm=dm, before_factor=admit, precision=prec)
        except Exception:
            dm.close()
            self._release(admitted[0])
            raise
        tm = st.get("timings", {})
        self._add_phases(_model_class(target, pack), upload=t_prep - t_up, assembly=tm.get("assembly", 0.0),
                         analysis=tm.get("constraints", 0.0), analysis_symbolic=tm.get("symbolic", 0.0),
                         factor=tm.get("factorization", 0.0))
        return st, admitted[0], mk

    def _add_phases(self, cls: str, **secs):
        with self.rlock:
            d = self.phase_s.setdefault(cls, {})
            for k, v in secs.items():
                d[k] = d.get(k, 0.0) + float(v)

    def _do_solve(self, be, reqs: List[Request]):
        models = [r.model for r in reqs]
        pack = PackedModel(models)
        nrhs = max(16, max((r.loads.shape[0] if r.device else
                            (r.loads.shape[1] if r.loads is not None else len(r.model.load_cases))) for r in reqs))
        st, reserved, mk = self._prepare(be, models[0], pack if len(models) > 1 else None, nrhs,
                                         mk=reqs[0].mesh if len(models) == 1 else None)
        t_sol = time.perf_counter()
        try:
            if reqs[0].device:
                Us, res, rep = self._device_solve(be, st["dm"], pack, [r.loads for r in reqs], self.tol)
            elif len(models) > 1:
                F, scales = pack.load_columns([r.loads for r in reqs])
                tol_c = 0.5 * self.tol / math.sqrt(len(models))
                U, rep = st["dm"].solve(F, tol_c, max(be.max_ir, 30), raise_on_stall=False)
                res = member_residuals(st["dm"], pack, U, F, st["free"], [len(sc) for sc in scales])
                Us = pack.split(U, scales)
            else:
                F = models[0].load_matrix() if reqs[0].loads is None else reqs[0].loads
                U, rep = st["dm"].solve(F, 0.5 * self.tol, max(be.max_ir, 30), raise_on_stall=False)
                # the solve's report carries the largest relative residual
                # over the columns, |f - K u| / |f| on the free DOFs, from the
                # library's compensated residual
                res = [np.full(F.shape[1], rep["rel_residual"])]
                Us = [U]
        except Exception:
            st["dm"].close()
            self._release(reserved)
            raise
        self._add_phases(_model_class(models[0], pack if len(models) > 1 else None),
                         solve=time.perf_counter() - t_sol)
        if (self.precision == lib.PREC_MIXED and mk is not None and st.get("precision") == lib.PREC_MIXED
                and rep.get("ir_iters", 0) > self.slow_refinement_steps):
            with self.rlock:
                self.fp64_meshes.add(mk)
        keys = self._register(st["dm"], st, pack, models, reserved=reserved, mesh=mk)
        for k, r in enumerate(reqs):
            self._finish(r, {"key": keys[k], "U": Us[k], "rel_residual": res[k], "batch": len(reqs),
                             "report": rep}, cls=_model_class(models[0], pack if len(models) > 1 else None))

    def _device_solve(self, be, dm, pack: PackedModel, loads: List, tol: float, only: Optional[int] = None):
        """Solve with loads and displacements in device memory.  loads[k]
        (CUDA tensor nrhs_k x ndof_k) belongs to member k (or to member
        `only`).  Every member's columns are scaled to unit norm in the packed
        load matrix and the tolerance divided by sqrt(members), so that the
        reported relative residual bounds each member's own.
        Returns (list of U tensors, list of residual arrays, report)."""
        import torch
        if be._tstream is None:
            be._tstream = torch.cuda.Stream()
        members = [only] if only is not None else list(range(len(loads)))
        with torch.cuda.stream(be._tstream):
            ncol = max(int(L.shape[0]) for L in loads)
            F = torch.zeros((ncol, pack.ndof), dtype=torch.float64, device="cuda")
            scales = []
            for k, L in zip(members, loads):
                sl = pack.dof_slice(k)
                nrm = torch.linalg.vector_norm(L, dim=1)
                sc = torch.where(nrm > 0, 1.0 / nrm, torch.ones_like(nrm))
                F[:L.shape[0], sl] = L * sc[:, None]
                scales.append(sc)
            U = torch.zeros_like(F)
        be._tstream.synchronize()
        tol_c = tol / math.sqrt(max(1, len(members))) * (0.5 if len(members) > 1 else 1.0)
        rep = dm.solve_device(F.data_ptr(), U.data_ptr(), ncol, tol_c, max(be.max_ir, 30), raise_on_stall=False)
        with torch.cuda.stream(be._tstream):
            Us = [U[:L.shape[0], pack.dof_slice(k)] / sc[:, None] for k, L, sc in zip(members, loads, scales)]
        be._tstream.synchronize()
        res = [np.full(int(L.shape[0]), rep["rel_residual"]) for L in loads]
        return Us, res, rep

    def _member_solve(self, res: Resident, loads, be=None, device: bool = False):
        if device:
            Us, rr, rep = self._device_solve(be, res.dm, res.pack, [loads], 0.5 * self.tol, only=res.index)
            return {"U": Us[0], "rel_residual": rr[0], "report": rep}
        pack = res.pack
        Lm = res.model.load_matrix() if loads is None else np.asarray(loads)
        if Lm.ndim == 1:
            Lm = Lm[:, None]
        # only this member carries load; the others' columns are zero
        F = np.zeros((pack.ndof, Lm.shape[1]), order="F")
        sl = pack.dof_slice(res.index)
        sc = []
        for c in range(F.shape[1]):
            nrm = float(np.linalg.norm(Lm[:, c]))
            s_ = 1.0 / nrm if nrm > 0 else 1.0
            F[sl, c] = Lm[:, c] * s_
            sc.append(s_)
        U, rep = res.dm.solve(F, 0.5 * self.tol, 30, raise_on_stall=False)
        # only this member carries load (the others' solutions are zero), so
        # the report's relative residual is this member's
        rel = np.full(F.shape[1], rep["rel_residual"])
        Um = np.asfortranarray(U[sl] / np.asarray(sc)[None, :])
        return {"U": Um, "rel_residual": rel, "report": rep}

    def _lookup(self, key: str) -> Resident:
        with self.rlock:
            res = self.registry.get(key)
            if res is None:
                raise KeyError(f"model {key} is not resident (evicted or unknown)")
            res.last_used = time.perf_counter()
            return res

    def _lookup_or_readmit(self, be, key: str) -> Resident:
        """The resident of `key`; a model freed meanwhile is prepared again
        from its host description and registered under the same key."""
        with self.rlock:
            res = self.registry.get(key)
            if res is not None:
                res.last_used = time.perf_counter()
                return res
            model = self.evicted.get(key)
        if model is None:
            raise KeyError(f"model {key} is unknown")
        st, reserved, mk = self._prepare(be, model, None, 32)
        pack = PackedModel([model])
        self._register(st["dm"], st, pack, [model], reserved=reserved, keys=[key], mesh=mk)
        with self.rlock:
            self.readmissions += 1
        return self._lookup(key)

    @staticmethod
    def _check_live(res: Resident, key: str):
        """Called with res.lock held: the group may have been evicted between
        the registry lookup and taking the lock."""
        if res.evicted:
            raise KeyError(f"model {key} is not resident (evicted or unknown)")

    def _do_resolve(self, be, req: Request):
        for _ in range(3):
            res = self._lookup_or_readmit(be, req.key)
            with res.lock:
                if res.evicted:
                    continue       # freed between lookup and lock: admit it again
                out = self._member_solve(res, req.loads, be, req.device)
            break
        else:
            raise KeyError(f"model {req.key} could not be kept resident")
        out["key"] = req.key
        self._finish(req, out)

    def _do_update(self, be, req: Request):
        """Thickness (section) update of a resident model: element kernels,
        assembly and the numeric factor rerun on the resident pattern and
        symbolic analysis, then the solve."""
        for _ in range(3):
            res = self._lookup_or_readmit(be, req.key)
            with res.lock:
                if res.evicted:
                    continue
                off = res.pack.q4_off[res.index]
                res.dm.update_q4_sections(np.asarray(req.elems, np.int32) + off, req.sections)
                res.pack._q4s[np.asarray(req.elems) + off] = req.sections
                # keep the host description current (a freed model is re-admitted from it)
                res.model.q4_sect_override = res.pack._q4s[off:res.pack.q4_off[res.index + 1]].copy()
                res.dm.assemble()
                res.dm.factor(res.state.get("precision", self.precision))
                out = self._member_solve(res, req.loads, be, req.device)
            break
        else:
            raise KeyError(f"model {req.key} could not be kept resident")
        out["key"] = req.key
        self._finish(req, out)
