"""SOL101 model container, section resolution, loads and synthetic generators.

This is the host-side mirror of the parts of OpenJFEM that stay on the CPU:
the model dictionary produced by the bulk-data parser (GRID / CQUAD4 /
CQUAD8 / CTETRA10 / PSHELL / PSOLID / MAT1 / SPC1 / PLOAD4 / FORCE), the
per-element section arrays of ``Solver.assemble_stiffness``
(src/solver/assembly.jl:3293-3440) and the load vector of
``_assemble_applied_force`` / ``resolve_loads`` (src/solver/solve_case.jl:57-111,
src/solver/loads.jl:497-586).

Everything is held in flat numpy arrays so that the 150k-element wing box and
the 384k-element solid block build in seconds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

Q4_SECT_STRIDE = 26
Q8_SECT_STRIDE = 22


@dataclass
class Mat1:
    E: float
    NU: float
    G: float = 0.0      # 0 = blank (derived as E/2(1+nu) where the reference does)
    RHO: float = 0.0


@dataclass
class PShell:
    T: float
    MID1: int
    MID2: int = 0
    MID3: int = 0
    BEND_RATIO: float = 1.0   # 12I/T^3
    TS_T: float = 5.0 / 6.0


@dataclass
class LoadCase:
    """One subcase: PLOAD4 pressures on shell elements and nodal forces.

    ``pload4``: (element index array into the Q4 list, pressure array).
    ``forces``: (node index array, (n,3) force vectors, global frame).
    ``cload``:  (node index array, (n,3) translational forces) -- consistent
                C3D10 face loads delivered as nodal loads (abaqus_input.jl:347-405).
    ``pload4_t3``: (element index array into the CTRIA3 list, pressure array).
    """
    sid: int
    pload4: Optional[Tuple[np.ndarray, np.ndarray]] = None
    pload4_t3: Optional[Tuple[np.ndarray, np.ndarray]] = None
    forces: Optional[Tuple[np.ndarray, np.ndarray]] = None
    cload: Optional[Tuple[np.ndarray, np.ndarray]] = None


@dataclass
class Sol101Model:
    name: str
    grid_ids: np.ndarray                     # (n,) sorted GRID ids
    xyz: np.ndarray                          # (n,3)
    node_R: Optional[np.ndarray] = None      # (n,9) column-major CD rotations
    q4_nodes: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    q4_pid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    q4_eid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    q8_nodes: np.ndarray = field(default_factory=lambda: np.zeros((0, 8), np.int32))
    q8_pid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    t3_nodes: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    t3_pid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    t10_nodes: np.ndarray = field(default_factory=lambda: np.zeros((0, 10), np.int32))
    t10_pid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    pshells: Dict[int, PShell] = field(default_factory=dict)
    psolids: Dict[int, int] = field(default_factory=dict)  # pid -> mid
    mats: Dict[int, Mat1] = field(default_factory=dict)
    k6rot: float = 100.0                    # PARAM,K6ROT (assembly.jl:1837-1851)
    spc1: List[Tuple[str, np.ndarray]] = field(default_factory=list)
    load_cases: List[LoadCase] = field(default_factory=list)
    seed: Optional[int] = None
    # per-element CQUAD4 section records set by a thickness update; when
    # present they replace the records derived from the PSHELL cards
    q4_sect_override: Optional[np.ndarray] = None

    def __post_init__(self):
        if self.node_R is None:
            R = np.zeros((len(self.grid_ids), 9))
            R[:, 0] = R[:, 4] = R[:, 8] = 1.0
            self.node_R = R

    @property
    def n_nodes(self) -> int:
        return int(len(self.grid_ids))

    @property
    def ndof(self) -> int:
        return 6 * self.n_nodes

    # ------------------------------------------------------------------ sections
    def q4_sections(self) -> np.ndarray:
        """Per-element Q4 section records (assembly.jl:3300-3440, isotropic MAT1).

        Cm = E h/(1-nu^2) [1 nu 0; nu 1 0; 0 0 (1-nu)/2]          (:3383-3384)
        Cb = pshell_bending_constitutive_matrix(MID2 mat, h, br)  (:3393-3395, :2174-2181)
        Cs = TS/T * h * G * I2, G = MAT(MID3).G or E/2(1+nu)       (:2085-2129)
        E_ref = E, k6rot = PARAM K6ROT (0 for membrane-only)       (:4008)
        """
        if self.q4_sect_override is not None:
            return self.q4_sect_override
        if len(self.q4_pid) == 0:
            return np.zeros((0, Q4_SECT_STRIDE))
        # one record per PSHELL, gathered per element (a mesh with a PSHELL per
        # skin row has hundreds of them)
        pids, inv = np.unique(self.q4_pid, return_inverse=True)
        recs = np.stack([np.asarray(_q4_section_record(self, int(pid)), dtype=np.float64) for pid in pids])
        return recs[inv.reshape(-1)]

    def q4_recovery_mask(self) -> np.ndarray:
        """CQUAD4 whose stresses the reference recovers: the PSHELL's MID2 and
        MID3 (when bending is active) are MID1 or a MAT1 with the same E, NU
        and G (_pshell_local_constitutive_gap with equivalent materials,
        stress_recovery.jl:176-215)."""
        def same_law(a: int, b: int) -> bool:
            if a == b:
                return True
            ma, mb = self.mats.get(a), self.mats.get(b)
            return ma is not None and mb is not None and (ma.E, ma.NU, ma.G) == (mb.E, mb.NU, mb.G)

        ok = {}
        for pid in np.unique(self.q4_pid):
            p = self.pshells[int(pid)]
            bending = float(p.BEND_RATIO) > 1e-12
            mids = [p.MID2, p.MID3] if bending else []
            ok[int(pid)] = all(mid <= 0 or same_law(p.MID1, mid) for mid in mids)
        return np.array([ok[int(pid)] for pid in self.q4_pid], dtype=bool)

    def q8_sections(self) -> np.ndarray:
        """CQUAD8 native section (assembly.jl:2585-2628 _quad8_native_section)."""
        out = np.zeros((len(self.q8_pid), Q8_SECT_STRIDE))
        for pid in np.unique(self.q8_pid):
            p = self.pshells[int(pid)]
            t = float(p.T)

            def iso(mid):
                if mid == 0:
                    return None
                m = self.mats[mid]
                E, nu = m.E, m.NU
                return (E / (1 - nu ** 2)) * np.array([[1.0, nu, 0.0], [nu, 1.0, 0.0], [0.0, 0.0, (1 - nu) / 2]])
            Qm, Qb = iso(p.MID1), iso(p.MID2)
            rec = np.zeros(Q8_SECT_STRIDE)
            if Qm is not None:
                rec[0:9] = (t * Qm).ravel(order="F")
                rec[20] = 1.0
            shear = math.inf
            dref = 0.0
            if Qb is not None:
                Db = (float(p.BEND_RATIO) * t ** 3 / 12) * Qb
                rec[9:18] = Db.ravel(order="F")
                rec[21] = 1.0
                dref = Db[0, 0]
                if p.MID3 != 0:
                    G3 = self.mats[p.MID3].G
                    if G3 <= 0:
                        raise ValueError("CQUAD8 native path needs a MAT1 G on MID3")
                    shear = G3 * float(p.TS_T) * t
            rec[18] = shear
            rec[19] = dref
            out[self.q8_pid == pid] = rec
        return out

    def t3_sections(self) -> np.ndarray:
        """Per-element CTRIA3 section records (assembly.jl:3300-3440 with n = 3):
        the CQUAD4 record's Cm, Cb, Cs, h and k6rot; Eref = the shear modulus
        (:3389, unused by the triangle's lumped drilling); flags 0."""
        return _t3_records(self, self.t3_pid)

    # ------------------------------------------------------------------ shells as assembled
    def q8_native_mask(self) -> np.ndarray:
        """CQUAD8 that keep the native eight-node stiffness: flat parallelograms
        with mid-side nodes at the edge midpoints (assembly.jl:2585-2628,
        quad8_shell.jl:34-46, tolerance 1e-6 of the longer edge from G1)."""
        if len(self.q8_nodes) == 0:
            return np.zeros(0, bool)
        P = np.asarray(self.xyz, float)[np.asarray(self.q8_nodes)]          # (n, 8, 3)
        scale = np.maximum(np.linalg.norm(P[:, 1] - P[:, 0], axis=1), np.linalg.norm(P[:, 3] - P[:, 0], axis=1))
        lim = 1e-6 * scale
        ok = scale > 0
        ok &= np.linalg.norm(P[:, 0] + P[:, 2] - P[:, 1] - P[:, 3], axis=1) <= lim
        for m, a, b in ((4, 0, 1), (5, 1, 2), (6, 2, 3), (7, 3, 0)):
            ok &= np.linalg.norm(P[:, m] - (P[:, a] + P[:, b]) / 2, axis=1) <= lim
        nrm = np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 3] - P[:, 0]), axis=1)
        ok &= nrm > 1e-12 * scale * scale
        return ok

    def device_q8(self) -> Tuple[np.ndarray, np.ndarray]:
        """(nodes, section records) of the CQUAD8 assembled natively."""
        keep = self.q8_native_mask()
        return (np.ascontiguousarray(np.asarray(self.q8_nodes, np.int32)[keep]).reshape(-1, 8),
                np.ascontiguousarray(self.q8_sections()[keep]).reshape(-1, Q8_SECT_STRIDE))

    def device_t3(self) -> Tuple[np.ndarray, np.ndarray]:
        """(nodes, section records) of every CTRIA3 as assembled: the model's
        own, then six per CQUAD8 without the native section, in element order
        (assembly.jl:3176-3196: [1,5,8] [5,2,6] [6,3,7] [7,4,8] [5,6,8] [6,7,8])."""
        keep = self.q8_native_mask()
        split = np.asarray(self.q8_nodes, np.int32)[~keep] if len(keep) else np.zeros((0, 8), np.int32)
        sub = np.asarray(split)[:, Q8_TRIANGLES].reshape(-1, 3)
        spid = np.repeat(np.asarray(self.q8_pid)[~keep], 6) if len(keep) else np.zeros(0, np.int64)
        nodes = np.vstack([np.asarray(self.t3_nodes, np.int32).reshape(-1, 3), sub.astype(np.int32)])
        pids = np.concatenate([np.asarray(self.t3_pid, np.int64), spid.astype(np.int64)])
        return np.ascontiguousarray(nodes), np.ascontiguousarray(_t3_records(self, pids))

    def t10_materials(self) -> np.ndarray:
        out = np.zeros((len(self.t10_pid), 2))
        for pid in np.unique(self.t10_pid):
            m = self.mats[self.psolids[int(pid)]]
            out[self.t10_pid == pid] = (m.E, m.NU)
        return out

    # ------------------------------------------------------------------ loads
    def load_vector(self, case: LoadCase, q4_pressure: bool = True) -> np.ndarray:
        """Global F (ndof) for one subcase (loads.jl:541-586, solve_case.jl:57-111).

        PLOAD4 on CQUAD4: area = |(x3-x1)x(x4-x2)|/2, force p*area/4 per node
        along the normal of that cross product.  FORCE: dir*mag.  The node_R
        rotation of the reference is the identity for basic-frame grids.
        """
        F = np.zeros(self.ndof)
        nn_tot = self.n_nodes
        if case.pload4 is not None and q4_pressure:
            eidx, p = case.pload4
            nodes = self.q4_nodes[eidx]
            X = self.xyz
            d13 = X[nodes[:, 2]] - X[nodes[:, 0]]
            d24 = X[nodes[:, 3]] - X[nodes[:, 1]]
            nv = np.cross(d13, d24)
            nn = np.linalg.norm(nv, axis=1)
            area = 0.5 * nn
            ldir = nv / nn[:, None]
            tf = area * p
            fnode = ldir * (tf / 4.0)[:, None]
            Fn = F.reshape(-1, 6)
            for k in range(4):
                for a in range(3):
                    Fn[:, a] += np.bincount(nodes[:, k], weights=fnode[:, a], minlength=nn_tot)
        if case.pload4_t3 is not None:
            # CTRIA3: p A / 3 per node along (x2 - x1) x (x3 - x1) (loads.jl:546-585)
            eidx, p = case.pload4_t3
            nodes = np.asarray(self.t3_nodes)[eidx]
            X = self.xyz
            nv = np.cross(X[nodes[:, 1]] - X[nodes[:, 0]], X[nodes[:, 2]] - X[nodes[:, 0]])
            nn = np.linalg.norm(nv, axis=1)
            fnode = (nv / nn[:, None]) * (0.5 * nn * p / 3.0)[:, None]
            Fn = F.reshape(-1, 6)
            for k in range(3):
                for a in range(3):
                    Fn[:, a] += np.bincount(nodes[:, k], weights=fnode[:, a], minlength=nn_tot)
        for item in (case.forces, case.cload):
            if item is None:
                continue
            nidx, vec = item
            Fn = F.reshape(-1, 6)
            for a in range(3):
                Fn[:, a] += np.bincount(nidx, weights=vec[:, a], minlength=nn_tot)
        R = self.node_R
        if not self._identity_frames():
            Rm = R.reshape(-1, 3, 3, order="C").transpose(0, 2, 1)  # column-major -> matrix
            Fn = F.reshape(-1, 6)
            Fn[:, 0:3] = np.einsum("nji,nj->ni", Rm, Fn[:, 0:3])
            Fn[:, 3:6] = np.einsum("nji,nj->ni", Rm, Fn[:, 3:6])
            F = Fn.reshape(-1)
        return F

    def _identity_frames(self) -> bool:
        """True when every grid's displacement frame is the basic frame
        (cached against the node_R array it was computed for)."""
        R = self.node_R
        c = getattr(self, "_ident_cache", None)
        if c is None or c[0] is not R:
            ident = bool((R[:, [0, 4, 8]] == 1.0).all() and (R[:, [1, 2, 3, 5, 6, 7]] == 0.0).all())
            self._ident_cache = (R, ident)
            return ident
        return c[1]

    def load_matrix(self) -> np.ndarray:
        """ndof x nrhs column-major (Fortran order) matrix of all subcases.

        With basic-frame grids, the CQUAD4 PLOAD4 of all subcases that load
        the same element list are applied at once: the per-element nodal force
        per unit pressure (p A / 4 along the element normal, as in
        load_vector) is a sparse (3 grids x elements) operator built once and
        multiplied by the subcases' pressures."""
        cases = self.load_cases
        F = np.empty((self.ndof, len(cases)), order="F")
        batch = len(cases) > 1 and self._identity_frames()
        for k, c in enumerate(cases):
            F[:, k] = self.load_vector(c, q4_pressure=not batch)
        if batch:
            groups: Dict[int, Tuple[np.ndarray, List[int]]] = {}
            for k, c in enumerate(cases):
                if c.pload4 is not None:
                    groups.setdefault(id(c.pload4[0]), (c.pload4[0], []))[1].append(k)
            for eidx, ks in groups.values():
                A = self._pload4_operator(eidx)
                P = np.empty((A.shape[1], len(ks)))
                for j, k in enumerate(ks):
                    P[:, j] = cases[k].pload4[1]
                G = A @ P
                for j, k in enumerate(ks):
                    F[:, k].reshape(-1, 6)[:, 0:3] += G[:, j].reshape(-1, 3)
        return F

    def _pload4_operator(self, eidx: np.ndarray):
        """CSC (3 n_nodes x len(eidx)): nodal force of a unit PLOAD4 on each
        listed CQUAD4 (cached for the element list and coordinates it was built
        from)."""
        import scipy.sparse as sp
        c = getattr(self, "_p4_cache", None)
        if c is not None and c[0] is eidx and c[1] is self.xyz:
            return c[2]
        nodes = self.q4_nodes[eidx]
        X = self.xyz
        nv = np.cross(X[nodes[:, 2]] - X[nodes[:, 0]], X[nodes[:, 3]] - X[nodes[:, 1]])
        nn = np.linalg.norm(nv, axis=1)
        fdir = (nv / nn[:, None]) * (0.5 * nn / 4.0)[:, None]
        ne = len(eidx)
        # column e holds the element's 12 entries (4 grids x 3 components)
        rows = (3 * nodes[:, :, None] + np.arange(3)[None, None, :]).reshape(-1)
        vals = np.broadcast_to(fdir[:, None, :], (ne, 4, 3)).reshape(-1)
        A = sp.csc_matrix((vals, rows, np.arange(0, 12 * ne + 1, 12)), shape=(3 * self.n_nodes, ne))
        self._p4_cache = (eidx, self.xyz, A)
        return A

    def spc_dofs(self) -> np.ndarray:
        """SPC1 DOFs (boundary_conditions.jl:1499-1540)."""
        out = []
        for comps, nodes in self.spc1:
            for ch in comps:
                c = int(ch) - 1
                out.append(6 * np.asarray(nodes, np.int64) + c)
        if not out:
            return np.zeros(0, np.int64)
        return np.unique(np.concatenate(out))


# the six CTRIA3 of a CQUAD8 without the native section (assembly.jl:3187-3188)
Q8_TRIANGLES = np.array([[0, 4, 7], [4, 1, 5], [5, 2, 6], [6, 3, 7], [4, 5, 7], [5, 6, 7]])


def _t3_records(model: Sol101Model, pids: np.ndarray) -> np.ndarray:
    out = np.zeros((len(pids), Q4_SECT_STRIDE))
    for pid in np.unique(pids):
        rec = _q4_section_record(model, int(pid)).copy()
        p = model.pshells[int(pid)]
        sm = model.mats[p.MID3] if p.MID3 != 0 else model.mats[p.MID1]
        G = float(sm.G)
        if G <= 0.0:
            G = float(sm.E) / (2 * (1 + float(sm.NU))) if float(sm.E) > 0.0 else 0.0
        rec[23] = G
        rec[25] = 0.0
        out[pids == pid] = rec
    return out


def _q4_section_record(model: Sol101Model, pid: int) -> np.ndarray:
    p = model.pshells[pid]
    mat = model.mats[p.MID1]
    h = float(p.T)
    br = float(p.BEND_RATIO)
    tst = float(p.TS_T)
    E_val, nu_val = float(mat.E), float(mat.NU)
    const_mem = E_val * h / (1 - nu_val * nu_val)
    Cm = const_mem * np.array([[1.0, nu_val, 0.0], [nu_val, 1.0, 0.0], [0.0, 0.0, (1 - nu_val) / 2]])
    bend_mat = model.mats.get(p.MID2, mat) if p.MID2 != 0 else mat
    if br > 1e-12:
        Eb, nub = float(bend_mat.E), float(bend_mat.NU)
        plane_coeff = Eb / max(1.0 - nub * nub, 1e-30)
        Cb = (1.0 * plane_coeff) * np.array([[1.0, nub, 0.0], [nub, 1.0, 0.0], [0.0, 0.0, (1.0 - nub) / 2.0]])
        Cb = Cb * (br * (h * h * h) / 12.0)
    else:
        Cb = np.zeros((3, 3))
    if p.MID3 == 0:
        # PSHELL blank MID3 selects the rigid-shear MacNeal route in SOL101
        # (assembly.jl:2780-2787); the device path does not implement it.
        flags = 1.0
        shear_mat = mat
    else:
        flags = 0.0
        shear_mat = model.mats[p.MID3]
    G_val = float(shear_mat.G)
    if G_val <= 0.0:
        Es, nus = float(shear_mat.E), float(shear_mat.NU)
        G_val = Es / (2 * (1 + nus)) if Es > 0.0 else 0.0
    Cs = (tst * h) * np.array([[G_val, 0.0], [0.0, G_val]])
    if br <= 1e-12:
        Cs = np.zeros((2, 2))
    rec = np.zeros(Q4_SECT_STRIDE)
    rec[0:9] = Cm.ravel(order="F")
    rec[9:18] = Cb.ravel(order="F")
    rec[18:22] = Cs.ravel(order="F")
    rec[22] = h
    rec[23] = E_val
    rec[24] = 0.0 if br <= 1e-12 else float(model.k6rot)
    rec[25] = flags
    return rec


# ============================================================================
# Synthetic generators (seeded PCG64).  Shapes, sizes and value distributions
# follow the benchmark configurations; no reference data is embedded.
# ============================================================================

def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def flat_plate(nx: int = 20, ny: int = 20, a: float = 0.5, b: float = 0.5,
               t: float = 0.002, E: float = 70e9, nu: float = 0.33, rho: float = 2700.0,
               pressure: float = 10e3, k6rot: float = 100.0) -> Sol101Model:
    """Clamped flat plate under uniform pressure (20x20 CQUAD4, 2,646 DOF).

    GRID ids 1..(nx+1)(ny+1) row-major, z = 0; PSHELL MID1=MID2=MID3=1;
    SPC1 123456 on every edge node; PLOAD4 on every element; one subcase.
    """
    xs = np.linspace(0.0, a, nx + 1)
    ys = np.linspace(0.0, b, ny + 1)
    X, Y = np.meshgrid(xs, ys)                     # row-major in y, then x
    xyz = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    ids = np.arange(1, xyz.shape[0] + 1, dtype=np.int64)
    nid = lambda i, j: j * (nx + 1) + i
    q4 = []
    for j in range(ny):
        for i in range(nx):
            q4.append([nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)])
    q4 = np.asarray(q4, np.int32)
    edge = np.where((np.isclose(xyz[:, 0], 0) | np.isclose(xyz[:, 0], a) |
                     np.isclose(xyz[:, 1], 0) | np.isclose(xyz[:, 1], b)))[0]
    m = Sol101Model(
        name=f"flat_plate_{nx}x{ny}", grid_ids=ids, xyz=xyz,
        q4_nodes=q4, q4_pid=np.ones(len(q4), np.int64), q4_eid=np.arange(1, len(q4) + 1),
        pshells={1: PShell(T=t, MID1=1, MID2=1, MID3=1)},
        mats={1: Mat1(E=E, NU=nu, RHO=rho)}, k6rot=k6rot,
        spc1=[("123456", edge)],
        load_cases=[LoadCase(sid=1, pload4=(np.arange(len(q4)), np.full(len(q4), pressure)))],
    )
    return m


def quad8_plate(nx: int = 8, ny: int = 6, a: float = 0.4, b: float = 0.3, t: float = 0.003,
                E: float = 70e9, nu: float = 0.33, skew: float = 0.0, tilt_deg: float = 0.0,
                n_cases: int = 1, force_sigma: float = 50.0, seed: int = 11,
                taper: float = 0.0) -> Sol101Model:
    """Cantilever plate of CQUAD8 (native shell path, quad8_shell.jl).

    Corner and mid-side nodes on the (2nx+1) x (2ny+1) lattice of the
    parallelogram spanned by (a, 0) and (skew * b, b); element centres are not
    nodes.  ``taper`` narrows the half x > a/2 linearly (y scaled by
    1 - taper (u - 1/2)), so its elements are trapezoids, which the reference
    assembles as six CTRIA3 each (nx even keeps every element on one side).
    ``tilt_deg`` rotates the whole plate about the x axis and then about
    z by half that angle, so the elements lie in a general plane.  PSHELL
    MID1 = MID2 = MID3 = 1 with MAT1 G given.  SPC1 123456 on the edge x = 0.
    Subcase k: seeded N(0, force_sigma) nodal forces on every free node.
    """
    idx = {}
    pts = []
    for j in range(2 * ny + 1):
        for i in range(2 * nx + 1):
            if i % 2 == 1 and j % 2 == 1:
                continue
            u, v = i / (2 * nx), j / (2 * ny)
            idx[(i, j)] = len(pts)
            pts.append([u * a + skew * b * v, v * b * (1.0 - taper * max(0.0, u - 0.5)), 0.0])
    xyz = np.asarray(pts, float)
    if tilt_deg:
        th = math.radians(tilt_deg)
        Rx = np.array([[1, 0, 0], [0, math.cos(th), -math.sin(th)], [0, math.sin(th), math.cos(th)]])
        ph = th / 2
        Rz = np.array([[math.cos(ph), -math.sin(ph), 0], [math.sin(ph), math.cos(ph), 0], [0, 0, 1]])
        xyz = xyz @ (Rz @ Rx).T
    q8 = []
    for j in range(ny):
        for i in range(nx):
            I, J = 2 * i, 2 * j
            q8.append([idx[(I, J)], idx[(I + 2, J)], idx[(I + 2, J + 2)], idx[(I, J + 2)],
                       idx[(I + 1, J)], idx[(I + 2, J + 1)], idx[(I + 1, J + 2)], idx[(I, J + 1)]])
    q8 = np.asarray(q8, np.int32)
    clamp = np.array([idx[(0, j)] for j in range(2 * ny + 1)], np.int64)
    free = np.setdiff1d(np.arange(len(xyz)), clamp)
    rng = _rng(seed)
    cases = [LoadCase(sid=k + 1, forces=(free, rng.normal(0.0, force_sigma, (len(free), 3))))
             for k in range(n_cases)]
    return Sol101Model(
        name=f"quad8_plate_{nx}x{ny}", grid_ids=np.arange(1, len(xyz) + 1, dtype=np.int64), xyz=xyz,
        q8_nodes=q8, q8_pid=np.ones(len(q8), np.int64),
        pshells={1: PShell(T=t, MID1=1, MID2=1, MID3=1)},
        mats={1: Mat1(E=E, NU=nu, G=E / (2 * (1 + nu)))},
        spc1=[("123456", clamp)], load_cases=cases, seed=seed)


def tria_plate(nx: int = 12, ny: int = 10, a: float = 0.6, b: float = 0.5, t: float = 0.002,
               E: float = 70e9, nu: float = 0.33, jitter: float = 0.2, tilt_deg: float = 25.0,
               pressure: float = 5e3, n_cases: int = 2, force_sigma: float = 20.0,
               seed: int = 5) -> Sol101Model:
    """Cantilever plate of CQUAD4 (cells with x < a/2) and CTRIA3 (two per cell,
    alternating diagonals, x > a/2).  Interior nodes move in-plane by up to
    ``jitter`` of a cell (seeded), so the triangles are irregular; the plate is
    tilted into a general plane as in ``quad8_plate``.  SPC1 123456 on x = 0.
    Subcase 1: PLOAD4 on every CQUAD4 and CTRIA3; subcase k > 1 adds seeded
    N(0, force_sigma) nodal forces on the free nodes."""
    rng = _rng(seed)
    hx, hy = a / nx, b / ny
    pts = np.zeros(((nx + 1) * (ny + 1), 3))
    nid = lambda i, j: j * (nx + 1) + i
    for j in range(ny + 1):
        for i in range(nx + 1):
            x, y = i * hx, j * hy
            if 0 < i < nx and 0 < j < ny:
                x += jitter * hx * rng.uniform(-0.5, 0.5)
                y += jitter * hy * rng.uniform(-0.5, 0.5)
            pts[nid(i, j)] = (x, y, 0.0)
    if tilt_deg:
        th = math.radians(tilt_deg)
        Rx = np.array([[1, 0, 0], [0, math.cos(th), -math.sin(th)], [0, math.sin(th), math.cos(th)]])
        ph = th / 2
        Rz = np.array([[math.cos(ph), -math.sin(ph), 0], [math.sin(ph), math.cos(ph), 0], [0, 0, 1]])
        pts = pts @ (Rz @ Rx).T
    q4, t3 = [], []
    for j in range(ny):
        for i in range(nx):
            n1, n2, n3, n4 = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            if 2 * i < nx:
                q4.append([n1, n2, n3, n4])
            elif (i + j) % 2 == 0:
                t3 += [[n1, n2, n3], [n1, n3, n4]]
            else:
                t3 += [[n1, n2, n4], [n2, n3, n4]]
    q4 = np.asarray(q4, np.int32).reshape(-1, 4)
    t3 = np.asarray(t3, np.int32).reshape(-1, 3)
    clamp = np.array([nid(0, j) for j in range(ny + 1)], np.int64)
    free = np.setdiff1d(np.arange(len(pts)), clamp)
    cases = [LoadCase(sid=1, pload4=(np.arange(len(q4)), np.full(len(q4), pressure)),
                      pload4_t3=(np.arange(len(t3)), np.full(len(t3), pressure)))]
    for k in range(1, n_cases):
        cases.append(LoadCase(sid=k + 1, forces=(free, rng.normal(0.0, force_sigma, (len(free), 3)))))
    return Sol101Model(
        name=f"tria_plate_{nx}x{ny}", grid_ids=np.arange(1, len(pts) + 1, dtype=np.int64), xyz=pts,
        q4_nodes=q4, q4_pid=np.ones(len(q4), np.int64), q4_eid=np.arange(1, len(q4) + 1),
        t3_nodes=t3, t3_pid=np.ones(len(t3), np.int64),
        pshells={1: PShell(T=t, MID1=1, MID2=1, MID3=1)},
        mats={1: Mat1(E=E, NU=nu)}, spc1=[("123456", clamp)], load_cases=cases, seed=seed)


def wing_panel(nx: int = 200, ny: int = 400, lx: float = 1.0, ly: float = 2.0,
               n_blades: int = 9, blade_nz: int = 20, blade_h: float = 0.1,
               t_skin=(1.5e-3, 4.0e-3), t_blade: float = 3e-3, n_cases: int = 8,
               pressure: float = 5e3, edge_sigma: float = 100.0, seed: int = 1,
               E: float = 70e9, nu: float = 0.33, rho: float = 2700.0,
               k6rot: float = 100.0) -> Sol101Model:
    """Stiffened wing-box panel: skin + equally spaced blade stiffeners.

    Skin: nx x ny CQUAD4 on [0,lx] x [0,ly] at z = 0, thickness per element
    row (constant y) ~ U[t_skin] from the seed.  Blades: planes x = lx*s/(n_blades+1),
    blade_nz x ny CQUAD4 over z in [0, blade_h], sharing the skin nodes on
    z = 0.  SPC1 123456 on every node at y = 0.  Subcase k: PLOAD4 `pressure`
    on the skin plus N(0, edge_sigma) per component on the free-edge nodes
    (y = ly), seeded per subcase.  Default sizes: 152,781 nodes, 152,000 CQUAD4.
    """
    rng = _rng(seed)
    dx = lx / nx
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys)
    skin_xyz = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    n_skin = skin_xyz.shape[0]
    sid = lambda i, j: j * (nx + 1) + i
    q4 = []
    pid = []
    for j in range(ny):
        for i in range(nx):
            q4.append([sid(i, j), sid(i + 1, j), sid(i + 1, j + 1), sid(i, j + 1)])
            pid.append(100 + j)
    n_skin_el = len(q4)
    blade_cols = []
    for s in range(1, n_blades + 1):
        xb = lx * s / (n_blades + 1)
        ib = int(round(xb / dx))
        blade_cols.append(ib)
    blade_xyz = []
    next_id = n_skin
    bmap = {}
    for bi, ib in enumerate(blade_cols):
        xb = xs[ib]
        for k in range(1, blade_nz + 1):
            z = blade_h * k / blade_nz
            for j in range(ny + 1):
                bmap[(bi, k, j)] = next_id
                blade_xyz.append([xb, ys[j], z])
                next_id += 1
    xyz = np.concatenate([skin_xyz, np.asarray(blade_xyz).reshape(-1, 3)], axis=0)

    def bnode(bi, k, j):
        return sid(blade_cols[bi], j) if k == 0 else bmap[(bi, k, j)]
    for bi in range(len(blade_cols)):
        for k in range(blade_nz):
            for j in range(ny):
                q4.append([bnode(bi, k, j), bnode(bi, k, j + 1), bnode(bi, k + 1, j + 1), bnode(bi, k + 1, j)])
                pid.append(2)
    q4 = np.asarray(q4, np.int32)
    pid = np.asarray(pid, np.int64)
    t_rows = rng.uniform(t_skin[0], t_skin[1], size=ny)
    pshells = {100 + j: PShell(T=float(t_rows[j]), MID1=1, MID2=1, MID3=1) for j in range(ny)}
    pshells[2] = PShell(T=t_blade, MID1=1, MID2=1, MID3=1)
    clamp = np.where(np.isclose(xyz[:, 1], 0.0))[0]
    tip = np.where(np.isclose(xyz[:, 1], ly))[0]
    cases = []
    for c in range(n_cases):
        crng = _rng([seed, 1000 + c])
        fvec = crng.normal(0.0, edge_sigma, size=(len(tip), 3))
        cases.append(LoadCase(sid=c + 1,
                              pload4=(np.arange(n_skin_el), np.full(n_skin_el, pressure)),
                              forces=(tip, fvec)))
    return Sol101Model(
        name=f"wing_panel_{nx}x{ny}_b{n_blades}x{blade_nz}", grid_ids=np.arange(1, xyz.shape[0] + 1),
        xyz=xyz, q4_nodes=q4, q4_pid=pid, q4_eid=np.arange(1, len(q4) + 1),
        pshells=pshells, mats={1: Mat1(E=E, NU=nu, RHO=rho)}, k6rot=k6rot,
        spc1=[("123456", clamp)], load_cases=cases, seed=seed)


def wing_panel_variant(base: Sol101Model, seed: int, n_cases: int, t_skin=(1.5e-3, 4.0e-3),
                       t_blade: float = 3e-3, pressure: float = 5e3, edge_sigma: float = 100.0) -> Sol101Model:
    """A wing-box panel of the same mesh as ``base`` (a ``wing_panel``): new
    per-row skin thicknesses U[t_skin] and ``n_cases`` subcases (PLOAD4
    `pressure` on the skin plus seeded N(0, edge_sigma) forces on the free-edge
    grids), drawn from ``seed``.  The mesh arrays are shared with ``base``."""
    rng = _rng([seed, 77])
    rows = sorted(p for p in base.pshells if p >= 100)
    t_rows = rng.uniform(t_skin[0], t_skin[1], size=len(rows))
    pshells = {p: PShell(T=float(t_rows[k]), MID1=1, MID2=1, MID3=1) for k, p in enumerate(rows)}
    pshells[2] = PShell(T=t_blade, MID1=1, MID2=1, MID3=1)
    skin = np.where(base.q4_pid >= 100)[0]
    ly = base.xyz[:, 1].max()
    tip = np.where(np.isclose(base.xyz[:, 1], ly))[0]
    cases = []
    for c in range(n_cases):
        crng = _rng([seed, 1000 + c])
        cases.append(LoadCase(sid=c + 1, pload4=(skin, np.full(len(skin), pressure)),
                              forces=(tip, crng.normal(0.0, edge_sigma, size=(len(tip), 3)))))
    return Sol101Model(name=f"{base.name}_v{seed}", grid_ids=base.grid_ids, xyz=base.xyz, node_R=base.node_R,
                       q4_nodes=base.q4_nodes, q4_pid=base.q4_pid, q4_eid=base.q4_eid, pshells=pshells,
                       mats=base.mats, k6rot=base.k6rot, spc1=base.spc1, load_cases=cases, seed=seed)


_KUHN_PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
_T10_EDGES = ((0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3))


def solid_block(n: int = 40, L: float = 0.3, E: float = 210e9, nu: float = 0.3,
                traction: float = 1e6, n_cases: int = 4, sigma: float = 0.01,
                seed: int = 3) -> Sol101Model:
    """Cube split into n^3 hexes, each Kuhn-split into 6 CTETRA10.

    Corner and mid-edge nodes live on the (2n+1)^3 lattice (all used).  Base
    z = 0: SPC 123.  Top z = L: normal traction as consistent quadratic face
    loads (0 at corners, p*A/3 at midside nodes, abaqus_input.jl:383-388),
    times (1 + N(0, sigma)) per node and subcase.  Compressive (-z).
    """
    m = 2 * n + 1
    h = L / (2 * n)
    g = np.arange(m)
    I, J, K = np.meshgrid(g, g, g, indexing="ij")
    lat = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1)  # index = (i*m + j)*m + k
    xyz = lat.astype(np.float64) * h

    def lid(i, j, k):
        return (i * m + j) * m + k
    cells = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), axis=-1).reshape(-1, 3)
    tets = []
    for perm in _KUHN_PERMS:
        verts = [np.zeros(3, np.int64)]
        cur = np.zeros(3, np.int64)
        for ax in perm:
            cur = cur.copy(); cur[ax] = 1
            verts.append(cur)
        V = np.asarray(verts)  # 4 x 3 unit-cube offsets
        # orientation: det of edges from v0
        d = np.linalg.det((V[1:] - V[0]).astype(float))
        if d < 0:
            V = V[[0, 2, 1, 3]]
        corner = [2 * cells + 2 * V[q] for q in range(4)]  # lattice coords (n_cells,3)
        nodes = [lid(c[:, 0], c[:, 1], c[:, 2]) for c in corner]
        for (a, b) in _T10_EDGES:
            mid = (corner[a] + corner[b]) // 2
            nodes.append(lid(mid[:, 0], mid[:, 1], mid[:, 2]))
        tets.append(np.stack(nodes, axis=1))
    t10 = np.concatenate(tets, axis=0).astype(np.int32)
    base = np.where(lat[:, 2] == 0)[0]
    # top faces: tet faces whose 3 corners are on z = L
    top = lat[:, 2] == m - 1
    faces = ((0, 1, 2, 4, 5, 6), (0, 1, 3, 4, 8, 7), (1, 2, 3, 5, 9, 8), (0, 2, 3, 6, 9, 7))
    fz = np.zeros(xyz.shape[0])
    for f in faces:
        c = t10[:, f[:3]]
        on = top[c].all(axis=1)
        if not on.any():
            continue
        tri = t10[on][:, list(f)]
        P = xyz[tri[:, :3]]
        area = 0.5 * np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1)
        for q in range(3, 6):
            np.add.at(fz, tri[:, q], -traction * area / 3.0)
    loaded = np.where(fz != 0.0)[0]
    cases = []
    for c in range(n_cases):
        crng = _rng([seed, 2000 + c])
        scale = 1.0 + crng.normal(0.0, sigma, size=len(loaded))
        vec = np.zeros((len(loaded), 3))
        vec[:, 2] = fz[loaded] * scale
        cases.append(LoadCase(sid=c + 1, cload=(loaded, vec)))
    return Sol101Model(
        name=f"solid_block_{n}", grid_ids=np.arange(1, xyz.shape[0] + 1), xyz=xyz,
        t10_nodes=t10, t10_pid=np.ones(len(t10), np.int64), psolids={1: 1},
        mats={1: Mat1(E=E, NU=nu, RHO=7850.0)}, spc1=[("123", base)],
        load_cases=cases, seed=seed)


def stiffened_panel(seed: int, n_cases: Optional[int] = None) -> Sol101Model:
    """One batched-serving panel: skin nx,ny ~ U{8..64} CQUAD4 (10 mm), 0-6
    blades of depth U{4..8} elements, t ~ U[1,6] mm, edges clamped or simply
    supported, 1-16 subcases of PLOAD4 U[1,20] kPa + N(0,50 N) nodal forces.

    Simply supported edges take SPC 3 on the edge; when no edge is clamped,
    SPC 12 at the skin corner (0, 0) and SPC 2 at the skin corner (lx, 0)
    remove the in-plane rigid-body motions.
    """
    rng = _rng(seed)
    nx = int(rng.integers(8, 65)); ny = int(rng.integers(8, 65))
    nb = int(rng.integers(0, 7)); depth = int(rng.integers(4, 9))
    t = float(rng.uniform(1e-3, 6e-3))
    el = 0.01
    # blades: spread evenly, at least one skin element apart
    nb = min(nb, max(0, nx - 1))
    m = wing_panel(nx=nx, ny=ny, lx=nx * el, ly=ny * el, n_blades=nb, blade_nz=depth,
                   blade_h=depth * el, t_skin=(t, t), t_blade=t, n_cases=1, seed=seed)
    xyz = m.xyz
    lx, ly = nx * el, ny * el
    edges = [np.isclose(xyz[:, 0], 0) & np.isclose(xyz[:, 2], 0),
             np.isclose(xyz[:, 0], lx) & np.isclose(xyz[:, 2], 0),
             np.isclose(xyz[:, 1], 0), np.isclose(xyz[:, 1], ly)]
    spc = []
    any_clamped = False
    for e in edges:
        nodes = np.where(e)[0]
        if rng.random() < 0.5:
            spc.append(("123456", nodes)); any_clamped = True
        else:
            spc.append(("3", nodes))
    if not any_clamped:
        # in-plane rigid motions: u, v at the skin corner (0, 0) and v at the
        # skin corner (lx, 0) (the in-plane rotation about z)
        c00 = np.where(edges[0] & edges[2])[0]
        c10 = np.where(edges[1] & edges[2])[0]
        spc.append(("12", c00[:1])); spc.append(("2", c10[:1]))
    drawn = int(rng.integers(1, 17))
    n_cases = drawn if n_cases is None else int(n_cases)
    n_skin_el = nx * ny
    free_nodes = np.setdiff1d(np.arange(len(xyz)), np.concatenate([s[1] for s in spc]))
    cases = []
    for c in range(n_cases):
        p = float(rng.uniform(1e3, 20e3))
        cases.append(LoadCase(sid=c + 1, pload4=(np.arange(n_skin_el), np.full(n_skin_el, p)),
                              forces=(free_nodes, rng.normal(0.0, 50.0, size=(len(free_nodes), 3)))))
    m.spc1 = spc
    m.load_cases = cases
    m.name = f"panel_{seed}_{nx}x{ny}_b{nb}x{depth}"
    m.seed = seed
    return m


def benchmark_config(index: int, **kw) -> Sol101Model:
    """The five benchmark shapes by index (0: plate, 1: wing panel, 2: solid)."""
    if index == 0:
        return flat_plate(**kw)
    if index == 1:
        return wing_panel(**kw)
    if index == 2:
        return solid_block(**kw)
    if index == 3:
        return stiffened_panel(kw.get("seed", 0))
    raise ValueError(index)
