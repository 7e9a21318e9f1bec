"""Device parity against the CPU oracle (runs on a B200; marked gpu).

Bars: element matrices to 1e-12 relative, CSC pattern
and slot map bit-exact, displacements / SPC forces to 1e-8 relative for the
FP64 path and relative residual <= 1e-10 for both paths after refinement.
"""
import numpy as np
import pytest

from jf_2026_05_25_b200 import backend as B
from jf_2026_05_25_b200 import build as jbuild
from jf_2026_05_25_b200 import lib
from jf_2026_05_25_b200 import model as M

pytestmark = pytest.mark.gpu

ELEM_RTOL = 1e-12
DISP_RTOL = 1e-8
RESID_TOL = 1e-10


@pytest.fixture(scope="module")
def ctx():
    jbuild.build()
    c = lib.Context(0)
    yield c
    c.close()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _rot(ax, deg):
    t = np.radians(deg)
    c, s = np.cos(t), np.sin(t)
    if ax == 0:
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    if ax == 1:
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


def _random_quads(rng, n):
    """Flat convex quads (rectangles, parallelograms, tapers) in random planes."""
    out = []
    for k in range(n):
        a, b = rng.uniform(0.005, 0.05, 2)
        sk = rng.uniform(-0.3, 0.3) * b if k % 3 else 0.0
        tp = rng.uniform(-0.25, 0.25) * a if k % 4 == 1 else 0.0
        P = np.array([[0, 0], [a, 0], [a + sk + tp, b], [sk, b]], float)
        P3 = np.c_[P, np.zeros(4)]
        R = _rot(0, rng.uniform(0, 180)) @ _rot(1, rng.uniform(0, 180)) @ _rot(2, rng.uniform(0, 360))
        out.append(P3 @ R.T + rng.uniform(-1, 1, 3))
    return out


def test_quad4_element_matrices(ctx, oracle_mod):
    rng = np.random.default_rng(7)
    quads = _random_quads(rng, 48)
    xyz = np.vstack(quads)
    q4 = np.arange(4 * len(quads), dtype=np.int32).reshape(-1, 4)
    pids = np.arange(len(quads)) % 3 + 1
    m = M.Sol101Model(name="q4set", grid_ids=np.arange(1, len(xyz) + 1), xyz=xyz, q4_nodes=q4, q4_pid=pids,
                      pshells={1: M.PShell(T=0.002, MID1=1, MID2=1, MID3=1), 2: M.PShell(T=0.004, MID1=1, MID2=1, MID3=1),
                               3: M.PShell(T=0.0015, MID1=1, MID2=1, MID3=1, BEND_RATIO=0.8, TS_T=0.7)},
                      mats={1: M.Mat1(E=70e9, NU=0.33)})
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    sect = m.q4_sections()
    worst = 0.0
    for e in range(len(quads)):
        Kd = dm.element_matrix(0, e)
        Ko = oracle_mod.q4_element(xyz[q4[e]], sect[e])
        worst = max(worst, _rel(Kd, Ko))
    assert worst <= ELEM_RTOL, worst


def test_quad8_element_matrices(ctx, oracle_mod):
    """CQUAD8 parallelograms in random planes, with random node_R frames on
    half of the grids, against the oracle restatement of quad8_shell.jl."""
    rng = np.random.default_rng(5)
    xyz, q8, nodeR = [], [], []
    for e in range(24):
        a, b = rng.uniform(0.01, 0.06, 2)
        ang = rng.uniform(50, 130)
        th = np.radians(ang)
        c = np.array([[0, 0, 0], [a, 0, 0], [a + b * np.cos(th), b * np.sin(th), 0], [b * np.cos(th), b * np.sin(th), 0]])
        P = np.vstack([c, (c[0] + c[1]) / 2, (c[1] + c[2]) / 2, (c[2] + c[3]) / 2, (c[3] + c[0]) / 2])
        R = _rot(0, rng.uniform(0, 180)) @ _rot(1, rng.uniform(0, 180)) @ _rot(2, rng.uniform(0, 360))
        xyz.append(P @ R.T + rng.uniform(-1, 1, 3))
        q8.append(np.arange(8 * e, 8 * e + 8))
        for k in range(8):
            Rn = _rot(2, rng.uniform(0, 360)) @ _rot(0, rng.uniform(0, 90)) if k % 2 else np.eye(3)
            nodeR.append(Rn.ravel(order="F"))
    xyz = np.vstack(xyz)
    q8 = np.asarray(q8, np.int32)
    nodeR = np.asarray(nodeR)
    pids = np.arange(len(q8)) % 2 + 1
    m = M.Sol101Model(name="q8set", grid_ids=np.arange(1, len(xyz) + 1), xyz=xyz, node_R=nodeR, q8_nodes=q8,
                      q8_pid=pids,
                      pshells={1: M.PShell(T=0.003, MID1=1, MID2=1, MID3=1),
                               2: M.PShell(T=0.006, MID1=1, MID2=1, MID3=1, BEND_RATIO=0.9, TS_T=0.8)},
                      mats={1: M.Mat1(E=70e9, NU=0.33, G=70e9 / 2.66)})
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    sect = m.q8_sections()
    worst = 0.0
    for e in range(len(q8)):
        Kd = dm.element_matrix(1, e)
        Ko = oracle_mod.q8_element(xyz[q8[e]], sect[e], nodeR[q8[e]])
        worst = max(worst, _rel(Kd, Ko))
    assert worst <= ELEM_RTOL, worst


def test_quad8_curved_element_becomes_triangles(ctx, oracle_mod):
    # a CQUAD8 that is not a flat parallelogram is assembled as six CTRIA3,
    # as the reference does (assembly.jl:3176-3196)
    m = M.quad8_plate(2, 2)
    m.xyz = m.xyz.copy()
    m.xyz[m.q8_nodes[0, 4], 2] += 0.01       # lift a mid-side node off the edge
    assert m.q8_native_mask().tolist() == [False, True, True, True]
    asm = oracle_mod.assemble(m)
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    assert np.array_equal(dm.slot_map(), asm["slot"])
    assert np.abs(dm.values() - asm["nzval"]).max() <= ELEM_RTOL * np.abs(asm["nzval"]).max()


def test_quad8_shape_check_still_guards_the_native_kernel(ctx):
    # the C ABI refuses a non-parallelogram CQUAD8 handed to the native kernel
    m = M.quad8_plate(2, 2)
    m.xyz = m.xyz.copy()
    m.xyz[m.q8_nodes[0, 4], 2] += 0.01
    m.q8_native_mask = lambda: np.ones(len(m.q8_nodes), bool)
    dm = lib.DeviceModel(ctx, m)
    with pytest.raises(lib.JfgError) as e:
        dm.assemble()
    assert e.value.status_name == "UNSUPPORTED"
    assert e.value.detail == 0


def test_tria3_element_matrices(ctx, oracle_mod):
    rng = np.random.default_rng(17)
    xyz, t3, nodeR = [], [], []
    for k in range(96):
        # triangles from slivers to obtuse, in random planes
        a = rng.uniform(0.004, 0.05)
        apex = np.array([rng.uniform(-0.5, 1.5) * a, rng.uniform(0.05, 1.5) * a])
        P = np.c_[np.array([[0.0, 0.0], [a, 0.0], apex]), np.zeros(3)]
        R = _rot(0, rng.uniform(0, 180)) @ _rot(1, rng.uniform(0, 180)) @ _rot(2, rng.uniform(0, 360))
        xyz.append(P @ R.T + rng.uniform(-1, 1, 3))
        t3.append(np.arange(3) + 3 * k)
        for _ in range(3):
            Rn = _rot(2, rng.uniform(0, 90)) @ _rot(0, rng.uniform(0, 90)) if k % 3 == 1 else np.eye(3)
            nodeR.append(Rn.ravel(order="F"))
    xyz = np.vstack(xyz)
    t3 = np.asarray(t3, np.int32)
    nodeR = np.asarray(nodeR)
    pids = np.arange(len(t3)) % 3 + 1
    m = M.Sol101Model(name="t3set", grid_ids=np.arange(1, len(xyz) + 1), xyz=xyz, node_R=nodeR, t3_nodes=t3,
                      t3_pid=pids,
                      pshells={1: M.PShell(T=0.003, MID1=1, MID2=1, MID3=1),
                               2: M.PShell(T=0.006, MID1=1, MID2=2, MID3=0, BEND_RATIO=0.9, TS_T=0.8),
                               3: M.PShell(T=0.002, MID1=2, BEND_RATIO=0.0)},
                      mats={1: M.Mat1(E=70e9, NU=0.33), 2: M.Mat1(E=110e9, NU=0.3, G=40e9)})
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    sect = m.t3_sections()
    worst = 0.0
    for e in range(len(t3)):
        Kd = dm.element_matrix(3, e)
        Ko = oracle_mod.t3_element(xyz[t3[e]], sect[e], nodeR[t3[e]])
        worst = max(worst, _rel(Kd, Ko))
    assert worst <= ELEM_RTOL, worst


def test_tetra10_element_matrices(ctx, oracle_mod):
    m = M.solid_block(n=2, n_cases=1)
    rng = np.random.default_rng(3)
    m.xyz = m.xyz + rng.uniform(-0.01, 0.01, m.xyz.shape) * (0.3 / 4)   # curved, still valid
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    worst = 0.0
    for e in range(0, len(m.t10_nodes), 5):
        Kd = dm.element_matrix(2, e)
        Ko = oracle_mod.t10_element(m.xyz[m.t10_nodes[e]], 210e9, 0.3)
        worst = max(worst, _rel(Kd, Ko))
    assert worst <= ELEM_RTOL, worst


MODELS = {
    "plate": lambda: M.flat_plate(),
    "q8_flat": lambda: M.quad8_plate(8, 6, skew=0.3, n_cases=2),
    "q8_tilted": lambda: M.quad8_plate(6, 5, skew=0.2, tilt_deg=30, n_cases=2),
    "wing_small": lambda: M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=3, seed=5),
    "solid_small": lambda: M.solid_block(n=4, n_cases=2),
    "tria_mixed": lambda: M.tria_plate(t=0.02),   # thinner tilted plates sit above the 1e-10 FP64 residual floor
    "q8_tapered": lambda: M.quad8_plate(8, 6, taper=0.6, tilt_deg=20, n_cases=2),
}


@pytest.mark.parametrize("name", sorted(MODELS))
def test_pattern_slot_map_and_values(ctx, oracle_mod, name):
    m = MODELS[name]()
    asm = oracle_mod.assemble(m)
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    colptr, rowval = dm.pattern()
    assert np.array_equal(colptr, asm["colptr"])
    assert np.array_equal(rowval, asm["rowval"])
    assert np.array_equal(dm.slot_map(), asm["slot"])
    v = dm.values()
    scale = np.abs(asm["nzval"]).max()
    assert np.abs(v - asm["nzval"]).max() <= ELEM_RTOL * scale
    # bitwise determinism of the gather assembly
    dm.assemble()
    assert np.array_equal(dm.values(), v)


@pytest.mark.parametrize("name", sorted(MODELS))
@pytest.mark.parametrize("prec", [lib.PREC_FP64, lib.PREC_MIXED])
def test_sol101_against_oracle(ctx, oracle_mod, name, prec):
    m = MODELS[name]()
    ref = oracle_mod.solve_reference(m)
    be = B.JFEMGPUBackend(precision=prec, tol=RESID_TOL)
    be._ctx = ctx
    res = B.solve_model(be, m)
    free = res["state"]["free"]
    assert np.array_equal(free, ref["free"])
    U = np.stack([s["raw_displacement"] for s in res["subcases"]], axis=1)
    for sc in res["subcases"]:
        assert sc["solver_diagnostics"]["linear_solver"]["rel_residual"] <= RESID_TOL
    # displacement error against the FP64 oracle, relative to the field maximum
    assert _rel(U, ref["u"]) <= DISP_RTOL
    # SPC forces (residual at the fixed DOFs)
    fixed = res["state"]["fixed"]
    R_dev = np.stack([np.asarray(list(sc["spc_forces"].values())).ravel() if sc["spc_forces"] else np.zeros(0)
                      for sc in res["subcases"]][0:1])
    Rref = ref["R"][fixed]
    Rdev = res["state"]["dm"].residual(U, m.load_matrix())[fixed]
    assert _rel(Rdev, Rref) <= DISP_RTOL
    assert R_dev.size > 0


def test_factor_is_deterministic(ctx):
    m = MODELS["wing_small"]()
    be = B.JFEMGPUBackend()
    be._ctx = ctx
    st = B.prepare(be, m)
    dm = st["dm"]
    d1 = dm.factor_diag()
    F = m.load_matrix()
    U1, _ = dm.solve(F)
    dm.factor(lib.PREC_FP64)
    d2 = dm.factor_diag()
    U2, _ = dm.solve(F)
    assert np.array_equal(d1, d2)
    assert np.array_equal(U1, U2)


def test_not_spd_reports_pivot(ctx):
    """A free rigid-body mode (no SPC, GPST off by eps 0) must surface as NOT_SPD."""
    m = M.flat_plate(nx=4, ny=4)
    m.spc1 = []
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    free = np.arange(m.ndof, dtype=np.int32)
    dm.set_free_dofs(free)
    with pytest.raises(lib.JfgError) as e:
        dm.factor(lib.PREC_FP64)
    assert e.value.status_name == "NOT_SPD"


def test_thickness_update_resolve(ctx, oracle_mod):
    m = MODELS["plate"]()
    be = B.JFEMGPUBackend()
    be._ctx = ctx
    st = B.prepare(be, m)
    dm = st["dm"]
    m.pshells[1] = M.PShell(T=0.0025, MID1=1, MID2=1, MID3=1)
    sect = m.q4_sections()
    dm.update_q4_sections(np.arange(len(sect)), sect)
    dm.assemble()
    dm.factor(lib.PREC_FP64)
    U, rep = dm.solve(m.load_matrix())
    ref = oracle_mod.solve_reference(m)
    assert _rel(U, ref["u"]) <= DISP_RTOL


def test_tensor_core_front_updates(ctx, monkeypatch):
    """The tcgen05 3xTF32 front-update kernel (switched on with
    JFG_TENSOR_CORES=1; JFG_TC_MIN=128 hands it the panel and Schur updates
    of every level with 128 output rows or more) against the SIMT FP32
    kernel on a model whose fronts span several 128 x 128 tiles.  The split
    v = trunc19(v) + rn19(lo) and the missing lo*lo term make the tensor-core
    factor a slightly weaker preconditioner than the FP32 one (one-sided
    errors of about 2^-21 per product on sums of squares): its diagonal stays
    within 1e-4 of the FP64 factor's, both mixed solves refine to the FP64
    residual bar and the FP64 displacements, the tensor-core one in at most
    one more refinement step."""
    m = M.solid_block(n=8, n_cases=1)
    F = m.load_matrix()
    be = B.JFEMGPUBackend(precision=lib.PREC_FP64)
    be._ctx = ctx
    st = B.prepare(be, m)
    d64 = st["dm"].factor_diag()
    U64, _ = st["dm"].solve(F, tol=RESID_TOL)
    monkeypatch.setenv("JFG_TC_MIN", "128")
    err, its = {}, {}
    for flag in ("0", "1"):
        monkeypatch.setenv("JFG_TENSOR_CORES", flag)
        be = B.JFEMGPUBackend(precision=lib.PREC_MIXED)
        be._ctx = ctx
        st = B.prepare(be, m)
        d = st["dm"].factor_diag()
        U, rep = st["dm"].solve(F, tol=RESID_TOL, max_ir=30)
        assert rep["rel_residual"] <= RESID_TOL
        assert rep["fallback_used"] == 0
        assert _rel(U, U64) <= DISP_RTOL
        err[flag] = (np.abs(d - d64) / np.abs(d64)).max()
        its[flag] = rep["ir_iters"]
    assert err["0"] <= 1e-4, err
    assert err["1"] <= 1e-4, err
    assert its["1"] <= its["0"] + 1, its


def test_dmma_front_update_matches_simt(ctx, monkeypatch):
    """The FP64 tensor-core (DMMA) update kernel against the SIMT FP64
    kernel (JFG_DMMA=0): the same factor diagonal to FP64 rounding and the
    same displacements."""
    m = M.solid_block(n=8, n_cases=1)
    F = m.load_matrix()
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("JFG_DMMA", flag)
        be = B.JFEMGPUBackend(precision=lib.PREC_FP64)
        be._ctx = ctx
        st = B.prepare(be, m)
        U, rep = st["dm"].solve(F, tol=RESID_TOL)
        assert rep["rel_residual"] <= RESID_TOL
        out[flag] = (st["dm"].factor_diag(), U)
    rel = np.abs(out["1"][0] - out["0"][0]) / np.abs(out["0"][0])
    assert rel.max() <= 1e-10, rel.max()
    assert _rel(out["1"][1], out["0"][1]) <= 1e-10


LARGE = {
    # 25^3 lattice of CTETRA10 grids, 45,000 free DOF
    "solid_12": lambda: M.solid_block(n=12, n_cases=2),
    # 80 x 120 skin + 9 blades of 8 x 120: 110,160 free DOF
    "wing_110k": lambda: M.wing_panel(nx=80, ny=120, blade_nz=8, n_cases=3, seed=9),
}


@pytest.fixture(scope="module")
def large_refs(oracle_mod):
    return {}


@pytest.mark.parametrize("name", sorted(LARGE))
@pytest.mark.parametrize("prec", [lib.PREC_FP64, lib.PREC_MIXED])
def test_sol101_large_against_oracle(ctx, oracle_mod, large_refs, name, prec):
    """Displacements of a CTETRA10 block and a >100k-DOF stiffened panel
    against the FP64 oracle (its own partition, ordering and supernodal
    Cholesky, refined with compensated residuals): 1e-8 relative to the field
    maximum for the FP64 and the mixed path, relative residual <= 1e-10."""
    m = LARGE[name]()
    if name not in large_refs:
        large_refs[name] = oracle_mod.solve_reference_chol(m)
    ref = large_refs[name]
    be = B.JFEMGPUBackend(precision=prec, tol=RESID_TOL, max_ir=40)
    be._ctx = ctx
    res = B.solve_model(be, m)
    assert np.array_equal(res["state"]["free"], ref["free"])
    U = np.stack([s["raw_displacement"] for s in res["subcases"]], axis=1)
    for sc in res["subcases"]:
        assert sc["solver_diagnostics"]["linear_solver"]["rel_residual"] <= RESID_TOL
    assert _rel(U, ref["u"]) <= DISP_RTOL
    fixed = res["state"]["fixed"]
    Rdev = res["state"]["dm"].residual(U, m.load_matrix())[fixed]
    assert _rel(Rdev, ref["R"][fixed]) <= DISP_RTOL
    res["state"]["dm"].close()


def _soft_root_plate():
    """A plate clamped along y = 0 through one row of elements 1e-3 times as
    thick as the rest: every grid's own 3x3 blocks are well conditioned (no
    AUTOSPC, no grid-point singularity), but the stiff part's rotations about
    the root line are held only by the soft row's bending (thickness cubed,
    1e-9), so in any elimination order two or three pivot ratios L_ii^2 / K_ii
    come out near 1e-10 while the next smallest stays above 1e-3."""
    m = M.flat_plate(nx=6, ny=6)
    soft = np.where(m.xyz[m.q4_nodes[:, 0], 1] < 1e-12)[0]
    m.q4_pid = m.q4_pid.copy()
    m.q4_pid[soft] = 2
    m.pshells[2] = M.PShell(T=2e-6, MID1=1, MID2=1, MID3=1)
    clamp = np.where(m.xyz[:, 1] < 1e-12)[0]
    m.spc1 = [("123456", clamp)]
    return m


def test_post_factor_pivot_check_refactors(ctx, oracle_mod):
    """The post-factorisation singular-pivot check of boundary_conditions.jl:
    1662-1710: DOFs whose pivot ratio L_ii^2 / K_ii falls below 1e-7 join the
    fixed set and K_ff is factored again.  The refactored solve meets the
    residual bar and matches the oracle on the same reduced free set."""
    m = _soft_root_plate()
    be = B.JFEMGPUBackend(tol=RESID_TOL)
    be._ctx = ctx
    res = B.solve_model(be, m)
    st = res["state"]
    n_sing = st["bc"]["post_factorization_singular_dofs"]
    assert n_sing > 0
    # the first factor's partition fixed only the SPC1 DOFs
    assert len(st["fixed"]) == len(m.spc_dofs()) + n_sing
    for sc in res["subcases"]:
        assert sc["solver_diagnostics"]["linear_solver"]["rel_residual"] <= RESID_TOL
    U = np.stack([s["raw_displacement"] for s in res["subcases"]], axis=1)
    assert np.all(U[st["fixed"]] == 0.0)
    ref = oracle_mod.solve_reference(m, free=st["free"])
    assert _rel(U, ref["u"]) <= DISP_RTOL
    st["dm"].close()


def test_warped_quad4_is_refused(ctx):
    """A warped CQUAD4 (grid out of the element plane) is outside the device's
    flat-element path: UNSUPPORTED, with the index of an offending element."""
    m = M.flat_plate(nx=4, ny=4)
    centre = int(np.argmin(np.linalg.norm(m.xyz - [0.25, 0.25, 0.0], axis=1)))
    m.xyz = m.xyz.copy()
    m.xyz[centre, 2] = 1e-3
    touching = set(np.where((m.q4_nodes == centre).any(axis=1))[0].tolist())
    dm = lib.DeviceModel(ctx, m)
    with pytest.raises(lib.JfgError) as e:
        dm.assemble()
    assert e.value.status_name == "UNSUPPORTED"
    assert e.value.detail in touching
    dm.close()


def test_non_default_quad4_flags_are_refused(ctx):
    """A PSHELL with blank MID3 selects the rigid transverse-shear route of the
    reference (assembly.jl:2780-2787), which the device does not implement:
    UNSUPPORTED with the index of an element of that property."""
    m = M.flat_plate(nx=4, ny=4)
    m.q4_pid = m.q4_pid.copy()
    m.q4_pid[5:] = 2
    m.pshells[2] = M.PShell(T=0.002, MID1=1, MID2=1, MID3=0)
    dm = lib.DeviceModel(ctx, m)
    with pytest.raises(lib.JfgError) as e:
        dm.assemble()
    assert e.value.status_name == "UNSUPPORTED"
    assert e.value.detail >= 5
    dm.close()


def test_t10_stress_recovery_matches_oracle(ctx, oracle_mod):
    """Device CTETRA10 centroid stresses, strains and von Mises
    (stress_recovery.jl:1823-1960) against the oracle on random displacement
    fields with rotated grid frames: 1e-12 relative to each field's maximum."""
    m = M.solid_block(n=3, n_cases=1)
    rng = np.random.default_rng(4)
    R = np.zeros((m.n_nodes, 9))
    for i in range(m.n_nodes):
        Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        R[i] = Q.ravel(order="F")
    m.node_R = R
    U = rng.normal(scale=1e-4, size=(m.ndof, 3))
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    got = dm.t10_stresses(U)
    ref = oracle_mod.t10_stresses(m, U)
    for a, b in ((0, 6), (6, 12), (12, 13)):
        assert _rel(got[..., a:b], ref[..., a:b]) <= ELEM_RTOL
    u1 = U[:, :1].copy(order="F")
    out = np.empty(13)
    with pytest.raises(lib.JfgError) as e:
        lib._check(lib.load().jfg_recover_stresses(dm.h, 1, 1, lib._p(u1), lib._p(out)))
    assert e.value.status_name == "UNSUPPORTED"
    dm.close()


# the CQUAD4 record's field groups: forces N, M, Q; the two fibres' stresses;
# membrane strain and curvature; the principal stress at -T/2
Q4_STRESS_GROUPS = ((0, 3), (3, 6), (6, 8), (8, 14), (14, 20), (20, 25), (25, 30), (30, 31))


def test_q4_stress_recovery_matches_oracle(ctx, oracle_mod):
    """Device CQUAD4 centre forces, fibre stresses and strains
    (recover_shell_stresses!, stress_recovery.jl:505-1237) against the
    oracle on random displacement fields with rotated grid frames, and on a
    solved stiffened panel: 1e-10 relative to each field group's maximum.
    The device takes Q from the MacNeal operator of its prep record and the
    Wilson-mode condensation in a different order than the oracle."""
    m = M.stiffened_panel(3)
    rng = np.random.default_rng(5)
    R = np.zeros((m.n_nodes, 9))
    for i in range(m.n_nodes):
        Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        R[i] = Q.ravel(order="F")
    m.node_R = R
    U = rng.normal(scale=1e-4, size=(m.ndof, 3))
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    got = dm.q4_stresses(U)
    ref = oracle_mod.q4_stresses(m, U)
    assert got.shape == ref.shape == (3, len(m.q4_nodes), 31)
    for a, b in Q4_STRESS_GROUPS:
        assert _rel(got[..., a:b], ref[..., a:b]) <= 1e-10, (a, b)
    dm.close()
    # a solved model: pressure and forces on the stiffened panel
    m = M.stiffened_panel(4)
    st = B.prepare(B.JFEMGPUBackend(tol=1e-10), m)
    U, _ = st["dm"].solve(m.load_matrix(), 1e-10, 30)
    got = st["dm"].q4_stresses(U)
    ref = oracle_mod.q4_stresses(m, U)
    for a, b in Q4_STRESS_GROUPS:
        assert _rel(got[..., a:b], ref[..., a:b]) <= 1e-10, (a, b)
    assert np.abs(got[..., 3:6]).max() > 0 and np.abs(got[..., 6:8]).max() > 0
    st["dm"].close()


def test_share_structure_gives_the_same_solution(ctx):
    """A second model of the same mesh (other thicknesses and loads) that
    takes over a resident model's pattern and symbolic analysis
    (jfg_model_share_structure) solves bit-for-bit like the same model
    analysed on its own; a different mesh is refused."""
    a = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=2, seed=5)
    b = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=2, seed=6)
    be = B.JFEMGPUBackend(tol=RESID_TOL)
    be._ctx = ctx
    st_a = B.prepare(be, a)
    alone = B.solve_model(be, b)
    U_alone = np.stack([sc["raw_displacement"] for sc in alone["subcases"]], axis=1)
    dm = lib.DeviceModel(ctx, b)
    dm.share_structure(st_a["dm"])
    dm.assemble()
    d, _ = dm.diag()
    free, fixed, _ = B.compute_free_dofs(b, d, dm.node_blocks())
    assert np.array_equal(free, st_a["free"])
    dm.set_free_dofs(free)
    assert np.array_equal(dm.perm(), st_a["dm"].perm())
    dm.factor(lib.PREC_FP64)
    U, rep = dm.solve(b.load_matrix())
    assert np.array_equal(U, U_alone)
    other = lib.DeviceModel(ctx, M.wing_panel(nx=20, ny=36, n_blades=3, blade_nz=4, n_cases=1))
    with pytest.raises(lib.JfgError) as e:
        other.share_structure(st_a["dm"])
    assert e.value.status_name == "BAD_INPUT"
    for x in (dm, other, st_a["dm"], alone["state"]["dm"]):
        x.close()


def test_async_factor_and_apply_on_a_caller_stream(ctx):
    """jfg_factor_async / jfg_apply_factor_async enqueue on the caller's
    stream and return; after jfg_wait the single factor application equals
    the refined solve within the parity bar, and a deferred pivot failure is
    reported by jfg_wait."""
    import torch
    m = M.flat_plate()
    be = B.JFEMGPUBackend(tol=RESID_TOL)
    be._ctx = ctx
    st = B.prepare(be, m)
    dm = st["dm"]
    F = m.load_matrix()
    U_ref, _ = dm.solve(F)
    s = torch.cuda.Stream()
    Fd = torch.from_numpy(np.ascontiguousarray(F.T)).cuda()
    Ud = torch.full_like(Fd, float("nan"))
    torch.cuda.synchronize()
    for prec in (lib.PREC_FP64, lib.PREC_MIXED):
        dm.assemble()
        dm.factor_async(prec, s.cuda_stream)
        dm.apply_factor_async(Fd.data_ptr(), Ud.data_ptr(), F.shape[1], s.cuda_stream)
        dm.wait()
        s.synchronize()
        U = Ud.cpu().numpy().T
        if prec == lib.PREC_FP64:
            assert _rel(U, U_ref) <= DISP_RTOL
        else:
            # one application of the FP32 factor: a preconditioner, not a solve
            free = st["free"]
            R = dm.residual(np.asfortranarray(U), F)[free]
            assert np.linalg.norm(R) <= 1e-2 * np.linalg.norm(F[free])
    bad = M.flat_plate(nx=4, ny=4)
    bad.spc1 = []
    dmb = lib.DeviceModel(ctx, bad)
    dmb.assemble()
    dmb.set_free_dofs(np.arange(bad.ndof, dtype=np.int32))
    dmb.factor_async(lib.PREC_FP64, s.cuda_stream)
    with pytest.raises(lib.JfgError) as e:
        dmb.wait()
    assert e.value.status_name == "NOT_SPD"
    for x in (dm, dmb):
        x.close()


@pytest.mark.parametrize("prec", [lib.PREC_FP64, lib.PREC_MIXED])
def test_wide_right_hand_side_sweeps_match_narrow(ctx, oracle_mod, prec):
    """24 load cases go through the 32-column solve kernels in one sweep; the
    result equals three separate solves of 8 (8-column kernels) and the FP64
    oracle within the parity bar."""
    m = M.stiffened_panel(3, n_cases=24)
    be = B.JFEMGPUBackend(precision=prec, tol=RESID_TOL)
    be._ctx = ctx
    st = B.prepare(be, m)
    dm = st["dm"]
    F = m.load_matrix()
    U, rep = dm.solve(F, RESID_TOL, 40)
    assert rep["rel_residual"] <= RESID_TOL
    parts = [dm.solve(np.asfortranarray(F[:, k:k + 8]), RESID_TOL, 40)[0] for k in (0, 8, 16)]
    assert _rel(U, np.hstack(parts)) <= DISP_RTOL
    ref = oracle_mod.solve_reference(m)
    assert _rel(U, ref["u"]) <= DISP_RTOL
    dm.close()


@pytest.mark.parametrize("prec", [lib.PREC_FP64, lib.PREC_MIXED])
def test_memory_figure_predicts_the_allocations(ctx, prec):
    """jfg_get_memory's figure for a factorisation and an 8-column solve,
    taken right after the analysis, equals the bytes the model holds once
    both have run; and the device's free memory fell by at least that much
    (allocations round up)."""
    import torch
    m = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=8, seed=5)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    dm = lib.DeviceModel(ctx, m)
    dm.assemble()
    d, _ = dm.diag()
    free, _, _ = B.compute_free_dofs(m, d, dm.node_blocks())
    dm.set_free_dofs(free)
    now0, peak = dm.memory(prec, 8)
    assert peak > now0 > 0
    dm.factor(prec)
    dm.solve(m.load_matrix(), RESID_TOL, 40, raise_on_stall=False)
    now1, _ = dm.memory(prec, 8)
    assert now1 == peak
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 >= 0.95 * now1
    dm.close()
