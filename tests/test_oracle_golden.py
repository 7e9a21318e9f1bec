"""The CPU oracle against the reference's own golden vectors and known answers."""
import json
import os

import numpy as np
import pytest

from jf_2026_05_25_b200 import model as M

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _q8_nodes(a, b, ang):
    r = np.radians(ang)
    c = np.array([[0, 0, 0], [a, 0, 0], [a + b * np.cos(r), b * np.sin(r), 0], [b * np.cos(r), b * np.sin(r), 0]], float)
    return np.vstack([c, (c[0] + c[1]) / 2, (c[1] + c[2]) / 2, (c[2] + c[3]) / 2, (c[3] + c[0]) / 2])


def q8_section(E, nu, t, mid3=True):
    Q = E / (1 - nu ** 2) * np.array([[1, nu, 0], [nu, 1, 0], [0, 0, (1 - nu) / 2]])
    s = np.zeros(22)
    s[0:9] = (t * Q).ravel(order="F")
    s[9:18] = ((t ** 3 / 12) * Q).ravel(order="F")
    s[18] = E / (2 * (1 + nu)) * t * 5 / 6 if mid3 else np.inf
    s[19] = E * t ** 3 / (12 * (1 - nu ** 2))
    s[20] = s[21] = 1
    return s


def test_quad8_reference_entries(oracle_mod):
    """CQUAD8 entries of an external reference solver (quad8_shell_test.jl:24-46, rtol 2e-6)."""
    g = json.load(open(os.path.join(GOLD, "quad8_entries.json")))
    for name, cs in g["cases"].items():
        K = oracle_mod.q8_element(_q8_nodes(cs["a"], cs["b"], cs["angle"]), q8_section(g["E"], cs["nu"], cs["t"], cs["mid3"]))
        for g1, d1, g2, d2, v in g["tables"][name]:
            assert K[6 * (g1 - 1) + d1 - 1, 6 * (g2 - 1) + d2 - 1] == pytest.approx(v, rel=g["rtol"])


def test_quad8_structure(oracle_mod):
    xyz = _q8_nodes(0.4, 0.25, 70.0)
    K = oracle_mod.q8_element(xyz, q8_section(7e10, 0.3, 0.004))
    assert np.array_equal(K, K.T)
    drill = [6 * k + 5 for k in range(8)]
    assert np.all(K[drill, :] == 0)
    u = np.zeros(48)
    for k in range(8):
        u[6 * k] = 1e-3 * xyz[k, 0]
        u[6 * k + 1] = -0.3 * 1e-3 * xyz[k, 1]
    area = 0.4 * 0.25 * np.sin(np.radians(70.0))
    assert u @ K @ u == pytest.approx(7e10 * 0.004 * 1e-6 * area, rel=1e-10)


def test_tetra10_energies(oracle_mod):
    """tetra10_test.jl:45-80: constant-strain patch and quadratic field energies."""
    X = np.array([[0, 0, 0], [2, 0, 0], [0, 3, 0], [0, 0, 4.]])
    edges = ((0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3))
    X10 = np.vstack([X] + [(X[i] + X[j]) / 2 for i, j in edges])
    E, nu, V = 210e9, 0.29, 4.0
    K = oracle_mod.t10_element(X10, E, nu)
    assert np.array_equal(K, K.T)
    A = np.array([[.002, .001, -.0004], [-.0002, -.0007, .0003], [.0008, -.0006, .0011]])
    u = (X10 @ A.T).ravel()
    strain = np.array([A[0, 0], A[1, 1], A[2, 2], A[0, 1] + A[1, 0], A[1, 2] + A[2, 1], A[2, 0] + A[0, 2]])
    c = E / ((1 + nu) * (1 - 2 * nu))
    D = np.zeros((6, 6)); D[:3, :3] = c * nu; np.fill_diagonal(D[:3, :3], c * (1 - nu))
    D[3, 3] = D[4, 4] = D[5, 5] = c * (1 - 2 * nu) / 2
    assert u @ K @ u == pytest.approx(V * strain @ D @ strain, rel=2e-14)
    q = np.zeros(30); q[0::3] = X10[:, 0] ** 2
    assert q @ K @ q == pytest.approx(1.6 * V * D[0, 0], rel=2e-14)
    R = np.zeros((30, 6))
    for i, (x, y, z) in enumerate(X10):
        R[3 * i:3 * i + 3, 0:3] = np.eye(3)
        R[3 * i:3 * i + 3, 3] = [0, -z, y]; R[3 * i:3 * i + 3, 4] = [z, 0, -x]; R[3 * i:3 * i + 3, 5] = [-y, x, 0]
    assert np.linalg.norm(K @ R) < 2e-14 * np.linalg.norm(K) * np.linalg.norm(R)


@pytest.mark.parametrize("a,b", [(1., 1.), (1., .6), (8., .1), (.1, 8.)])
def test_quad4_section_kinematic_energies(oracle_mod, a, b):
    """quad4_section_kinematic_enrichment_test.jl:6-45 (k6rot=0, independent A and D)."""
    h = .004
    A = 1e7 * np.array([[7., 1.4, 0.], [1.4, 3., 0.], [0., 0., 1.8]])
    D = np.array([[18., 5., 1.1], [5., 8., -.7], [1.1, -.7, 4.]])
    S = np.eye(2) * 1e6
    x = np.array([[0., 0.], [a, 0.], [a, b], [0., b]])
    K = oracle_mod.q4_local(x, A, D, S, h, 0.0)
    qx = np.zeros(24); qy = np.zeros(24); g = np.array([1., -1., 1., -1.]) / 2
    for i in range(4):
        qx[6 * i + 3] = g[i]; qy[6 * i + 4] = g[i]
    rx = A[0, 1] / A[0, 0]; ry = A[0, 1] / A[1, 1]
    ex = (D[1, 1] - 2 * D[0, 1] * rx + D[0, 0] * rx ** 2) * a / (3 * b)
    ey = (D[0, 0] - 2 * D[0, 1] * ry + D[1, 1] * ry ** 2) * b / (3 * a)
    assert qx @ K @ qx == pytest.approx(ex, rel=1e-10)
    assert qy @ K @ qy == pytest.approx(ey, rel=1e-10)
    assert abs(qx @ K @ qy) < 1e-9 * np.linalg.norm(D)
    assert np.linalg.eigvalsh(0.5 * (K + K.T)).min() >= -3e-12 * np.linalg.norm(K, 2)
    assert np.linalg.norm(K - K.T) <= 3e-12 * np.linalg.norm(K)
    P = np.zeros((24, 3))
    for i in range(4):
        xx, yy = x[i]; j = 6 * i
        P[j + 2] = [-xx ** 2 / 2, -yy ** 2 / 2, -xx * yy / 2]; P[j + 3] = [0., -yy, -xx / 2]; P[j + 4] = [xx, 0., yy / 2]
    assert np.allclose(P.T @ K @ P, a * b * D, rtol=1e-9, atol=1e-9 * np.abs(a * b * D).max())


def _deck_model(d, mid3_from_mid1=True):
    gids = np.array(sorted(int(k) for k in d["grids"]))
    idx = {int(k): i for i, k in enumerate(gids)}
    xyz = np.array([d["grids"][str(i)] for i in gids])
    q4 = np.array([[idx[n] for n in e[2]] for e in d["cquad4"]], np.int32)
    mt, ps = d["mat1"], d["pshell"]
    m = M.Sol101Model(name="deck", grid_ids=gids, xyz=xyz, q4_nodes=q4, q4_pid=np.full(len(q4), ps["PID"]),
                      pshells={ps["PID"]: M.PShell(T=ps["T"], MID1=ps["MID1"], MID2=ps["MID2"], MID3=ps["MID1"])},
                      mats={mt["MID"]: M.Mat1(E=mt["E"], NU=mt["NU"], G=mt["G"])}, k6rot=d["k6rot"],
                      spc1=[(s[0], np.array([idx[n] for n in s[1]])) for s in d["spc1"]])
    m.load_cases = [M.LoadCase(sid=1, forces=(np.array([idx[f[0]] for f in d["force"]]),
                                              np.array([f[1] * np.array(f[2]) for f in d["force"]])))]
    return m, idx


@pytest.mark.parametrize("case", ["MH_curved_beam_in_plane", "MH_curved_beam_refined"])
def test_curved_beam_current_source_scalar(oracle_mod, case):
    """Flat tapered CQUAD4 membrane: the reference's SOL101 result with the
    present source (validation/comparison.csv, 12 significant digits).  The
    out-of-plane block is decoupled and unloaded, so MID3 does not enter."""
    g = json.load(open(os.path.join(GOLD, "curved_beam_membrane.json")))
    c = g["cases"][case]
    m, idx = _deck_model(c["deck"])
    res = oracle_mod.solve_reference(m)
    v = res["u"][6 * idx[c["node"]] + c["dof"] - 1, 0]
    assert v == pytest.approx(c["jfem_current"], rel=1e-9)


def _mystran_model():
    g = json.load(open(os.path.join(GOLD, "mystran_sol101_simple.json")))
    md = g["model"]
    gids = np.array(sorted(int(k) for k in md["grids"]))
    idx = {int(k): i for i, k in enumerate(gids)}
    xyz = np.array([md["grids"][str(i)] for i in gids])
    ps, mt = md["pshell"], md["mat1"]
    m = M.Sol101Model(name="mystran", grid_ids=gids, xyz=xyz,
                      q4_nodes=np.array([[idx[n] for n in md["cquad4"][2]]], np.int32), q4_pid=np.array([91]),
                      pshells={91: M.PShell(T=ps["T"], MID1=20, MID2=20, MID3=20, BEND_RATIO=1.0, TS_T=ps["TS_T"])},
                      mats={20: M.Mat1(E=mt["E"], NU=mt["NU"], G=mt["G"])}, k6rot=0.0,
                      spc1=[("123456", np.array([idx[1011], idx[1012]]))])
    f = md["subcases"][0]["force"]
    m.load_cases = [M.LoadCase(sid=1, forces=(np.array([idx[a] for a, _, _ in f]),
                                              np.array([mag * np.array(dv) for _, mag, dv in f]))),
                    M.LoadCase(sid=2, pload4=(np.array([0]), np.array([1.1]))),
                    M.LoadCase(sid=3, pload4=(np.array([0]), np.array([1.1])))]
    return m, idx, g


def test_mystran_current_source_scalar(oracle_mod):
    """T1 at GRID 1013 of the MYSTRAN patch, present source (comparison.csv)."""
    m, idx, _ = _mystran_model()
    cur = json.load(open(os.path.join(GOLD, "curved_beam_membrane.json")))["mystran_T1_node_1013_current"]
    res = oracle_mod.solve_reference(m)
    assert res["u"][6 * idx[1013], 0] == pytest.approx(cur, rel=1e-12)


def test_mystran_recorded_revision_sanity(oracle_mod):
    """The JU.JSON of this case keeps an older recorded revision (the changelog
    notes later element corrections); the present element must stay within
    the drift that those corrections introduced (membrane 0.3 %, plate 0.06 %)."""
    m, idx, g = _mystran_model()
    res = oracle_mod.solve_reference(m)
    for k, tol in ((0, 5e-3), (1, 1e-3), (2, 1e-3)):
        for gid, vals in g["results"][k]["displacements"].items():
            ref = np.array(vals)
            mine = res["u"][6 * idx[int(gid)]:6 * idx[int(gid)] + 6, k]
            scale = max(np.abs(ref).max(), 1e-30)
            assert np.abs(mine - ref).max() <= tol * scale
    assert res["rel_residual"].max() < 1e-12


# ---------------------------------------------------------------------------
# CQUAD4 drilling, bending and patch pins from the reference's own unit tests
# ---------------------------------------------------------------------------

def _isapprox(x, y, rtol, atol=0.0):
    """Julia's isapprox for arrays: norm(x - y) <= max(atol, rtol * max(norm(x), norm(y)))."""
    return np.linalg.norm(x - y) <= max(atol, rtol * max(np.linalg.norm(x), np.linalg.norm(y)))


def _dn(r, s):
    return np.array([[-(1 - s), 1 - s, 1 + s, -(1 + s)], [-(1 - r), -(1 + r), 1 + r, 1 - r]]) / 4.0


def independent_drill(x, Cm, k):
    """Closed-form lumped drilling penalty of utils/test/quad4_offset_drilling_test.jl:7-16.

    alpha = k * 1e-6 * Cm[2,2] * 4|det J0|; at each corner i the constraint row
    b has 1/2 dN/dy on u, -1/2 dN/dx on v and 1 on theta_z of node i, weighted
    by |det J_i| / |det J0|."""
    J0 = _dn(0.0, 0.0) @ x
    alpha = k * 1e-6 * Cm[2, 2] * 4.0 * abs(np.linalg.det(J0))
    D = np.zeros((24, 24))
    for i, (r, s) in enumerate(((-1., -1.), (1., -1.), (1., 1.), (-1., 1.))):
        J = _dn(r, s) @ x
        grad = np.linalg.solve(J, _dn(r, s))
        b = np.zeros(24)
        for j in range(4):
            b[6 * j] = grad[1, j] / 2
            b[6 * j + 1] = -grad[0, j] / 2
        b[6 * i + 5] = 1.0
        D += alpha * abs(np.linalg.det(J)) / max(abs(np.linalg.det(J0)), 1e-30) * np.outer(b, b)
    return D


_DRILL_SHAPES = (np.array([[0., 0.], [1., 0.], [1., .6], [0., .6]]),
                 np.array([[0., 0.], [.7, 0.], [1.1, .5], [.4, .5]]),
                 np.array([[0., 0.], [1., 0.], [.8, .6], [.1, .6]]))


def _drill_laws(h, anisotropic):
    """quad4_offset_drilling_test.jl:17-21."""
    if anisotropic:
        Q = 1e9 * np.array([[110., 22., 6.], [22., 40., -3.], [6., -3., 20.]])
    else:
        Q = 70e9 / (1 - .3 ** 2) * np.array([[1., .3, 0.], [.3, 1., 0.], [0., 0., .35]])
    return h * Q, h ** 3 / 12 * Q, (5 / 6) * (70e9 / 2.6) * h * np.eye(2)


@pytest.mark.parametrize("aniso", [False, True], ids=["isotropic", "anisotropic"])
@pytest.mark.parametrize("h", [.0015, .03])
@pytest.mark.parametrize("shape", [0, 1, 2])
def test_quad4_drilling_is_the_independent_closed_form(oracle_mod, shape, h, aniso):
    """K(k6rot) - K(0) equals the independent drilling matrix for k6rot = 0, 1,
    100 at the reference test's tolerance (quad4_offset_drilling_test.jl:42-47:
    rtol 2e-9, atol 2e-7).  K6ROT = 100 is the default of every benchmark model."""
    x = _DRILL_SHAPES[shape]
    A, B, Cs = _drill_laws(h, aniso)
    K0 = oracle_mod.q4_local(x, A, B, Cs, h, 0.0)
    for k in (0.0, 1.0, 100.0):
        K = oracle_mod.q4_local(x, A, B, Cs, h, k)
        D = independent_drill(x, A, k)
        assert _isapprox(K - K0, D, rtol=2e-9, atol=2e-7)
        assert np.linalg.norm(K - K.T) < 5e-13 * np.linalg.norm(K)


@pytest.mark.parametrize("nu", [0.0, .23, .33, .45])
@pytest.mark.parametrize("a,b", [(1., .6), (1., 1.), (4., 1.)])
def test_quad4_bending_poisson_relaxation(oracle_mod, a, b, nu):
    """utils/test/quad4_bending_poisson_relaxation_test.jl:6-33: the normalised
    rotational hourglass fields relax their Poisson curvature through the
    internal modes, energy D*(1-nu^2)*a/(3b) (rtol 2e-12), and every constant
    curvature field still carries the complete D (P'KP = ab*D, rtol 2e-12)."""
    E, h = 7e10, .003
    x = np.array([[0., 0.], [a, 0.], [a, b], [0., b]])
    A = E * h / (1 - nu ** 2) * np.array([[1., nu, 0.], [nu, 1., 0.], [0., 0., (1 - nu) / 2]])
    D = A * h ** 2 / 12
    S = np.eye(2) * (5 / 6) * E * h / (2 * (1 + nu))
    K = oracle_mod.q4_local(x, A, D, S, h, 0.0)
    g = np.array([1., -1., 1., -1.]) / 2
    qx = np.zeros(24); qy = np.zeros(24)
    for i in range(4):
        qx[6 * i + 3] = g[i]; qy[6 * i + 4] = g[i]
    assert qx @ K @ qx == pytest.approx(D[1, 1] * (1 - nu ** 2) * a / (3 * b), rel=2e-12)
    assert qy @ K @ qy == pytest.approx(D[0, 0] * (1 - nu ** 2) * b / (3 * a), rel=2e-12)
    assert abs(qx @ K @ qy) < 2e-12 * np.linalg.norm(D)
    assert np.linalg.eigvalsh(0.5 * (K + K.T)).min() / np.linalg.norm(K, 2) > -2e-12
    P = np.zeros((24, 3))
    for i in range(4):
        xx, yy = x[i]; j = 6 * i
        P[j + 2] = [-xx ** 2 / 2, -yy ** 2 / 2, -xx * yy / 2]
        P[j + 3] = [0., -yy, -xx / 2]
        P[j + 4] = [xx, 0., yy / 2]
    assert _isapprox(P.T @ K @ P, a * b * D, rtol=2e-12)


def _laminate_qbar(E1, E2, nu12, G12, th):
    """Rotated orthotropic plane-stress stiffness (classical lamination theory),
    as src/ModelBuilder.jl:22-47 laminate_plane_stress_qbar."""
    nu21 = nu12 * E2 / max(E1, 1e-30)
    d = 1.0 - nu12 * nu21
    Q11, Q22, Q12, Q66 = E1 / d, E2 / d, nu12 * E2 / d, G12
    c, s = np.cos(th), np.sin(th)
    c2, s2, cs = c * c, s * s, c * s
    q = np.zeros((3, 3))
    q[0, 0] = Q11 * c2 ** 2 + 2 * (Q12 + 2 * Q66) * c2 * s2 + Q22 * s2 ** 2
    q[1, 1] = Q11 * s2 ** 2 + 2 * (Q12 + 2 * Q66) * c2 * s2 + Q22 * c2 ** 2
    q[0, 1] = q[1, 0] = (Q11 + Q22 - 4 * Q66) * c2 * s2 + Q12 * (c2 ** 2 + s2 ** 2)
    q[0, 2] = q[2, 0] = (Q11 - Q12 - 2 * Q66) * cs * c2 + (Q12 - Q22 + 2 * Q66) * cs * s2
    q[1, 2] = q[2, 1] = (Q11 - Q12 - 2 * Q66) * cs * s2 + (Q12 - Q22 + 2 * Q66) * cs * c2
    q[2, 2] = (Q11 + Q22 - 2 * Q12 - 2 * Q66) * c2 * s2 + Q66 * (c2 ** 2 + s2 ** 2)
    return q


def _laminate_shear(G13, G23, th):
    """src/ModelBuilder.jl:49-56 laminate_transverse_shear_qbar."""
    c, s = np.cos(th), np.sin(th)
    return np.array([[c * c * G13 + s * s * G23, c * s * (G13 - G23)],
                     [c * s * (G13 - G23), s * s * G13 + c * c * G23]])


@pytest.mark.parametrize("angle", [0.0, np.pi / 6, -np.pi / 5])
@pytest.mark.parametrize("shape", [0, 1, 2])
def test_quad4_affine_bending_patch(oracle_mod, shape, angle):
    """utils/test/quad4_affine_hourglass_test.jl:7-29 (bending block): for a
    rotated laminate, the three constant-curvature fields give P'KP = area*D
    (2e-10), the rigid rotations carry no force (2e-12) and K is symmetric.
    The reference test runs the membrane without incompatible modes; the
    bending block checked here does not depend on the membrane options."""
    xy = (np.array([[0., 0.], [1., 0.], [1., .5], [0., .5]]),
          np.array([[0., 0.], [1., 0.], [1.3, .5], [.3, .5]]),
          np.array([[0., 0.], [1., 0.], [.7, .5], [.1, .5]]))[shape]
    q = _laminate_qbar(135e9, 8.5e9, .27, 4.8e9, angle)
    h = .002
    A, D = h * q, h ** 3 / 12 * q
    C = (5 * h / 6) * _laminate_shear(5.1e9, 3.2e9, angle)
    K = oracle_mod.q4_local(xy, A, D, C, h, 0.0)
    P = np.zeros((24, 3)); R = np.zeros((24, 3))
    for i in range(4):
        x, y = xy[i]; j = 6 * i
        P[j + 2] = [-x * x / 2, -y * y / 2, -x * y / 2]
        P[j + 3] = [0., -y, -x / 2]; P[j + 4] = [x, 0., y / 2]
        R[j + 2] = [1., y, -x]; R[j + 3, 1] = 1.; R[j + 4, 2] = 1.
    area = abs(sum(xy[i, 0] * xy[(i + 1) % 4, 1] - xy[(i + 1) % 4, 0] * xy[i, 1] for i in range(4))) / 2
    assert np.linalg.norm(P.T @ K @ P - area * D) < 2e-10 * np.linalg.norm(area * D)
    assert np.linalg.norm(K @ R) < 2e-12 * np.linalg.norm(K) * np.linalg.norm(R)
    assert np.linalg.norm(K - K.T) < 2e-12 * np.linalg.norm(K)


# ---------------------------------------------------------------------------
# Applied loads: the oracle's restatement of PLOAD4 / FORCE / node frames
# ---------------------------------------------------------------------------

def _random_frames(n, seed):
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 9))
    for i in range(n):
        Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        out[i] = Q.ravel(order="F")
    return out


@pytest.mark.parametrize("name", ["plate", "plate_frames", "wing_small", "panel", "solid"])
def test_oracle_loads_match_the_host_loads(oracle_mod, name):
    """The oracle's own PLOAD4 / FORCE / nodal-load restatement
    (loads.jl:546-585, solve_case.jl:78-82) against the host's load vectors,
    including grids with rotated displacement frames."""
    if name.startswith("plate"):
        m = M.flat_plate()
        if name == "plate_frames":
            m.node_R = _random_frames(m.n_nodes, 5)
    elif name == "wing_small":
        m = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=3)
    elif name == "panel":
        m = M.stiffened_panel(7)
    else:
        m = M.solid_block(n=3, n_cases=2)
    Fo = oracle_mod.load_matrix(m)
    Fh = m.load_matrix()
    scale = np.abs(Fo).max()
    assert np.abs(Fo - Fh).max() <= 1e-13 * scale


def test_pressure_and_face_load_totals(oracle_mod):
    """Known answers: a flat plate under p carries p * area in total; the
    C3D10 consistent face load on the top of the block (corner nodes 0,
    mid-side nodes p*A/3 per face, abaqus_input.jl:383-388) sums to p * L^2."""
    m = M.flat_plate(pressure=10e3)
    F = oracle_mod.load_matrix(m)[:, 0].reshape(-1, 6)
    assert F[:, 2].sum() == pytest.approx(10e3 * 0.5 * 0.5, rel=1e-13)
    assert np.abs(F[:, 3:]).max() == 0.0
    s = M.solid_block(n=3, n_cases=1, sigma=0.0, traction=1e6, L=0.3)
    F = oracle_mod.load_matrix(s)[:, 0].reshape(-1, 6)
    assert F[:, 2].sum() == pytest.approx(-1e6 * 0.3 * 0.3, rel=1e-13)
    corner = np.all((np.round(s.xyz / (0.3 / 6)) % 2) == 0, axis=1)
    assert np.abs(F[corner, 2]).max() == 0.0


def test_t10_stress_recovery_uniform_strain(oracle_mod):
    """Known answer for the CTETRA10 centroid recovery (stress_recovery.jl:
    1823-1960): an affine displacement u = A x gives every element the strain
    sym(A) (engineering shears) and the stress D strain, also when the grids
    carry rotated displacement frames (u_node = node_R' u)."""
    m = M.solid_block(n=2, n_cases=1)
    m.node_R = _random_frames(m.n_nodes, 3)
    A = np.array([[.002, .001, -.0004], [-.0002, -.0007, .0003], [.0008, -.0006, .0011]])
    ub = m.xyz @ A.T
    R = m.node_R.reshape(-1, 3, 3).transpose(0, 2, 1)          # R[n] = node_R as a matrix
    U = np.zeros((m.ndof, 1))
    U.reshape(-1, 6)[:, :3] = np.einsum("nji,nj->ni", R, ub)   # node_R' u
    S = oracle_mod.t10_stresses(m, U)[0]
    eps = np.array([A[0, 0], A[1, 1], A[2, 2], A[0, 1] + A[1, 0], A[1, 2] + A[2, 1], A[2, 0] + A[0, 2]])
    E, nu = 210e9, 0.3
    c = E / ((1 + nu) * (1 - 2 * nu))
    D = np.zeros((6, 6)); D[:3, :3] = c * nu; np.fill_diagonal(D[:3, :3], c * (1 - nu))
    D[3, 3] = D[4, 4] = D[5, 5] = c * (1 - 2 * nu) / 2
    sig = D @ eps
    vm = np.sqrt(sig[0] ** 2 + sig[1] ** 2 + sig[2] ** 2 - sig[0] * sig[1] - sig[1] * sig[2] - sig[2] * sig[0]
                 + 3 * (sig[3] ** 2 + sig[4] ** 2 + sig[5] ** 2))
    assert np.allclose(S[:, 6:12], eps[None, :], rtol=1e-12, atol=1e-15)
    assert np.allclose(S[:, 0:6], sig[None, :], rtol=1e-10, atol=1e-3)
    assert np.allclose(S[:, 12], vm, rtol=1e-10)
