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
