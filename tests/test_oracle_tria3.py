"""CTRIA3 in the oracle, pinned to the reference's own triangle tests, and the
host rules around it (CQUAD8 split, triangle pressures).  CPU only.

The reference's triangle tests hold properties rather than matrix entries:
utils/test/tria_bending_flexibility_guard_test.jl (guard cases; symmetry,
positive semi-definiteness, rigid-body null space and unit scaling of the
element over a grid of orthotropic sections and shapes) and
utils/test/tria_orthogonal_residual_energy_test.jl (the guard's bounds in
orthogonal work coordinates).  The same checks run here on the restatement.
"""
import numpy as np
import pytest

from jf_2026_05_25_b200 import model as M


def _rotate3(Q, beta):
    """FEMKernels.jl:1458-1495 rotate_constitutive_3x3!: T' Q T."""
    if abs(beta) <= 1e-12:
        return Q
    c, s = np.cos(beta), np.sin(beta)
    c2, s2, cs = c * c, s * s, c * s
    T = np.array([[c2, s2, cs], [s2, c2, -cs], [-2 * cs, 2 * cs, c2 - s2]])
    return T.T @ Q @ T


def _rotate2(C, beta):
    """FEMKernels.jl:1497-1513 rotate_constitutive_2x2!."""
    if abs(beta) <= 1e-12:
        return C
    c, s = np.cos(beta), np.sin(beta)
    a11, a12, a22 = C[0, 0], C[0, 1], C[1, 1]
    o12 = c * s * a11 + (c * c - s * s) * a12 - c * s * a22
    return np.array([[c * c * a11 - 2 * c * s * a12 + s * s * a22, o12],
                     [o12, s * s * a11 + 2 * c * s * a12 + c * c * a22]])


def test_guard_inactive_and_slender_cases(oracle_mod):
    # tria_bending_flexibility_guard_test.jl:10-20
    ordinary = np.array([[2.0, 0.1, 0.2], [0.1, 3.0, -0.1], [0.2, -0.1, 1.0]])
    changed, Z = oracle_mod.tria3_guard(ordinary, 1.0, 1.0, 0.6, 0.8, 4.0)
    assert not changed and np.array_equal(Z, ordinary)
    slender = np.array([[1e-8, 2e-5, 0.0], [2e-5, 2.0, 0.0], [0.0, 0.0, 1.0]])
    changed, Z = oracle_mod.tria3_guard(slender, 0.004, 1.0, 0.8, 0.6, 3.0)
    assert changed
    assert np.array_equal(Z[2, :], slender[2, :]) and np.array_equal(Z[:, 2], slender[:, 2])
    assert np.linalg.eigvalsh(Z).min() > 0


def _make_flexibility(P, La, Lb, c, s, Dn):
    back = np.array([[1.0, 0.0], [c, s]])
    H = back @ P @ back.T
    scale = 6 * (La / Lb) * s * Dn
    q, z = np.array([-0.13, 0.21]), 1.7
    Z = np.zeros((3, 3))
    Z[:2, :2] = H * np.outer([La, Lb], [La, Lb]) / scale + np.outer(q, q) / z
    Z[:2, 2] = q
    Z[2, :2] = q
    Z[2, 2] = z
    return Z


def _orthogonal_block(Z, La, Lb, c, s, Dn):
    scale = 6 * (La / Lb) * s * Dn
    H = scale * (Z[:2, :2] - np.outer(Z[:2, 2], Z[2, :2]) / Z[2, 2]) / np.outer([La, Lb], [La, Lb])
    Q = np.array([[1.0, 0.0], [-c / s, 1 / s]])
    return Q @ H @ Q.T


def test_guard_orthogonal_residual_bounds(oracle_mod):
    # tria_orthogonal_residual_energy_test.jl:23-47
    for c in (-0.4, 0.0, 0.6):
        for La, Lb in ((0.03, 1.2), (1.0, 0.7), (3.0, 7.0)):
            for a in (-0.2, 1e-5, 0.3, 2.0):
                for b in (-1.1, 0.02, 0.8):
                    s, d, normal = np.sqrt(1 - c * c), 0.7, 2.3
                    Z0 = _make_flexibility(np.array([[a, b], [b, d]]), La, Lb, c, s, normal)
                    changed, Z = oracle_mod.tria3_guard(Z0, La, Lb, c, s, normal)
                    got = _orthogonal_block(Z, La, Lb, c, s, normal)
                    assert np.isclose(got[1, 1], d, rtol=2e-8, atol=2e-10)
                    assert got[0, 0] >= 1e-4 - 3e-10
                    assert got[0, 1] ** 2 <= 0.85 * got[0, 0] * got[1, 1] + 2e-10
                    assert np.linalg.eigvalsh(0.5 * (Z + Z.T)).min() > 0
                    assert np.array_equal(Z[2, :], Z0[2, :]) and np.array_equal(Z[:, 2], Z0[:, 2])
                    if a >= 1e-4 and b * b <= 0.85 * a * d:
                        assert not changed and np.array_equal(Z, Z0)
                    else:
                        assert changed
                        assert np.isclose(got[0, 0], max(a, 1e-4), rtol=2e-6, atol=3e-10)


def test_guard_rejects_non_positive_normal_flexibility(oracle_mod):
    Z = _make_flexibility(np.array([[0.3, 0.0], [0.0, -0.5]]), 1.0, 1.0, 0.0, 1.0, 1.0)
    with pytest.raises(ValueError):
        oracle_mod.tria3_guard(Z, 1.0, 1.0, 0.0, 1.0, 1.0)


@pytest.mark.parametrize("ratio", [1.0, 2.0, 5.0])
@pytest.mark.parametrize("angle", [0.0, 0.43, 1.07])
@pytest.mark.parametrize("shape", [0, 1])
def test_element_properties(oracle_mod, ratio, angle, shape):
    # tria_bending_flexibility_guard_test.jl:22-50
    X = [np.array([[0.0, 0.0], [0.0042, 0.0], [0.803, 0.596]]),
         np.array([[0.0, 0.0], [0.005, 0.0], [0.0, 1.0]])][shape]
    E2, nu, h = 7e10, 0.3, 0.0025
    E1 = ratio * E2
    g12 = np.sqrt(E1 * E2) / (2 * (1 + nu))
    den = 1 - nu * nu * E2 / E1
    Q = _rotate3(np.array([[E1 / den, nu * E2 / den, 0.0], [nu * E2 / den, E2 / den, 0.0], [0.0, 0.0, g12]]), angle)
    C = _rotate2(np.array([[E1 / (2 * (1 + nu)), 0.0], [0.0, E2 / (2 * (1 + nu))]]), angle)

    def kernel(x, t, scale=1.0):
        return oracle_mod.tria3_local(x, scale * Q * t, scale * Q * t ** 3 / 12, scale * C * (5 * t / 6), 100.0)
    K = kernel(X, h)
    nK = np.linalg.norm(K, 2)
    assert np.allclose(K, K.T, rtol=1e-13, atol=1e-13 * np.abs(K).max())
    assert np.linalg.eigvalsh(0.5 * (K + K.T)).min() >= -2e-12 * nK
    for axis in range(3):
        for rotation in (False, True):
            d = np.zeros(3)
            d[axis] = 1.0
            u = np.zeros(18)
            for i in range(3):
                p = np.array([X[i, 0], X[i, 1], 0.0])
                u[6 * i:6 * i + 3] = np.cross(d, p) if rotation else d
                if rotation:
                    u[6 * i + 3:6 * i + 6] = d
            assert np.linalg.norm(K @ u) <= 2e-11 * nK * np.linalg.norm(u)
    assert np.allclose(kernel(X, h, 7.3), 7.3 * K, rtol=2e-9, atol=2e-9 * np.abs(K).max())
    sc = 9.0
    Ld = np.diag(np.tile([sc, sc, sc, 1.0, 1.0, 1.0], 3))
    assert np.allclose(Ld.T @ kernel(sc * X, sc * h) @ Ld, sc ** 3 * K, rtol=2e-9, atol=2e-9 * sc ** 3 * np.abs(K).max())


def test_degenerate_triangle_is_zero(oracle_mod):
    # FEMKernels.jl:9380: area below 1e-12 gives a zero matrix
    D = np.eye(3)
    K = oracle_mod.tria3_local(np.array([[0.0, 0.0], [1e-7, 0.0], [0.0, 1e-7]]), D, D, np.eye(2), 100.0)
    assert not K.any()


def test_membrane_patch_and_drilling(oracle_mod):
    # a linear in-plane field u = a x + b y has the constant CST strain, so
    # u' K_mem u = area e' Dm e; the lumped drilling penalises theta_z minus
    # the membrane rotation with K6ROT 1e-6 Dm[3,3] 2A per node
    X = np.array([[0.0, 0.0], [0.03, 0.004], [0.011, 0.025]])
    Dm = np.array([[2.0, 0.6, 0.0], [0.6, 2.0, 0.0], [0.0, 0.0, 0.7]]) * 1e8
    K = oracle_mod.tria3_local(X, Dm, np.zeros((3, 3)), np.zeros((2, 2)), 0.0)
    A = 0.5 * abs(np.cross(X[1] - X[0], X[2] - X[0]))
    g = np.array([[1.3e-3, -0.4e-3], [0.7e-3, 2.1e-3]])   # [du/dx du/dy; dv/dx dv/dy]
    u = np.zeros(18)
    for i in range(3):
        u[6 * i:6 * i + 2] = g @ X[i]
    e = np.array([g[0, 0], g[1, 1], g[0, 1] + g[1, 0]])
    assert np.isclose(u @ K @ u, A * e @ Dm @ e, rtol=1e-13)
    Kd = oracle_mod.tria3_local(X, Dm, np.zeros((3, 3)), np.zeros((2, 2)), 100.0) - K
    w = 0.5 * (g[1, 0] - g[0, 1])
    for i in range(3):
        u[6 * i + 5] = w + 1e-3 * (i + 1)          # theta_z off the membrane rotation
    alpha = 100.0 * 1e-6 * Dm[2, 2] * 2 * A
    assert np.isclose(u @ Kd @ u, alpha * sum((1e-3 * (i + 1)) ** 2 for i in range(3)), rtol=1e-10)


def test_split_rule_matches_the_oracle(oracle_mod):
    m = M.quad8_plate(6, 4, taper=0.5, tilt_deg=15)
    keep = m.q8_native_mask()
    assert keep.sum() == 12 and (~keep).sum() == 12      # the half x > a/2 is tapered
    q8n, q8s = m.device_q8()
    t3n, t3s = m.device_t3()
    oq8n, oq8s, ot3n, ot3s = oracle_mod.shells_as_assembled(m)
    assert np.array_equal(q8n, oq8n) and np.array_equal(q8s, oq8s)
    assert np.array_equal(t3n, ot3n) and len(t3n) == 6 * 12
    assert np.allclose(t3s, ot3s, rtol=1e-14, atol=0.0)
    # the triangles tile each element: their areas add up to the element's
    X = m.xyz
    tri = 0.5 * np.linalg.norm(np.cross(X[t3n[:, 1]] - X[t3n[:, 0]], X[t3n[:, 2]] - X[t3n[:, 0]]), axis=1)
    q8 = m.q8_nodes[~keep]
    quad = 0.5 * np.linalg.norm(np.cross(X[q8[:, 2]] - X[q8[:, 0]], X[q8[:, 3]] - X[q8[:, 1]]), axis=1)
    assert np.allclose(tri.reshape(-1, 6).sum(axis=1), quad, rtol=1e-12)


def test_triangle_sections_match_the_oracle(oracle_mod):
    m = M.tria_plate(nx=4, ny=2)
    m.pshells[2] = M.PShell(T=0.004, MID1=1, MID2=2, MID3=0, BEND_RATIO=0.8, TS_T=0.7)
    m.pshells[3] = M.PShell(T=0.001, MID1=2, BEND_RATIO=0.0)
    m.mats[2] = M.Mat1(E=120e9, NU=0.29, G=45e9)
    m.t3_pid = np.arange(len(m.t3_nodes)) % 3 + 1
    _, _, _, ot3s = oracle_mod.shells_as_assembled(m)
    assert np.allclose(m.t3_sections(), ot3s, rtol=1e-14, atol=0.0)


def test_triangle_pressure_matches_the_oracle(oracle_mod):
    m = M.tria_plate(nx=6, ny=4)
    for case in m.load_cases:
        assert np.allclose(m.load_vector(case), oracle_mod.load_vector(m, case), rtol=1e-14, atol=1e-14)
    # total pressure force = p times the area, along each facet normal
    F = m.load_vector(m.load_cases[0]).reshape(-1, 6)[:, :3].sum(axis=0)
    X = m.xyz
    t3, q4 = m.t3_nodes, m.q4_nodes
    n3 = np.cross(X[t3[:, 1]] - X[t3[:, 0]], X[t3[:, 2]] - X[t3[:, 0]])
    n4 = np.cross(X[q4[:, 2]] - X[q4[:, 0]], X[q4[:, 3]] - X[q4[:, 1]])
    assert np.allclose(F, 5e3 * 0.5 * (n3.sum(axis=0) + n4.sum(axis=0)), rtol=1e-12)
