"""The oracle's CQUAD4 stress recovery (or_q4_stress, the restatement of
recover_shell_stresses! on the default isotropic PSHELL path,
src/solver/stress_recovery.jl:505-1237) pinned to the properties the
reference's own tests assert:

- the area-mean shear resultant is work-conjugate with the element
  stiffness under uniform transverse-shear motions
  (utils/test/pshell_shear_recovery_test.jl:26-62,
  utils/test/macneal_shear_resultants_test.jl:16-28), rtol 2e-10;
- the three transverse rigid motions carry no shear resultant
  (macneal_shear_resultants_test.jl:29-38), and the resultant is linear in u
  (:39);
- a uniform membrane strain and a uniform curvature give N = h C eps and
  M = -(h^3/12) C kappa (utils/test/shell_corner_thickness_recovery_test.jl:67-68,
  rtol 3e-12), with the fibre stresses C (eps -+ h/2 kappa) and the strain
  rows eps and -kappa (stress_recovery.jl:1118-1123, :1239-1255);
- N and M are the thickness moments of the fibre stresses
  (utils/test/pcomp_projected_recovery_work_test.jl:130-131).
"""
import numpy as np
import pytest

from jf_2026_05_25_b200 import model as M

E, NU, G, H = 7e10, 0.29, 2e10, 0.1
SHAPES = ([[-1.0, -0.5], [1.0, -0.5], [1.0, 0.5], [-1.0, 0.5]],
          [[-1.0, -0.5], [1.0, -0.5], [1.4, 0.5], [-0.6, 0.5]],
          [[-1.0, -0.5], [1.0, -0.5], [0.7, 0.5], [-0.8, 0.5]])


def _quad(xy, tst=5.0 / 6.0, k6rot=100.0):
    """One CQUAD4 on grids 1-4 (the reference tests' deck) and its section."""
    xyz = np.hstack([np.asarray(xy, float), np.zeros((4, 1))])
    m = M.Sol101Model(name="q4", grid_ids=np.arange(1, 5), xyz=xyz,
                      q4_nodes=np.array([[0, 1, 2, 3]], np.int32), q4_pid=np.ones(1, np.int64),
                      q4_eid=np.ones(1, np.int64),
                      pshells={1: M.PShell(T=H, MID1=1, MID2=1, MID3=1, TS_T=tst)},
                      mats={1: M.Mat1(E=E, NU=NU, G=G)}, k6rot=k6rot)
    return m


def _frame(X):
    """Element frame rows (v1, v2, v3) and centred local coordinates, as the
    reference takes them for a flat quadrilateral (diagonal mode)."""
    gxi = 0.25 * (-X[0] + X[1] + X[2] - X[3])
    geta = 0.25 * (-X[0] - X[1] + X[2] + X[3])
    v3 = np.cross(gxi, geta)
    v3 /= np.linalg.norm(v3)
    d13, d24 = X[2] - X[0], X[3] - X[1]
    xr = d13 / np.linalg.norm(d13) - d24 / np.linalg.norm(d24)
    v1 = xr - xr.dot(v3) * v3
    v1 /= np.linalg.norm(v1)
    Rel = np.vstack([v1, np.cross(v3, v1), v3])
    return Rel, (X - X.mean(0)) @ Rel.T


def _to_global(Rel, local24):
    g = np.zeros(24)
    for k in range(4):
        g[6 * k:6 * k + 3] = Rel.T @ local24[6 * k:6 * k + 3]
        g[6 * k + 3:6 * k + 6] = Rel.T @ local24[6 * k + 3:6 * k + 6]
    return g


def _recover(oracle_mod, m, u):
    return oracle_mod.q4_stresses(m, np.asarray(u, float)[:, None])[0, 0]


@pytest.mark.parametrize("shape", range(len(SHAPES)))
@pytest.mark.parametrize("tst", (0.25, 5.0 / 6.0))
def test_shear_resultant_is_work_conjugate(oracle_mod, shape, tst):
    m = _quad(SHAPES[shape], tst=tst)
    Rel, loc = _frame(m.xyz)
    area = 0.5 * abs(sum(loc[i, 0] * loc[(i + 1) % 4, 1] - loc[i, 1] * loc[(i + 1) % 4, 0] for i in range(4)))
    K = oracle_mod.q4_element(m.xyz, m.q4_sections()[0])
    for pattern in ("unit_shear", "general"):
        local = 1e-3 * np.sin(np.arange(1.0, 25.0)) if pattern == "general" else np.zeros(24)
        if pattern == "unit_shear":
            local[4::6] = 1e-3
        u = _to_global(Rel, local)
        q = _recover(oracle_mod, m, u)[6:8]
        if pattern == "unit_shear":
            assert np.linalg.norm(q) > 1e-6
        for gamma in ([1.0, 0.0], [0.0, 1.0], [0.4, -0.7]):
            v = np.zeros(24)
            v[3::6] = -gamma[1]
            v[4::6] = gamma[0]
            work = _to_global(Rel, v) @ K @ u
            assert area * np.dot(gamma, q) == pytest.approx(work, rel=2e-10, abs=1e-8)


@pytest.mark.parametrize("shape", range(len(SHAPES)))
def test_rigid_transverse_motions_carry_no_shear(oracle_mod, shape):
    m = _quad(SHAPES[shape])
    Rel, loc = _frame(m.xyz)
    u = _to_global(Rel, 1e-3 * np.sin(np.arange(1.0, 25.0)))
    q = _recover(oracle_mod, m, u)[6:8]
    assert np.abs(_recover(oracle_mod, m, 3 * u)[6:8] - 3 * q).max() <= 1e-12 * np.abs(q).max()
    for comp in range(3):
        rigid = np.zeros(24)
        for i in range(4):
            rigid[6 * i + 2] = (1.0, loc[i, 1], -loc[i, 0])[comp]
            rigid[6 * i + 3] = 1.0 if comp == 1 else 0.0
            rigid[6 * i + 4] = 1.0 if comp == 2 else 0.0
        assert np.linalg.norm(_recover(oracle_mod, m, _to_global(Rel, rigid))[6:8]) < 1e-12 * max(1.0, np.abs(q).max())


def test_uniform_fields_recover_exactly(oracle_mod):
    """Uniform membrane strain plus uniform curvature on distorted quadrilaterals
    in random planes: the centre forces, fibre stresses and strain rows."""
    rng = np.random.default_rng(3)
    C = E / (1 - NU * NU) * np.array([[1, NU, 0], [NU, 1, 0], [0, 0, (1 - NU) / 2]])
    for trial in range(6):
        xy = np.asarray(SHAPES[trial % 3]) + 0.05 * rng.standard_normal((4, 2))
        Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        m = _quad(xy)
        m.xyz = np.asarray(xy) @ Q[:, :2].T + rng.standard_normal(3)
        Rel, loc = _frame(m.xyz)
        eps = rng.standard_normal(3) * 1e-3
        kap = rng.standard_normal(3) * 1e-2
        local = np.zeros(24)
        for k in range(4):
            x, y = loc[k, 0], loc[k, 1]
            local[6 * k:6 * k + 2] = [eps[0] * x + eps[2] / 2 * y, eps[2] / 2 * x + eps[1] * y]
            local[6 * k + 3:6 * k + 5] = [-kap[1] * y - kap[2] / 2 * x, kap[0] * x + kap[2] / 2 * y]
        rec = _recover(oracle_mod, m, _to_global(Rel, local))
        N, Mo = H * C @ eps, -(H ** 3 / 12) * C @ kap
        assert np.abs(rec[0:3] - N).max() <= 3e-12 * np.abs(N).max()
        assert np.abs(rec[3:6] - Mo).max() <= 3e-12 * np.abs(Mo).max()
        s1, s2 = C @ (eps - H / 2 * kap), C @ (eps + H / 2 * kap)
        assert np.abs(rec[8:11] - s1).max() <= 3e-12 * np.abs(s1).max()
        assert np.abs(rec[14:17] - s2).max() <= 3e-12 * np.abs(s2).max()
        assert np.abs(rec[20:23] - eps).max() <= 3e-12 * np.abs(eps).max()
        assert np.abs(rec[25:28] + kap).max() <= 1e-10 * np.abs(kap).max()
        # thickness moments of the fibre stresses
        assert np.abs(H * (rec[8:11] + rec[14:17]) / 2 - rec[0:3]).max() <= 3e-12 * np.abs(N).max()
        assert np.abs(-(H ** 2 / 12) * (rec[14:17] - rec[8:11]) - rec[3:6]).max() <= 3e-12 * np.abs(Mo).max()


def test_principal_values_and_von_mises(oracle_mod):
    """Each fibre row's major/minor are the eigenvalues of (sx, sy, txy), its
    von Mises sqrt(sx^2 - sx sy + sy^2 + 3 txy^2); the strain rows use half
    the engineering shear (stress_recovery.jl:1239-1255)."""
    m = M.stiffened_panel(3)
    rng = np.random.default_rng(11)
    U = rng.standard_normal((m.ndof, 1)) * 1e-4
    S = oracle_mod.q4_stresses(m, U)[0]
    for off in (8, 14):
        sx, sy, txy = S[:, off], S[:, off + 1], S[:, off + 2]
        ev = np.linalg.eigvalsh(np.stack([np.stack([sx, txy], -1), np.stack([txy, sy], -1)], -2))
        scale = np.abs(S[:, off:off + 3]).max()
        assert np.abs(S[:, off + 4] - ev[:, 1]).max() <= 1e-12 * scale
        assert np.abs(S[:, off + 5] - ev[:, 0]).max() <= 1e-12 * scale
        vm = np.sqrt(sx * sx - sx * sy + sy * sy + 3 * txy * txy)
        assert np.abs(S[:, off + 3] - vm).max() <= 1e-12 * scale
    assert np.abs(S[:, 30] - S[:, 12]).max() <= 1e-12 * np.abs(S[:, 8:11]).max()
    for off in (20, 25):
        ex, ey, g = S[:, off], S[:, off + 1], S[:, off + 2] / 2
        ev = np.linalg.eigvalsh(np.stack([np.stack([ex, g], -1), np.stack([g, ey], -1)], -2))
        scale = np.abs(S[:, off:off + 3]).max()
        assert np.abs(S[:, off + 3] - ev[:, 1]).max() <= 1e-12 * scale
        assert np.abs(S[:, off + 4] - ev[:, 0]).max() <= 1e-12 * scale


def test_recovery_mask_follows_the_constitutive_gap():
    """MID2 / MID3 of another MAT1 law leave an element unrecovered; an equal
    alias keeps it (pshell_equivalent_material_recovery_test.jl:27-36)."""
    m = _quad(SHAPES[0])
    assert m.q4_recovery_mask().tolist() == [True]
    m.mats[2] = M.Mat1(E=E, NU=NU, G=G, RHO=1000.0)
    m.pshells[1] = M.PShell(T=H, MID1=1, MID2=2, MID3=2)
    assert m.q4_recovery_mask().tolist() == [True]
    m.mats[3] = M.Mat1(E=E, NU=NU, G=G / 2)
    m.pshells[1] = M.PShell(T=H, MID1=1, MID2=1, MID3=3)
    assert m.q4_recovery_mask().tolist() == [False]
    m.pshells[1] = M.PShell(T=H, MID1=1, MID2=3, MID3=1, BEND_RATIO=0.0)
    assert m.q4_recovery_mask().tolist() == [True]
