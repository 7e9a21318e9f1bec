"""Host-side checks that need no GPU: library exports, symbolic analysis,
partition logic and the synthetic generators."""
import ctypes
import os

import numpy as np
import pytest

from jf_2026_05_25_b200 import backend as B
from jf_2026_05_25_b200 import build as jbuild
from jf_2026_05_25_b200 import lib
from jf_2026_05_25_b200 import model as M


@pytest.fixture(scope="module")
def libjfg():
    jbuild.build()
    return lib.load()


def test_library_exports_every_declared_symbol(libjfg):
    names = lib.exported_symbols()
    assert "jfg_solve" in names and "jfg_assemble" in names
    for n in names:
        assert hasattr(libjfg, n), n


def test_create_without_device_reports_cuda_error(libjfg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    with pytest.raises(lib.JfgError) as e:
        lib.Context(0)
    assert e.value.status_name == "CUDA_ERROR"


@pytest.mark.parametrize("mk", [lambda: M.flat_plate(), lambda: M.wing_panel(nx=16, ny=24, n_blades=3, blade_nz=3, n_cases=2),
                                lambda: M.solid_block(n=3, n_cases=2)])
def test_symbolic_permutation_solves_with_oracle(libjfg, oracle_mod, mk):
    mdl = mk()
    asm = oracle_mod.assemble(mdl)
    K = oracle_mod.csc_matrix(asm)
    free, _, _ = oracle_mod.partition(mdl, K)
    info, perm = lib.symbolic_dry_run(asm["colptr"], asm["rowval"], free, mdl.xyz)
    assert np.array_equal(np.sort(perm), np.arange(len(free)))
    assert info["nnz_L"] > 0 and info["n_levels"] >= 1
    Kff = K[free][:, free].tocsc()
    F = mdl.load_matrix()[free]
    U, oinfo = oracle_mod.chol_solve(len(free), Kff.indptr.astype(np.int64), Kff.indices, Kff.data, perm, F)
    # the amalgamated device structure stores at least the exact fill
    assert info["nnz_L"] >= oinfo["nnz_L"]
    ref = oracle_mod.solve_reference(mdl, asm=asm, free=free)
    assert np.abs(U - ref["u"][free]).max() <= 1e-6 * np.abs(ref["u"]).max()


def _host_blocks(K, nn):
    Kc = K.tocsc()
    out = np.zeros((nn, 18))
    for n in range(nn):
        for off in (0, 1):
            idx = [6 * n + 3 * off + a for a in range(3)]
            out[n, 9 * off:9 * off + 9] = Kc[idx][:, idx].toarray().ravel(order="F")
    return out


@pytest.mark.parametrize("mk", [lambda: M.flat_plate(nx=6, ny=5), lambda: M.solid_block(n=2, n_cases=1)])
def test_partition_matches_oracle(oracle_mod, mk):
    mdl = mk()
    asm = oracle_mod.assemble(mdl)
    K = oracle_mod.csc_matrix(asm)
    free_o, fixed_o, _ = oracle_mod.partition(mdl, K)
    free_b, fixed_b, diag = B.compute_free_dofs(mdl, K.diagonal(), _host_blocks(K, mdl.n_nodes))
    assert np.array_equal(free_o, free_b)
    assert np.array_equal(fixed_o, fixed_b)


def test_partition_gpst_finds_oblique_drilling(oracle_mod):
    """K6ROT=0 on a plate rotated out of the basic planes: the singular
    drilling direction is oblique, so only the grid-point test finds it."""
    mdl = M.flat_plate(nx=3, ny=3, k6rot=0.0)
    th = np.radians(30.0)
    R = np.array([[1, 0, 0], [0, np.cos(th), -np.sin(th)], [0, np.sin(th), np.cos(th)]])
    mdl.xyz = mdl.xyz @ R.T
    asm = oracle_mod.assemble(mdl)
    K = oracle_mod.csc_matrix(asm)
    free_b, fixed_b, d = B.compute_free_dofs(mdl, K.diagonal(), _host_blocks(K, mdl.n_nodes))
    free_o, _, do = oracle_mod.partition(mdl, K)
    assert d["autospc_gpst_dofs"] > 0 and do["autospc_gpst"] == d["autospc_gpst_dofs"]
    assert np.array_equal(free_b, free_o)


def _node_pairs(conn, n_nodes):
    """Distinct (row node, column node) pairs coupled by at least one element."""
    conn = np.asarray(conn, np.int64)
    k = conn.shape[1]
    a = np.repeat(conn, k, axis=1).ravel()
    b = np.tile(conn, (1, k)).ravel()
    return len(np.unique(a * n_nodes + b))


def test_wing_panel_counts():
    """Sizes of the stiffened wing-box panel, including nnz(K) = 49,332,276:
    every pair of grids sharing a CQUAD4 couples 6 x 6 DOFs."""
    m = M.wing_panel()
    assert m.n_nodes == 152781 and len(m.q4_nodes) == 152000
    assert m.ndof == 916686
    assert m.ndof - len(m.spc_dofs()) == 914400
    assert len(m.load_cases) == 8
    assert 36 * _node_pairs(m.q4_nodes, m.n_nodes) == 49332276


def test_flat_plate_counts(oracle_mod):
    m = M.flat_plate()
    assert m.n_nodes == 441 and m.ndof == 2646
    asm = oracle_mod.assemble(m)
    assert len(asm["rowval"]) == 133956 == 36 * _node_pairs(m.q4_nodes, m.n_nodes)
    K = oracle_mod.csc_matrix(asm)
    free, _, _ = oracle_mod.partition(m, K)
    assert len(free) == 2166


def test_solid_block_counts():
    m = M.solid_block(n=40)
    assert m.n_nodes == 531441 and len(m.t10_nodes) == 384000
    assert 3 * (m.n_nodes - len(np.unique(m.spc_dofs() // 6))) == 1574640
    # CTETRA10 triplets touch translational DOFs only: 3 x 3 per grid pair
    assert 9 * _node_pairs(m.t10_nodes, m.n_nodes) == 134475849


def test_backend_names():
    assert B.normalize_backend_name("GPU") == "jfem_gpu"
    assert B.backend_from_model({"backend": "reference"}) == "reference_parity"
    assert B.backend_from_model(None, env={"JFEM_BACKEND": "b200"}) == "jfem_gpu"
    with pytest.raises(ValueError):
        B.normalize_backend_name("nope")


def test_packed_model_matches_members(oracle_mod):
    """A pack of independent panels is block diagonal: the host symbolic
    analysis of the pack (a forest) with the oracle Cholesky reproduces every
    member's own solution, and the unit-norm column scaling is undone."""
    from jf_2026_05_25_b200 import serving as S
    ms = [M.stiffened_panel(s) for s in (3, 11)]
    pk = S.PackedModel(ms)
    assert pk.ndof == sum(m.ndof for m in ms)
    asm = oracle_mod.assemble(pk)
    K = oracle_mod.csc_matrix(asm)
    free, _, _ = oracle_mod.partition(pk, K)
    info, perm = lib.symbolic_dry_run(asm["colptr"], asm["rowval"], free, pk.xyz)
    Kff = K[free][:, free].tocsc()
    F, sc = pk.load_columns()
    U, _ = oracle_mod.chol_solve(len(free), Kff.indptr, Kff.indices, Kff.data, perm, F[free])
    Uf = np.zeros((pk.ndof, F.shape[1]))
    Uf[free] = U
    for k, m in enumerate(ms):
        ref = oracle_mod.solve_reference(m)
        Uk = pk.split(Uf, sc)[k]
        assert Uk.shape == ref["u"].shape
        assert np.abs(Uk - ref["u"]).max() <= 1e-8 * np.abs(ref["u"]).max()


def test_autotune_candidates_cover_update_kernels():
    """The default tuning grid covers leaf size x amalgamation thresholds x
    FP64 update kernel; for the mixed factor every schedule is also timed with
    the tensor-core FP32 updates on and off, and explicit candidates are
    taken as given."""
    from jf_2026_05_25_b200 import autotune as AT
    from jf_2026_05_25_b200 import lib
    base = AT.candidate_list(lib.PREC_FP64)
    assert base == AT.DEFAULT_CANDIDATES and len(base) == 18
    mixed = AT.candidate_list(lib.PREC_MIXED)
    assert len(mixed) == 2 * len(base)
    assert {c["JFG_TENSOR_CORES"] for c in mixed} == {"0", "1"}
    assert all({k: v for k, v in c.items() if k != "JFG_TENSOR_CORES"} in base for c in mixed)
    given = [{"JFG_ND_LEAF": "16"}]
    assert AT.candidate_list(lib.PREC_MIXED, given) == given
    assert "JFG_TENSOR_CORES" in AT.KNOBS


@pytest.mark.parametrize("mk", [
    lambda: M.wing_panel_variant(M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=1), 7, 5),
    lambda: M.stiffened_panel(11, n_cases=6),
    lambda: M.flat_plate(),
], ids=["wing_variant", "stiffened_panel", "plate"])
def test_load_matrix_batches_pressures_like_per_case_vectors(oracle_mod, mk):
    """load_matrix applies the CQUAD4 PLOAD4 of all subcases through one
    sparse unit-pressure operator; every column equals load_vector of its
    subcase and the oracle's independent restatement (loads.jl:546-585)."""
    m = mk()
    F = m.load_matrix()
    ref = np.stack([m.load_vector(c) for c in m.load_cases], axis=1)
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.abs(F - ref).max() <= 1e-14 * scale
    assert np.abs(F - oracle_mod.load_matrix(m)).max() <= 1e-13 * scale
    # a second call reuses the operator and gives the same matrix
    assert np.array_equal(m.load_matrix(), F)


def test_section_records_gathered_per_pshell():
    """q4_sections gathers one record per PSHELL: every element carries its
    own PSHELL's record."""
    m = M.wing_panel_variant(M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=1), 3, 1)
    S = m.q4_sections()
    assert S.shape == (len(m.q4_pid), M.Q4_SECT_STRIDE)
    for pid in np.unique(m.q4_pid)[:20]:
        rec = np.asarray(M._q4_section_record(m, int(pid)))
        assert np.array_equal(S[m.q4_pid == pid], np.broadcast_to(rec, (int((m.q4_pid == pid).sum()), len(rec))))
