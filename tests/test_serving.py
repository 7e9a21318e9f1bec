"""Serving on the device (gpu): packed batches and the continuous-batching
server give every model the same result as solving it alone, within the
parity tolerance, and meet the residual bar on each model's own DOFs."""
import numpy as np
import pytest

from jf_2026_05_25_b200 import backend as B
from jf_2026_05_25_b200 import build as jbuild
from jf_2026_05_25_b200 import lib
from jf_2026_05_25_b200 import model as M
from jf_2026_05_25_b200 import serving as S

pytestmark = pytest.mark.gpu

DISP_RTOL = 1e-8
RESID_TOL = 1e-10
SEEDS = (3, 11, 25, 29, 23)


@pytest.fixture(scope="module")
def alone():
    jbuild.build()
    ctx = lib.Context(0)
    out = {}
    for s in SEEDS:
        m = M.stiffened_panel(s)
        be = B.JFEMGPUBackend(tol=RESID_TOL)
        be._ctx = ctx
        res = B.solve_model(be, m)
        out[s] = np.stack([sc["raw_displacement"] for sc in res["subcases"]], axis=1)
        res["state"]["dm"].close()
    yield out
    ctx.close()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_packed_batch_matches_alone(alone):
    models = [M.stiffened_panel(s) for s in SEEDS]
    be = B.JFEMGPUBackend(tol=RESID_TOL)
    out = S.solve_pack(be, models, RESID_TOL)
    for k, s in enumerate(SEEDS):
        assert out["U"][k].shape == alone[s].shape
        assert _rel(out["U"][k], alone[s]) <= DISP_RTOL
        assert out["residuals"][k].max() <= RESID_TOL
    out["state"]["dm"].close()


def test_server_mix_resolve_update_and_latency(alone):
    srv = S.SolveServer(slots=2, tol=RESID_TOL, small_dof=20000, pack_dof=40000)
    try:
        futs = {s: srv.solve(M.stiffened_panel(s)) for s in SEEDS}
        res = {s: f.result(timeout=600) for s, f in futs.items()}
        for s in SEEDS:
            assert _rel(res[s]["U"], alone[s]) <= DISP_RTOL
            assert res[s]["rel_residual"].max() <= RESID_TOL
        # re-solve of a resident model with doubled loads: linear response
        s0 = SEEDS[0]
        m0 = M.stiffened_panel(s0)
        r2 = srv.resolve(res[s0]["key"], 2.0 * m0.load_matrix()).result(timeout=600)
        assert _rel(r2["U"], 2.0 * alone[s0]) <= DISP_RTOL
        assert r2["rel_residual"].max() <= RESID_TOL
        # thickness update of every CQUAD4 of a resident model: same result as
        # a fresh solve of the updated model
        s1 = SEEDS[1]
        m1 = M.stiffened_panel(s1)
        sect = m1.q4_sections()
        ref_model = M.stiffened_panel(s1)
        for p in ref_model.pshells.values():
            p.T *= 1.1
        new_sect = ref_model.q4_sections()
        r3 = srv.update(res[s1]["key"], np.arange(len(sect)), new_sect).result(timeout=600)
        be = B.JFEMGPUBackend(tol=RESID_TOL)
        fresh = B.solve_model(be, ref_model)
        Uref = np.stack([sc["raw_displacement"] for sc in fresh["subcases"]], axis=1)
        assert _rel(r3["U"], Uref) <= DISP_RTOL
        st = srv.stats()
        assert st["requests"] == len(SEEDS) + 2
        assert 0 < st["p50_ms"] <= st["p99_ms"]
    finally:
        srv.close()


def test_server_evicts_under_budget_and_readmits(alone):
    """With a budget too small for two models, the second evicts the first;
    a later re-solve of the first re-admits it from its host description and
    still gives the model's own result."""
    srv = S.SolveServer(slots=1, tol=RESID_TOL, hbm_budget_bytes=1.0, small_dof=0)
    try:
        a = srv.solve(M.stiffened_panel(SEEDS[0])).result(timeout=600)
        b = srv.solve(M.stiffened_panel(SEEDS[1])).result(timeout=600)
        assert a["key"] != b["key"]
        assert a["key"] not in srv.registry
        r = srv.resolve(a["key"]).result(timeout=600)
        assert srv.stats()["readmissions"] == 1
        assert _rel(r["U"], alone[SEEDS[0]]) <= DISP_RTOL
        with pytest.raises(KeyError):
            srv.resolve("no-such-model").result(timeout=600)
    finally:
        srv.close()


def test_server_shares_the_structure_of_a_resident_mesh():
    """Two wing panels of one mesh (different thicknesses): the second takes
    over the first's pattern and symbolic analysis and matches its own
    stand-alone solve; a thickness update and re-solve keep working."""
    a = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=2, seed=5)
    b = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=2, seed=6)
    be = B.JFEMGPUBackend(tol=RESID_TOL)
    ref = B.solve_model(be, b)
    Ub = np.stack([sc["raw_displacement"] for sc in ref["subcases"]], axis=1)
    ref["state"]["dm"].close()
    srv = S.SolveServer(slots=2, tol=RESID_TOL, small_dof=0)
    try:
        srv.solve(a).result(timeout=600)
        rb = srv.solve(b).result(timeout=600)
        assert srv.stats()["shared_structures"] == 1
        assert _rel(rb["U"], Ub) <= DISP_RTOL
        assert rb["rel_residual"].max() <= RESID_TOL
    finally:
        srv.close()


def test_autotune_picks_a_candidate_and_keeps_results(alone):
    """The autotuner times candidate schedules (nested-dissection leaf size,
    amalgamation thresholds, DMMA or SIMT updates) and every candidate gives
    the same displacements; the tuned options are cached per size class."""
    from jf_2026_05_25_b200 import autotune as AT
    m = M.stiffened_panel(SEEDS[0])
    cands = [{"JFG_ND_LEAF": "16", "JFG_RELAX_COLS": "16,48,128", "JFG_RELAX_ZEROS": "0.5,0.1,0.03", "JFG_DMMA": "1"},
             {"JFG_ND_LEAF": "48", "JFG_RELAX_COLS": "32,96,256", "JFG_RELAX_ZEROS": "0.7,0.2,0.08", "JFG_DMMA": "0"}]
    out = AT.tune(m, cands, repeats=1)
    assert out["best"] in cands
    assert AT.tuned_options(m) == out["best"]
    for opt in cands:
        AT.apply(opt)
        try:
            be = B.JFEMGPUBackend(tol=RESID_TOL)
            res = B.solve_model(be, m)
            U = np.stack([sc["raw_displacement"] for sc in res["subcases"]], axis=1)
            assert _rel(U, alone[SEEDS[0]]) <= DISP_RTOL
        finally:
            AT.apply({})


def test_server_device_resident_loads_match_host(alone):
    """Loads given as CUDA tensors (and displacements returned as CUDA
    tensors) give the same result as host buffers, for a packed batch of new
    models and for a re-solve."""
    import torch
    srv = S.SolveServer(slots=1, tol=RESID_TOL, small_dof=20000, pack_dof=40000)
    try:
        models = {s: M.stiffened_panel(s) for s in SEEDS[:3]}
        futs = {s: srv.solve(m, device_loads=torch.from_numpy(np.ascontiguousarray(m.load_matrix().T)).cuda())
                for s, m in models.items()}
        res = {s: f.result(timeout=600) for s, f in futs.items()}
        for s in models:
            U = res[s]["U"].cpu().numpy().T
            assert _rel(U, alone[s]) <= DISP_RTOL
            assert res[s]["rel_residual"].max() <= RESID_TOL
        s0 = SEEDS[0]
        F2 = torch.from_numpy(np.ascontiguousarray((3.0 * models[s0].load_matrix()).T)).cuda()
        r2 = srv.resolve(res[s0]["key"], F2).result(timeout=600)
        assert _rel(r2["U"].cpu().numpy().T, 3.0 * alone[s0]) <= DISP_RTOL
    finally:
        srv.close()


def test_mixed_server_moves_slow_meshes_to_the_fp64_factor():
    """In a mixed-precision server a mesh whose refinement needs more than
    `slow_refinement_steps` steps takes the FP64 factor for its later models
    (the threshold is 0 here, so the first model marks its mesh); both
    results meet the bar and match the FP64 solve."""
    a = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=2, seed=5)
    b = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=2, seed=6)
    ref = B.solve_model(B.JFEMGPUBackend(tol=RESID_TOL), b)
    Ub = np.stack([sc["raw_displacement"] for sc in ref["subcases"]], axis=1)
    ref["state"]["dm"].close()
    srv = S.SolveServer(slots=1, tol=RESID_TOL, small_dof=0, precision=lib.PREC_MIXED, slow_refinement_steps=0)
    try:
        ra = srv.solve(a).result(timeout=600)
        rb = srv.solve(b).result(timeout=600)
        st = srv.stats()
        assert st["fp64_meshes"] == 1 and st["fp64_factorisations"] == 1
        assert ra["rel_residual"].max() <= RESID_TOL and rb["rel_residual"].max() <= RESID_TOL
        assert rb["report"]["precision"] == lib.PREC_FP64
        assert _rel(rb["U"], Ub) <= DISP_RTOL
    finally:
        srv.close()


@pytest.mark.parametrize("prec", [lib.PREC_FP64, lib.PREC_MIXED])
def test_server_wing_boxes_and_solids_against_the_oracle(oracle_mod, prec):
    """Two wing-box panels of one mesh and two CTETRA10 blocks of one mesh,
    queued together on a four-slot server (single-model requests: the
    second model of each mesh waits for the first and shares its pattern
    and analysis), one of each with host load matrices passed in, and a
    re-solve of a block: every result equals the FP64 oracle's within the
    parity tolerance, on both precisions."""
    base = M.wing_panel(nx=24, ny=36, n_blades=3, blade_nz=4, n_cases=1, seed=5)
    wings = [M.wing_panel_variant(base, s, 3) for s in (1, 2)]
    blocks = [M.solid_block(n=6, n_cases=2, seed=s) for s in (3, 4)]
    srv = S.SolveServer(slots=4, precision=prec, tol=RESID_TOL, small_dof=1000, pack_dof=2000)
    try:
        futs = [srv.solve(wings[0]), srv.solve(wings[1], loads=wings[1].load_matrix()),
                srv.solve(blocks[0]), srv.solve(blocks[1], loads=blocks[1].load_matrix())]
        res = [f.result(timeout=900) for f in futs]
        assert srv.shared_structures >= 2
        for mdl, r in zip(wings + blocks, res):
            ref = oracle_mod.solve_reference(mdl)
            assert _rel(r["U"], ref["u"]) <= DISP_RTOL
            assert r["rel_residual"].max() <= RESID_TOL
        F2 = 3.0 * blocks[0].load_matrix()
        r2 = srv.resolve(res[2]["key"], F2).result(timeout=900)
        ref = oracle_mod.solve_reference(blocks[0])
        assert _rel(r2["U"], 3.0 * ref["u"]) <= DISP_RTOL
        tl = srv.stats()["timeline"]
        assert tl["shell"]["n"] == 2 and tl["solid"]["n"] == 2
    finally:
        srv.close()
