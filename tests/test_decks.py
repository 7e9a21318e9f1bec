"""Bulk-data decks of the generated models (for running the reference on the
same inputs): write, read back, and get the same model and loads."""
import os

import numpy as np

from jf_2026_05_25_b200 import decks as D
from jf_2026_05_25_b200 import model as M


def _same(a, b, exact):
    """exact: equal arrays; otherwise equal to the 12 significant digits a
    16-character field keeps."""
    def eq(x, y):
        if exact:
            return np.array_equal(x, y)
        return np.allclose(x, y, rtol=1e-12, atol=1e-12 * max(np.abs(x).max(initial=0.0), 1e-300))
    assert np.array_equal(a.grid_ids, b.grid_ids)
    assert eq(a.xyz, b.xyz)
    for f in ("q4_nodes", "q8_nodes", "t3_nodes", "t10_nodes"):
        assert np.array_equal(getattr(a, f), getattr(b, f))
    if len(a.t3_nodes):
        assert eq(a.t3_sections(), b.t3_sections())
    if len(a.q4_nodes):
        assert eq(a.q4_sections(), b.q4_sections())
    if len(a.q8_nodes):
        assert eq(a.q8_sections(), b.q8_sections())
    if len(a.t10_nodes):
        assert eq(a.t10_materials(), b.t10_materials())
    assert np.array_equal(np.sort(a.spc_dofs()), np.sort(b.spc_dofs()))
    # FORCE is written as magnitude x direction, so loads are compared to the
    # field precision even when the geometry must match exactly
    Fa, Fb = a.load_matrix(), b.load_matrix()
    assert Fa.shape == Fb.shape
    assert np.allclose(Fa, Fb, rtol=1e-12, atol=1e-12 * np.abs(Fa).max())


def test_round_trip_plate_wing_q8_solid(tmp_path):
    models = [M.flat_plate(nx=6, ny=5),
              M.wing_panel(nx=12, ny=10, n_blades=2, blade_nz=3, n_cases=3, seed=4),
              M.quad8_plate(4, 3, n_cases=2),
              M.tria_plate(nx=6, ny=4, n_cases=2),
              M.solid_block(n=2, n_cases=1)]
    for k, m in enumerate(models):
        path = D.write_bdf(m, os.path.join(tmp_path, f"m{k}.bdf"))
        r1 = D.read_bdf(path)
        _same(m, r1, exact=False)
        # the deck is the reference input: writing what was read changes nothing
        r2 = D.read_bdf(D.write_bdf(r1, os.path.join(tmp_path, f"m{k}b.bdf")))
        _same(r1, r2, exact=True)


def test_reference_driver_is_written(tmp_path):
    p = D.write_reference_driver(os.path.join(tmp_path, "reproduce_reference.jl"))
    txt = open(p).read()
    assert "input_to_model" in txt and "solve_model" in txt


def test_solid_block_abaqus_round_trip(tmp_path):
    """CTETRA10 models go to the reference as Abaqus C3D10 input (its bulk-
    data CTETRA keeps only four grids): all ten nodes per element, the base
    translations as *BOUNDARY, one step with *CLOAD OP=NEW per subcase."""
    m = M.solid_block(n=2, n_cases=3)
    path = D.write_inp(m, os.path.join(tmp_path, "block.inp"))
    txt = open(path).read()
    assert "*ELEMENT, TYPE=C3D10" in txt and txt.count("*STEP") == 3 and txt.count("*CLOAD, OP=NEW") == 3
    r = D.read_inp(path)
    _same(m, r, exact=True)
    r2 = D.read_inp(D.write_inp(r, os.path.join(tmp_path, "block2.inp")))
    _same(r, r2, exact=True)
