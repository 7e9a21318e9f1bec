"""Regenerate the golden fixtures in this directory from the reference tree.

Run in a container that has the OpenJFEM reference checked out; its path is
the one required argument.  It reads test and validation files as text only:

* utils/test/quad8_shell_test.jl -- CQUAD8 single-element stiffness entries
  produced by an external reference solver (rtol 2e-6 in the reference test).
* validation/cases/MYSTRAN_sol101_simple/{model.bdf, results/sol101_simple.JU.JSON}
  -- one flat CQUAD4, three subcases, full-precision displacements and SPC
  forces written by the reference's own SOL101 parity path.

The fixtures are committed; the tests never read the reference tree.
"""
import json
import os
import re
import sys


def quad8_tables(ref):
    src = open(os.path.join(ref, "utils/test/quad8_shell_test.jl")).read()
    out = {}
    for name in ("SQUARE_THIN", "SQUARE_THICK", "RECTANGLE_5_1", "RHOMBUS_60", "SQUARE_NO_MID3"):
        m = re.search(r"const %s = \((.*?)\)\n" % name, src, re.S)
        body = m.group(1)
        rows = re.findall(r"\((\d+),(\d+),(\d+),(\d+),([-+0-9.eE]+)\)", body)
        out[name] = [[int(a), int(b), int(c), int(d), float(v)] for a, b, c, d, v in rows]
    return {
        "source": "utils/test/quad8_shell_test.jl:24-46",
        "E": 7e10,
        "cases": {
            "SQUARE_THIN": {"a": 0.3, "b": 0.3, "angle": 90.0, "t": 0.003, "nu": 0.33, "mid3": True},
            "SQUARE_THICK": {"a": 0.3, "b": 0.3, "angle": 90.0, "t": 0.03, "nu": 0.33, "mid3": True},
            "RECTANGLE_5_1": {"a": 0.5, "b": 0.1, "angle": 90.0, "t": 0.003, "nu": 0.33, "mid3": True},
            "RHOMBUS_60": {"a": 0.3, "b": 0.3, "angle": 60.0, "t": 0.003, "nu": 0.33, "mid3": True},
            "SQUARE_NO_MID3": {"a": 0.3, "b": 0.3, "angle": 90.0, "t": 0.003, "nu": 0.33, "mid3": False},
        },
        "tables": out,
        "rtol": 2e-6,
    }


def mystran(ref):
    base = os.path.join(ref, "validation/cases/MYSTRAN_sol101_simple")
    ju = json.load(open(os.path.join(base, "results/sol101_simple.JU.JSON")))
    disp = ju["displacements"]
    spc = ju["spc_forces"]
    n_sub = 3
    per = len(disp) // n_sub
    comps = ("t1", "t2", "t3", "r1", "r2", "r3")
    cases = []
    for k in range(n_sub):
        d = {str(r["grid_id"]): [r[c] for c in comps] for r in disp[k * per:(k + 1) * per]}
        cases.append({"displacements": d})
    per_s = len(spc) // n_sub
    for k in range(n_sub):
        cases[k]["spc_forces"] = {str(r["grid_id"]): [r[c] for c in comps] for r in spc[k * per_s:(k + 1) * per_s]}
    rel = [sd["details"]["linear_solver"]["relative_residual"] for sd in ju["solver_diagnostics"]
           if "details" in sd and "linear_solver" in sd["details"]]
    return {
        "source": "validation/cases/MYSTRAN_sol101_simple (model.bdf, results/sol101_simple.JU.JSON)",
        "model": {
            "grids": {"1011": [0.0, 0.0, 0.0], "1012": [50.0, 0.0, 0.0], "1013": [50.0, 50.0, 0.0],
                      "1014": [0.0, 50.0, 0.0]},
            "cquad4": [11, 91, [1011, 1012, 1013, 1014]],
            "pshell": {"PID": 91, "MID1": 20, "T": 0.1, "MID2": 20, "BEND_RATIO": 1.0, "MID3": 20,
                       "TS_T": 0.83333},
            "mat1": {"MID": 20, "E": 1.0e7, "G": 4.0e6, "NU": 0.25},
            "k6rot": 0.0,
            "spc1": ["123456", [1011, 1012]],
            "subcases": [
                {"force": [[1011, 1000.0, [1.0, 1.0, 0.0]], [1012, 1000.0, [1.0, 1.0, 0.0]],
                           [1013, 1000.0, [1.0, 1.0, 0.0]]]},
                {"pload2": [11, 1.1]},
                {"pload4": [11, 1.1]},
            ],
        },
        "results": cases,
        "relative_residuals": rel,
    }


def _nastran_float(s):
    s = s.strip()
    if not s:
        return None
    # "1.0+7" style exponents
    m = re.match(r"^([-+]?[0-9.]+)([-+][0-9]+)$", s)
    if m and "e" not in s.lower():
        return float(m.group(1) + "e" + m.group(2))
    return float(s)


def free_field_deck(path):
    """GRID / CQUAD4 / SPC1 / FORCE / MAT1 / PSHELL / PARAM,K6ROT of a free-field deck."""
    out = {"grids": {}, "cquad4": [], "spc1": [], "force": [], "mat1": {}, "pshell": {}, "k6rot": 100.0}
    for line in open(path):
        if line.startswith("$") or "," not in line:
            continue
        f = [x.strip() for x in line.rstrip("\n").split(",")]
        card = f[0].upper()
        if card == "GRID":
            out["grids"][int(f[1])] = [_nastran_float(f[3]), _nastran_float(f[4]), _nastran_float(f[5])]
        elif card == "CQUAD4":
            out["cquad4"].append([int(f[1]), int(f[2]), [int(x) for x in f[3:7]]])
        elif card == "SPC1":
            out["spc1"].append([f[2], [int(x) for x in f[3:] if x]])
        elif card == "FORCE":
            out["force"].append([int(f[2]), _nastran_float(f[4]), [_nastran_float(x) for x in f[5:8]]])
        elif card == "MAT1":
            out["mat1"] = {"MID": int(f[1]), "E": _nastran_float(f[2]), "G": _nastran_float(f[3]) or 0.0,
                           "NU": _nastran_float(f[4])}
        elif card == "PSHELL":
            out["pshell"] = {"PID": int(f[1]), "MID1": int(f[2]), "T": _nastran_float(f[3]),
                             "MID2": int(f[4]) if len(f) > 4 and f[4] else 0}
        elif card == "PARAM" and f[1].upper() == "K6ROT":
            out["k6rot"] = _nastran_float(f[2])
    return out


def curved_beams(ref):
    """Flat, tapered CQUAD4 membrane decks and the current-source scalars.

    validation/comparison.csv holds the run of the present source (the per-case
    JU.JSON files keep older recorded revisions); its ``jfem`` column is the
    reference's own SOL101 result for these decks.
    """
    import csv
    rows = {r["case_id"]: r for r in csv.DictReader(open(os.path.join(ref, "validation/comparison.csv")))}
    out = {"source": "validation/cases/MH_curved_beam_{in_plane,refined}/model.bdf; validation/comparison.csv",
           "cases": {}}
    for case, node in (("MH_curved_beam_in_plane", 7), ("MH_curved_beam_refined", 75)):
        deck = free_field_deck(os.path.join(ref, "validation/cases", case, "model.bdf"))
        out["cases"][case] = {"deck": deck, "node": node, "dof": 2,
                              "jfem_current": float(rows[case]["jfem"]),
                              "published": float(rows[case]["reference"])}
    out["mystran_T1_node_1013_current"] = float(rows["MYSTRAN_sol101_simple"]["jfem"])
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the OpenJFEM reference checkout>")
    ref = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    json.dump(quad8_tables(ref), open(os.path.join(here, "quad8_entries.json"), "w"), indent=1)
    json.dump(mystran(ref), open(os.path.join(here, "mystran_sol101_simple.json"), "w"), indent=1)
    json.dump(curved_beams(ref), open(os.path.join(here, "curved_beam_membrane.json"), "w"), indent=1)
    print("wrote fixtures to", here)


if __name__ == "__main__":
    main()
