"""Nastran bulk-data decks of the generated models, so the reference's own
Julia SOL101 path can be run on identical inputs elsewhere.

``write_bdf`` writes SOL 101 with one SUBCASE per load case: GRID (large
field, full double precision), CQUAD4 / CQUAD8 / CTETRA (10 grids), PSHELL,
PSOLID, MAT1, SPC1, PLOAD4, FORCE and PARAM,K6ROT.  The reference's bulk-data
CTETRA reader keeps four grids, so CTETRA10 models go to the reference as
Abaqus keyword input (``write_inp``: C3D10 and *CLOAD), which keeps all ten.  ``read_bdf`` reads those
decks back (used by the round-trip tests; it understands exactly the cards
written here).  ``write_reference_driver`` writes ``reproduce_reference.jl``,
a driver for a machine with Julia and the reference package: it builds each
deck with the reference's ``bdf_to_model`` and solves it with its
``solve_model`` (JFEMSolver.jl:69, :2132), then stores every subcase's raw
displacements, SPC forces and the element stiffness capture as JSON goldens.
Julia is not installed here, so the driver is shipped, not run.

Thickness per CQUAD4 is carried by one PSHELL per distinct section, so the
seeded per-row skin thicknesses of the wing panel survive the round trip.
"""
from __future__ import annotations

import math
import os
from typing import Dict, List, Tuple

import numpy as np

from . import model as M


def _f16(v: float) -> str:
    """A real in a 16-character large field: exact when repr fits, otherwise
    the most significant digits that fit (Nastran exponent form, 1.25-3)."""
    v = float(v)
    s = repr(v)
    if len(s) <= 16:
        return s.rjust(16)
    for prec in range(15, 0, -1):
        m, e = ("%.*e" % (prec, v)).split("e")
        t = m + ("-" if e.startswith("-") else "+") + (e.lstrip("+-").lstrip("0") or "0")
        if len(t) <= 16:
            return t.rjust(16)
    raise ValueError(f"{v} does not fit a 16-character field")


def _f8(v) -> str:
    """A small-field value (integers and short reals)."""
    if isinstance(v, (int, np.integer)):
        return str(int(v)).rjust(8)
    v = float(v)
    for fmt in ("%.6g", "%.5g", "%.4g", "%.3g"):
        s = fmt % v
        if "e" in s:
            m, e = s.split("e")
            if "." not in m:
                m += "."
            s = m + ("-" if e.startswith("-") else "+") + e.lstrip("+-").lstrip("0")
        if len(s) <= 8:
            if "." not in s and "e" not in s and "+" not in s[1:] and "-" not in s[1:]:
                s += "."
            if len(s) <= 8:
                return s.rjust(8)
    raise ValueError(f"{v} does not fit an 8-character field")


def _card(name: str, fields: List) -> List[str]:
    """Small-field card with continuation lines (8 data fields per line)."""
    out, line = [], name.ljust(8)
    for k, f in enumerate(fields):
        if k > 0 and k % 8 == 0:
            out.append(line)
            line = " " * 8
        line += f if isinstance(f, str) else _f8(f)
    out.append(line)
    return out


def write_bdf(model, path: str, title: str = "") -> str:
    """Write `model` as a SOL 101 deck; returns the path."""
    gid = np.asarray(model.grid_ids, np.int64)
    lines = ["SOL 101", "CEND", f"TITLE = {title or model.name}", "DISP = ALL", "SPCFORCE = ALL", "SPC = 1"]
    for lc in model.load_cases:
        lines += [f"SUBCASE {lc.sid}", f"  LOAD = {100 + lc.sid}"]
    lines += ["BEGIN BULK", "PARAM,K6ROT," + repr(float(model.k6rot))]
    for m_id, mt in sorted(model.mats.items()):
        lines.append("MAT1*".ljust(8) + str(m_id).rjust(16) + _f16(mt.E) + (_f16(mt.G) if mt.G else " " * 16) +
                     _f16(mt.NU))
        lines.append("*".ljust(8) + _f16(mt.RHO))
    # one PSHELL per distinct property id (thicknesses keep full precision)
    for pid, p in sorted(model.pshells.items()):
        lines.append("PSHELL*".ljust(8) + str(pid).rjust(16) + str(p.MID1).rjust(16) + _f16(p.T) +
                     str(p.MID2).rjust(16))
        lines.append("*".ljust(8) + _f16(p.BEND_RATIO) + str(p.MID3).rjust(16) + _f16(p.TS_T) + " " * 16)
    for pid, mid in sorted(model.psolids.items()):
        lines += _card("PSOLID", [pid, mid])
    R = model.node_R
    ident = np.allclose(R, np.tile([1, 0, 0, 0, 1, 0, 0, 0, 1], (model.n_nodes, 1)))
    if not ident:
        raise ValueError("write_bdf writes basic-frame grids only (node_R must be the identity)")
    for k in range(model.n_nodes):
        x, y, z = model.xyz[k]
        lines.append("GRID*".ljust(8) + str(int(gid[k])).rjust(16) + "".rjust(16) + _f16(x) + _f16(y))
        lines.append("*".ljust(8) + _f16(z))
    eid = 1
    q4eid = getattr(model, "q4_eid", None)
    for e, nd in enumerate(model.q4_nodes):
        this = int(q4eid[e]) if q4eid is not None and len(q4eid) == len(model.q4_nodes) else eid
        lines += _card("CQUAD4", [this, int(model.q4_pid[e])] + [int(gid[n]) for n in nd])
        eid = max(eid, this) + 1
    t3_first = eid
    for e, nd in enumerate(getattr(model, "t3_nodes", ())):
        lines += _card("CTRIA3", [eid, int(model.t3_pid[e])] + [int(gid[n]) for n in nd])
        eid += 1
    for e, nd in enumerate(model.q8_nodes):
        lines += _card("CQUAD8", [eid, int(model.q8_pid[e])] + [int(gid[n]) for n in nd])
        eid += 1
    for e, nd in enumerate(model.t10_nodes):
        lines += _card("CTETRA", [eid, int(model.t10_pid[e])] + [int(gid[n]) for n in nd])
        eid += 1
    for comp, nodes in model.spc1:
        ids = [int(gid[n]) for n in np.asarray(nodes)]
        for k in range(0, len(ids), 6):
            lines += _card("SPC1", [1, comp.rjust(8)] + ids[k:k + 6])
    q4e = np.asarray(q4eid) if q4eid is not None and len(q4eid) == len(model.q4_nodes) else None
    for lc in model.load_cases:
        sid = 100 + lc.sid
        if lc.pload4 is not None:
            eidx, pres = lc.pload4
            for k, e in enumerate(np.asarray(eidx)):
                ee = int(q4e[e]) if q4e is not None else int(e) + 1
                lines.append("PLOAD4*".ljust(8) + str(sid).rjust(16) + str(ee).rjust(16) + _f16(pres[k]))
        if getattr(lc, "pload4_t3", None) is not None:
            eidx, pres = lc.pload4_t3
            for k, e in enumerate(np.asarray(eidx)):
                lines.append("PLOAD4*".ljust(8) + str(sid).rjust(16) + str(t3_first + int(e)).rjust(16) +
                             _f16(pres[k]))
        for part in (lc.forces, lc.cload):
            if part is None:
                continue
            nidx, vec = part
            for k, n in enumerate(np.asarray(nidx)):
                v = np.asarray(vec[k], float)
                mag = float(np.linalg.norm(v))
                if mag == 0.0:
                    continue
                d = v / mag
                lines.append("FORCE*".ljust(8) + str(sid).rjust(16) + str(int(gid[n])).rjust(16) +
                             "0".rjust(16) + _f16(mag))
                lines.append("*".ljust(8) + _f16(d[0]) + _f16(d[1]) + _f16(d[2]))
    lines.append("ENDDATA")
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


# ----------------------------------------------------------------------------
# reader (the cards written above)
# ----------------------------------------------------------------------------

def _fields(card_lines: List[str]) -> Tuple[str, List[str]]:
    first = card_lines[0]
    name = first[:8].strip()
    large = name.endswith("*")
    w = 16 if large else 8
    vals = []
    for k, ln in enumerate(card_lines):
        body = ln[8:]
        n = 4 if large else 8
        for i in range(n):
            vals.append(body[i * w:(i + 1) * w].strip())
    return name.rstrip("*"), vals


def _real(s: str) -> float:
    s = s.strip()
    if not s:
        return 0.0
    try:
        return float(s)
    except ValueError:   # Nastran exponent without 'E' (1.5-3)
        for i in range(len(s) - 1, 0, -1):
            if s[i] in "+-" and s[i - 1] not in "eE":
                return float(s[:i] + "E" + s[i:])
        raise


def read_bdf(path: str) -> "M.Sol101Model":
    lines = [ln.rstrip("\n") for ln in open(path)]
    bulk = lines[lines.index("BEGIN BULK") + 1:]
    cards: List[List[str]] = []
    k6rot = 100.0
    for ln in bulk:
        if ln.startswith("ENDDATA"):
            break
        if ln.startswith("PARAM,K6ROT,"):
            k6rot = float(ln.split(",")[2])
            continue
        if ln.startswith(" ") or ln.startswith("*"):
            cards[-1].append(ln)
        else:
            cards.append([ln])
    grids, mats, pshells, psolids = {}, {}, {}, {}
    q4, q8, t3, t10, spc, loads = [], [], [], [], [], {}
    for c in cards:
        name, v = _fields(c)
        if name == "GRID":
            grids[int(v[0])] = (_real(v[2]), _real(v[3]), _real(v[4]))
        elif name == "MAT1":
            mats[int(v[0])] = M.Mat1(E=_real(v[1]), NU=_real(v[3]), G=_real(v[2]), RHO=_real(v[4]))
        elif name == "PSHELL":
            pshells[int(v[0])] = M.PShell(T=_real(v[2]), MID1=int(v[1]), MID2=int(v[3]), MID3=int(v[5]),
                                          BEND_RATIO=_real(v[4]), TS_T=_real(v[6]))
        elif name == "PSOLID":
            psolids[int(v[0])] = int(v[1])
        elif name == "CQUAD4":
            q4.append((int(v[0]), int(v[1]), [int(x) for x in v[2:6]]))
        elif name == "CQUAD8":
            q8.append((int(v[0]), int(v[1]), [int(x) for x in v[2:10]]))
        elif name == "CTRIA3":
            t3.append((int(v[0]), int(v[1]), [int(x) for x in v[2:5]]))
        elif name == "CTETRA":
            t10.append((int(v[0]), int(v[1]), [int(x) for x in v[2:12]]))
        elif name == "SPC1":
            spc.append((v[1], [int(x) for x in v[2:] if x]))
        elif name == "PLOAD4":
            loads.setdefault(int(v[0]), {"p4": [], "f": []})["p4"].append((int(v[1]), _real(v[2])))
        elif name == "FORCE":
            mag = _real(v[3])
            d = np.array([_real(v[4]), _real(v[5]), _real(v[6])])
            loads.setdefault(int(v[0]), {"p4": [], "f": []})["f"].append((int(v[1]), mag * d))
    gid = np.array(sorted(grids), np.int64)
    pos = {g: i for i, g in enumerate(gid)}
    xyz = np.array([grids[g] for g in gid], float)
    q4eid = np.array([e for e, _, _ in q4], np.int64)
    epos = {e: i for i, e in enumerate(q4eid)}
    t3pos = {e: i for i, (e, _, _) in enumerate(t3)}
    model = M.Sol101Model(
        name=os.path.basename(path), grid_ids=gid, xyz=xyz,
        q4_nodes=np.array([[pos[g] for g in n] for _, _, n in q4], np.int32).reshape(-1, 4),
        q4_pid=np.array([p for _, p, _ in q4], np.int64), q4_eid=q4eid,
        q8_nodes=np.array([[pos[g] for g in n] for _, _, n in q8], np.int32).reshape(-1, 8),
        q8_pid=np.array([p for _, p, _ in q8], np.int64),
        t3_nodes=np.array([[pos[g] for g in n] for _, _, n in t3], np.int32).reshape(-1, 3),
        t3_pid=np.array([p for _, p, _ in t3], np.int64),
        t10_nodes=np.array([[pos[g] for g in n] for _, _, n in t10], np.int32).reshape(-1, 10),
        t10_pid=np.array([p for _, p, _ in t10], np.int64),
        pshells=pshells, psolids=psolids, mats=mats, k6rot=k6rot,
        spc1=[(comp, np.array([pos[g] for g in ids], np.int64)) for comp, ids in spc])
    for sid in sorted(loads):
        ld = loads[sid]
        p4 = p4t = None
        on_q4 = [(e, p) for e, p in ld["p4"] if e in epos]
        on_t3 = [(e, p) for e, p in ld["p4"] if e not in epos and e in t3pos]
        if on_q4:
            p4 = (np.array([epos[e] for e, _ in on_q4]), np.array([p for _, p in on_q4]))
        if on_t3:
            p4t = (np.array([t3pos[e] for e, _ in on_t3]), np.array([p for _, p in on_t3]))
        fr = None
        if ld["f"]:
            nodes = np.array([pos[g] for g, _ in ld["f"]])
            fr = (nodes, np.array([f for _, f in ld["f"]]))
        model.load_cases.append(M.LoadCase(sid=sid - 100, pload4=p4, pload4_t3=p4t, forces=fr))
    return model


# ----------------------------------------------------------------------------
# Abaqus keyword input for CTETRA10 models
# ----------------------------------------------------------------------------

def write_inp(model, path: str, title: str = "") -> str:
    """Abaqus keyword input of a CTETRA10 model: the reference's entry for
    ten-node tetrahedra (its bulk-data CTETRA reader keeps only four grids,
    src/parsing/extract_elements.jl:205-229; the Abaqus reader keeps all ten,
    src/abaqus_input.jl:7-12).  *NODE (full double precision), *ELEMENT
    TYPE=C3D10 (corners, then mid-edge nodes 1-2, 2-3, 3-1, 1-4, 2-4, 3-4, the
    node order of the generated elements), one *MATERIAL / *ELASTIC and
    *SOLID SECTION per solid property, the SPC1 translations as a model-level
    *BOUNDARY on node sets, and one *STEP / *STATIC per subcase whose nodal
    loads are a *CLOAD with OP=NEW (the reference turns step k into subcase k,
    :455-545).  Shell elements have no Abaqus form here."""
    if len(model.q4_nodes) or len(model.q8_nodes):
        raise ValueError("write_inp writes CTETRA10 models only")
    gid = np.asarray(model.grid_ids)
    lines = ["*HEADING", title or model.name, "*NODE"]
    for i in range(model.n_nodes):
        x, y, z = model.xyz[i]
        lines.append(f"{int(gid[i])}, {float(x)!r}, {float(y)!r}, {float(z)!r}")
    pids = np.asarray(model.t10_pid)
    eid0 = 1
    for pid in np.unique(pids):
        lines.append(f"*ELEMENT, TYPE=C3D10, ELSET=P{int(pid)}")
        for e in np.where(pids == pid)[0]:
            lines.append(", ".join([str(eid0 + int(e))] + [str(int(gid[n])) for n in model.t10_nodes[e]]))
    for mid in sorted({model.psolids[int(p)] for p in np.unique(pids)}):
        m = model.mats[mid]
        lines += [f"*MATERIAL, NAME=M{mid}", "*ELASTIC", f"{float(m.E)!r}, {float(m.NU)!r}"]
        if m.RHO:
            lines += ["*DENSITY", f"{float(m.RHO)!r}"]
    for pid in np.unique(pids):
        lines.append(f"*SOLID SECTION, ELSET=P{int(pid)}, MATERIAL=M{model.psolids[int(pid)]}")
    for k, (comps, nodes) in enumerate(model.spc1):
        name = f"SPC{k + 1}"
        lines.append(f"*NSET, NSET={name}")
        ids = [str(int(gid[n])) for n in np.asarray(nodes)]
        for a in range(0, len(ids), 16):
            lines.append(", ".join(ids[a:a + 16]))
        lines.append("*BOUNDARY")
        for ch in comps:
            if int(ch) > 3:
                continue          # continuum grids carry translations only
            lines.append(f"{name}, {int(ch)}, {int(ch)}")
    for c in model.load_cases:
        lines += [f"*STEP, NAME=SUBCASE{c.sid}", "*STATIC", "*CLOAD, OP=NEW"]
        acc = {}
        for item in (c.forces, c.cload):
            if item is None:
                continue
            nidx, vec = item
            for n, v in zip(np.asarray(nidx), np.asarray(vec, float)):
                a = acc.setdefault(int(n), np.zeros(3))
                a += v
        if c.pload4 is not None:
            raise ValueError("PLOAD4 has no CTETRA10 form; deliver face loads as nodal loads")
        for n in sorted(acc):
            for d in range(3):
                if acc[n][d] != 0.0:
                    lines.append(f"{int(gid[n])}, {d + 1}, {float(acc[n][d])!r}")
        lines.append("*END STEP")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def read_inp(path: str) -> "M.Sol101Model":
    """Read back a deck written by ``write_inp`` (exactly those keywords)."""
    nodes, elems, mats, sections, nsets, bnd, steps = {}, {}, {}, {}, {}, [], []
    key, opts, cur = None, {}, None
    for raw in open(path):
        line = raw.strip()
        if not line or line.startswith("**"):
            continue
        if line.startswith("*"):
            parts = [t.strip() for t in line[1:].split(",")]
            key = parts[0].upper()
            opts = dict((t.split("=", 1)[0].upper(), t.split("=", 1)[1] if "=" in t else "") for t in parts[1:])
            if key == "STEP":
                cur = {"name": opts.get("NAME", ""), "loads": []}
                steps.append(cur)
            elif key == "MATERIAL":
                mats[opts["NAME"]] = {}
            elif key == "SOLID SECTION":
                sections[opts["ELSET"]] = opts["MATERIAL"]
            elif key == "NSET":
                nsets[opts["NSET"]] = []
            continue
        f = [t.strip() for t in line.split(",")]
        if key == "NODE":
            nodes[int(f[0])] = [float(v) for v in f[1:4]]
        elif key == "ELEMENT":
            elems[int(f[0])] = (opts["ELSET"], [int(v) for v in f[1:11]])
        elif key == "ELASTIC":
            mats[list(mats)[-1]]["E"], mats[list(mats)[-1]]["NU"] = float(f[0]), float(f[1])
        elif key == "DENSITY":
            mats[list(mats)[-1]]["RHO"] = float(f[0])
        elif key == "NSET":
            nsets[list(nsets)[-1]] += [int(v) for v in f if v]
        elif key == "BOUNDARY":
            bnd.append((f[0], int(f[1]), int(f[2])))
        elif key == "CLOAD":
            cur["loads"].append((int(f[0]), int(f[1]), float(f[2])))
    gids = np.array(sorted(nodes), dtype=np.int64)
    idx = {g: i for i, g in enumerate(gids)}
    xyz = np.array([nodes[g] for g in gids])
    eids = sorted(elems)
    t10 = np.array([[idx[g] for g in elems[e][1]] for e in eids], np.int32)
    set_pid = {name: int(name[1:]) for name in sections}
    pid = np.array([set_pid[elems[e][0]] for e in eids], np.int64)
    mid_of = {name: int(name[1:]) for name in mats}
    psolids = {set_pid[s]: mid_of[m] for s, m in sections.items()}
    mats_out = {mid_of[n]: M.Mat1(E=v["E"], NU=v["NU"], RHO=v.get("RHO", 0.0)) for n, v in mats.items()}
    spc = {}
    for name, a, b in bnd:
        spc.setdefault(name, "")
        spc[name] += "".join(str(c) for c in range(a, b + 1))
    spc1 = [(comps, np.array([idx[g] for g in nsets[name]])) for name, comps in spc.items()]
    cases = []
    for k, st in enumerate(steps):
        vec = {}
        for g, d, v in st["loads"]:
            vec.setdefault(idx[g], np.zeros(3))[d - 1] += v
        ns = np.array(sorted(vec), np.int64)
        cases.append(M.LoadCase(sid=k + 1, cload=(ns, np.array([vec[n] for n in ns]).reshape(-1, 3))))
    return M.Sol101Model(name=os.path.basename(path), grid_ids=gids, xyz=xyz, t10_nodes=t10, t10_pid=pid,
                         psolids=psolids, mats=mats_out, spc1=spc1, load_cases=cases)


DRIVER = r'''# reproduce_reference.jl -- run the reference's own SOL101 on decks written by
# jf_2026_05_25_b200.decks (write_bdf for shell models, write_inp for CTETRA10
# models) and store its results as JSON goldens.
#
#   julia --project=<reference checkout> reproduce_reference.jl out_dir deck1.bdf [deck2.inp ...]
#
# For every deck: model = input_to_model(deck) (JFEMSolver.jl:44-46: Abaqus
# keyword input for .inp, bulk data otherwise), results = solve_model(model)
# (JFEMSolver.jl:2132, parity backend), then <deck>.golden.json with, per
# subcase, raw_displacement (ndof, global DOF order 6*(sorted GRID index) +
# component) and the SPC forces.
using OpenJFEM
using JSON

out_dir = ARGS[1]
mkpath(out_dir)
for deck in ARGS[2:end]
    model = OpenJFEM.input_to_model(deck)
    results = OpenJFEM.solve_model(model)
    gold = Dict{String,Any}("deck" => basename(deck), "ndof" => results["ndof"], "subcases" => Any[])
    for sc in results["subcases"]
        push!(gold["subcases"], Dict("raw_displacement" => collect(sc["raw_displacement"]),
                                     "spc_forces" => sc["spc_forces"]))
    end
    open(joinpath(out_dir, basename(deck) * ".golden.json"), "w") do io
        JSON.print(io, gold)
    end
end
'''


def write_reference_driver(path: str) -> str:
    with open(path, "w") as f:
        f.write(DRIVER)
    return path
