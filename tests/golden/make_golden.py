"""Generate the golden fixtures under tests/golden/ from the reference's decks.

Run once in a checkout that has the reference beside it, giving the
reference's root directory as the only argument:

    python tests/golden/make_golden.py <reference-root>

The GPU box never runs this.

For each example deck it writes ``<name>.json`` holding the model exactly as
the reference's parser would build it for these decks (node ids and
coordinates, CPS4/C3D8 connectivity by node id, element set ALL, one
material, model-wide thickness, the step's BCs and CLOADs) plus the stable
QA values the reference publishes for that deck:

* examples/cantilever.inp   - docs/examples.md:38-40, README.md:163,
                              docs/qa/v0.2.0-gate.md:119-123
* examples/cantilever3d.inp - docs/examples.md:102-104, docs/qa/v0.2.0-gate.md:63
* examples/plate_hole.inp   - docs/examples.md:60-64, docs/benchmarks/kirsch.md:14-16

The reader understands only the keywords these decks use (*NODE, *ELEMENT,
*NSET, *ELSET [GENERATE], *MATERIAL, *ELASTIC, *SOLID SECTION, *STEP,
*STATIC, *BOUNDARY, *CLOAD, *END STEP); it mirrors the reference parser's
semantics for them (crates/solvix-io/src/parser.rs:146-845: set names upper
cased, *BOUNDARY "set, first, last" expands to dofs first..=last, *CLOAD on
a set expands per node in set order, the last *SOLID SECTION data line sets
the model-wide thickness).
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

GOLDEN = {
    "cantilever": {
        "deck": "examples/cantilever.inp",
        "nodes": 205, "elements": 160, "iterations": 390, "residual": "6.933e-11",
        "max_disp_mm": "13.832", "max_von_mises_mpa": "79.483",
        "source": "docs/examples.md:38-40; README.md:163; docs/qa/v0.2.0-gate.md:119-123",
    },
    "cantilever3d": {
        "deck": "examples/cantilever3d.inp",
        "nodes": 1025, "elements": 640, "iterations": 562, "residual": "9.367e-11",
        "max_disp_mm": "13.719", "max_von_mises_mpa": "80.559",
        "source": "docs/examples.md:102-104; docs/qa/v0.2.0-gate.md:63",
    },
    "plate_hole": {
        "deck": "examples/plate_hole.inp",
        "nodes": 81, "elements": 64, "iterations": 77, "residual": "4.313e-11",
        "max_disp_mm": "0.006", "max_von_mises_mpa": "2.085",
        "max_nodal_von_mises_mpa": "2.927",
        "source": "docs/examples.md:60-64; docs/benchmarks/kirsch.md:14-16",
    },
}

KINDS = {"CPS3": 0, "CPS4": 1, "CPS8": 2, "CPE4": 3, "CPE8": 4, "C3D8": 5, "C3D4": 6, "B31": 7}


def _params(parts):
    out = {}
    for p in parts[1:]:
        if "=" in p:
            k, v = p.split("=", 1)
            out[k.strip().lower()] = v.strip()
        else:
            out[p.strip().lower()] = ""
    return out


def read_deck(text: str) -> dict:
    nodes, elements = [], []
    nsets, elsets = {}, {}
    materials, assignments = [], []
    thickness = 1.0
    bcs, cloads = [], []
    kw, params = None, {}
    cur_mat = None
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line.startswith("**"):
            continue
        if line.startswith("*"):
            parts = [s.strip() for s in line[1:].split(",")]
            kw = parts[0].lower()
            params = _params(parts)
            if kw == "material":
                cur_mat = {"name": params["name"].upper(), "E": None, "nu": None}
                materials.append(cur_mat)
            if kw == "solid section":
                assignments.append([params["elset"].upper(), params["material"].upper()])
            continue
        f = [s.strip() for s in line.split(",") if s.strip() != ""]
        if kw == "node":
            xyz = [float(x) for x in f[1:]] + [0.0] * (4 - len(f))
            nodes.append([int(f[0]), xyz[:3]])
        elif kw == "element":
            eid = int(f[0])
            elements.append([eid, KINDS[params["type"].upper()], [int(x) for x in f[1:]]])
            if "elset" in params:
                elsets.setdefault(params["elset"].upper(), []).append(eid)
        elif kw in ("nset", "elset"):
            name = params.get(kw).upper()
            if "generate" in params:
                a, b, s = (int(x) for x in f)
                ids = list(range(a, b + 1, s))
            else:
                ids = [int(x) for x in f]
            target = nsets if kw == "nset" else elsets
            target.setdefault(name, []).extend(ids)
        elif kw == "elastic":
            cur_mat["E"], cur_mat["nu"] = float(f[0]), float(f[1])
        elif kw == "solid section":
            thickness = float(f[0])
        elif kw == "boundary":
            node_ids = nsets[f[0].upper()] if not f[0].isdigit() else [int(f[0])]
            d1 = int(f[1])
            d2 = int(f[2]) if len(f) >= 3 else d1
            bcs.append({"node_ids": list(node_ids), "dofs": list(range(d1, d2 + 1))})
        elif kw == "cload":
            node_ids = nsets[f[0].upper()] if not f[0].isdigit() else [int(f[0])]
            for nid in node_ids:
                cloads.append({"node_id": nid, "dof": int(f[1]), "value": float(f[2])})
    return {
        "nodes": nodes, "elements": elements,
        "elsets": [{"name": k, "element_ids": v} for k, v in elsets.items()],
        "materials": materials, "mat_assignments": assignments, "thickness": thickness,
        "boundary_conditions": bcs, "cloads": cloads,
    }


def main(ref_root: str) -> None:
    for name, gold in GOLDEN.items():
        with open(os.path.join(ref_root, gold["deck"])) as fh:
            model = read_deck(fh.read())
        out = {"model": model, "golden": gold}
        path = os.path.join(HERE, f"{name}.json")
        with open(path, "w") as fh:
            json.dump(out, fh, separators=(",", ":"))
        print(f"wrote {path}: {len(model['nodes'])} nodes, {len(model['elements'])} elements")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference-root>")
    main(sys.argv[1])
