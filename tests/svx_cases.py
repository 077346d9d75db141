"""Shared test cases: fixture loading, deck generators, Rust-style formatting.

Deck generators follow the patterns the reference documents for its bench
and refinement decks (crates/solvix-cli/src/bench.rs:616-784,
docs/benchmarks/cantilever.md:1-17): coordinates are written with six
decimals and read back, exactly as the parser sees them.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from solvix_b200.model import (BoundaryCondition, ConcentratedLoad, ElemKind,  # noqa: E402
                               Element, ElementSet, Material, Mesh, Model, Node)

GOLDEN_DIR = os.path.join(HERE, "golden")

E_STEEL = 210e9
NU_STEEL = 0.3


def fmt_e3(x: float) -> str:
    """Rust ``{:.3e}`` (crates/solvix-cli/src/main.rs:322-324)."""
    if not math.isfinite(x):
        x = 0.0
    m, e = f"{x:.3e}".split("e")
    return f"{m}e{int(e)}"


def fmt_mm(m: float) -> str:
    """main.rs:314-316."""
    return f"{(m if math.isfinite(m) else 0.0) * 1000.0:.3f}"


def fmt_mpa(pa: float) -> str:
    """main.rs:318-320."""
    return f"{(pa if math.isfinite(pa) else 0.0) / 1e6:.3f}"


def max_disp(displacements) -> float:
    """run_summary's max |u| over nodes (main.rs:386-391)."""
    d = np.asarray(displacements).reshape(-1, 3)
    best = 0.0
    for row in d:
        v = math.sqrt(row[0] * row[0] + row[1] * row[1] + row[2] * row[2])
        best = max(best, v)
    return best


def model_from_json(m: dict) -> Model:
    mesh = Mesh([Node(i, tuple(c)) for i, c in m["nodes"]],
                [Element(i, ElemKind(k), conn) for i, k, conn in m["elements"]])
    return Model(
        mesh=mesh,
        thickness=m["thickness"],
        materials=[Material(x["name"], x["E"], x["nu"]) for x in m["materials"]],
        elsets=[ElementSet(s["name"], s["element_ids"]) for s in m["elsets"]],
        mat_assignments=[tuple(a) for a in m["mat_assignments"]],
        boundary_conditions=[BoundaryCondition(b["node_ids"], b["dofs"])
                             for b in m["boundary_conditions"]],
        cloads=[ConcentratedLoad(c["node_id"], c["dof"], c["value"]) for c in m["cloads"]],
    )


def load_golden(name: str):
    with open(os.path.join(GOLDEN_DIR, f"{name}.json")) as fh:
        d = json.load(fh)
    return model_from_json(d["model"]), d["golden"]


def _six(x: float) -> float:
    return float(f"{x:.6f}")


def cantilever_deck(nx: int, ny: int, length=2.0, height=0.1, thickness=0.01,
                    total=1000.0) -> Model:
    """Row-major CPS4 cantilever of the bench / refinement decks: left edge
    clamped (dofs 1-2), the tip nodes share the downward load, each value
    written with three decimals (-200.0 on 4-row meshes, -111.111 on 8-row)."""
    wx, wy = length / nx, height / ny

    def nid(i, j):
        return j * (nx + 1) + i + 1

    nodes = [Node(nid(i, j), (_six(i * wx), _six(j * wy), 0.0))
             for j in range(ny + 1) for i in range(nx + 1)]
    elems = [Element(j * nx + i + 1, ElemKind.Cps4,
                     [nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)])
             for j in range(ny) for i in range(nx)]
    fix = [nid(0, j) for j in range(ny + 1)]
    tip = [nid(nx, j) for j in range(ny + 1)]
    load = float(f"{-total / (ny + 1):.3f}")
    return Model(
        mesh=Mesh(nodes, elems), thickness=thickness,
        materials=[Material("STEEL", E_STEEL, NU_STEEL)],
        elsets=[ElementSet("ALL", list(range(1, nx * ny + 1)))],
        mat_assignments=[("ALL", "STEEL")],
        boundary_conditions=[BoundaryCondition(fix, [1, 2])],
        cloads=[ConcentratedLoad(t, 2, load) for t in tip],
    )


def patch_deck() -> Model:
    """The 9-node distorted CPS4 patch of the bench (bench.rs:742-784)."""
    pts = [(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0), (0.5, 0.0), (1.0, 0.5),
           (0.5, 1.0), (0.0, 0.5), (0.35, 0.55)]
    conn = [[1, 5, 9, 8], [5, 2, 6, 9], [9, 6, 3, 7], [8, 9, 7, 4]]
    return Model(
        mesh=Mesh([Node(k + 1, (_six(x), _six(y), 0.0)) for k, (x, y) in enumerate(pts)],
                  [Element(k + 1, ElemKind.Cps4, c) for k, c in enumerate(conn)]),
        thickness=0.01,
        materials=[Material("STEEL", E_STEEL, NU_STEEL)],
        elsets=[ElementSet("ALL", [1, 2, 3, 4])],
        mat_assignments=[("ALL", "STEEL")],
        boundary_conditions=[BoundaryCondition([1], [1]), BoundaryCondition([8], [1]),
                             BoundaryCondition([4], [1]), BoundaryCondition([1], [2])],
        cloads=[ConcentratedLoad(2, 1, 2500.0), ConcentratedLoad(6, 1, 5000.0),
                ConcentratedLoad(3, 1, 2500.0)],
    )


def quad_mesh(nx, ny, width, height) -> Mesh:
    """Structured quad mesh, row-major ids from 1 (assembly.rs:554-580)."""
    nodes = [Node(j * (nx + 1) + i + 1, (width * i / nx, height * j / ny, 0.0))
             for j in range(ny + 1) for i in range(nx + 1)]

    def nid(i, j):
        return j * (nx + 1) + i + 1

    elems = [Element(j * nx + i + 1, ElemKind.Cps4,
                     [nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)])
             for j in range(ny) for i in range(nx)]
    return Mesh(nodes, elems)


def hex_mesh(nx, ny, nz, lx, ly, lz) -> Mesh:
    """Structured hex mesh, k-major ids from 1, bottom face CCW then top
    (assembly.rs:584-624)."""
    def nid(i, j, k):
        return k * (ny + 1) * (nx + 1) + j * (nx + 1) + i + 1

    nodes = [Node(nid(i, j, k), (lx * i / nx, ly * j / ny, lz * k / nz))
             for k in range(nz + 1) for j in range(ny + 1) for i in range(nx + 1)]
    elems = [Element(k * nx * ny + j * nx + i + 1, ElemKind.C3d8,
                     [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                      nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1),
                      nid(i, j + 1, k + 1)])
             for k in range(nz) for j in range(ny) for i in range(nx)]
    return Mesh(nodes, elems)


def steel_model(mesh: Mesh, thickness=1.0) -> Model:
    """quad_model / solid_model of lib.rs:804-832 (steel, E=210e9, nu=0.3)."""
    return Model(mesh=mesh, thickness=thickness,
                 materials=[Material("steel", E_STEEL, NU_STEEL)],
                 elsets=[ElementSet("all", mesh.elem_ids.tolist())],
                 mat_assignments=[("all", "steel")])


def hex_cantilever(nx, ny, nz) -> Model:
    """solver.rs:161-180: hex beam 2 x 0.1 x 0.1 clamped at x = 0, tip load
    -10 kN in y at the middle of the x = L face."""
    m = steel_model(hex_mesh(nx, ny, nz, 2.0, 0.1, 0.1))
    root = [k * (ny + 1) * (nx + 1) + j * (nx + 1) + 1
            for k in range(nz + 1) for j in range(ny + 1)]
    m.boundary_conditions.append(BoundaryCondition(root, [1, 2, 3]))
    tip = (nz // 2) * (ny + 1) * (nx + 1) + (ny // 2) * (nx + 1) + nx + 1
    m.cloads = [ConcentratedLoad(tip, 2, -10000.0)]
    return m


# Published refinement table (README.md:149-155; docs/benchmarks/cantilever.md:13-17).
REFINEMENT = [
    (10, 4, 201, "5.985"),
    (20, 4, 315, "10.953"),
    (40, 4, 390, "13.832"),
    (80, 8, 838, "14.877"),
    (160, 8, 943, "15.147"),
]
