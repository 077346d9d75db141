"""Edge pressure (*DLOAD Pn) and gravity (*DLOAD GRAV) through the public
solve() on the device, restating the reference's known-answer tests
(crates/solvix-core/src/lib.rs:1630-1719): a pressure equals its
consistent nodal forces and reproduces a uniform stress patch, and the base
reactions of a column under its own weight sum to the weight."""
import copy

import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import Method, solve, solve_with_method
from solvix_b200.model import BoundaryCondition, ConcentratedLoad, DistributedLoad, Step
from svx_cases import quad_mesh, steel_model

pytestmark = pytest.mark.gpu

BOTH_METHODS = (Method.Auto, Method.Ldlt)  # lib.rs:907


def quad_model(nx, ny, width, height):
    """lib.rs:804-817 (steel, thickness 1)."""
    return steel_model(quad_mesh(nx, ny, width, height))


def fix_left_edge_x(m, nx, ny):
    """lib.rs:890-903: ux on the left edge, uy pinned at node 1 only."""
    m.boundary_conditions.append(BoundaryCondition([j * (nx + 1) + 1 for j in range(ny + 1)],
                                                   [1]))
    m.boundary_conditions.append(BoundaryCondition([1], [2]))


def test_edge_pressure_matches_equivalent_cload(ctx):
    # lib.rs:1630-1683
    m = quad_model(1, 1, 1.0, 1.0)
    fix_left_edge_x(m, 1, 1)
    p = 1.0e6
    pressurized = copy.deepcopy(m)
    pressurized.steps = [Step(boundary_conditions=list(m.boundary_conditions),
                              dloads=[DistributedLoad(1, 2, p)])]
    m.cloads = [ConcentratedLoad(2, 1, -p / 2.0), ConcentratedLoad(4, 1, -p / 2.0)]
    a = solve(pressurized, ctx=ctx)
    b = solve(m, ctx=ctx)
    assert np.max(np.abs(a.displacements - b.displacements)) < 1e-9
    for method in BOTH_METHODS:
        sol = solve_with_method(pressurized, method, ctx=ctx)
        assert abs(sol.von_mises[0] - p) / p < 1e-6
        rx = sum(r.value for r in sol.reactions if r.dof == 1)
        assert abs(rx - p) < 1e-6 * p


def test_gravity_column_base_reactions_balance_weight(ctx):
    # lib.rs:1685-1719
    w, length, t = 0.1, 1.0, 0.01
    m = quad_model(1, 8, w, length)
    m.thickness = t
    m.steps = [Step(boundary_conditions=[BoundaryCondition([1, 2], [2]),
                                         BoundaryCondition([1], [1])],
                    gravity=(9.81, (0.0, -1.0, 0.0)))]
    sol = solve(m, ctx=ctx)
    ry = sum(r.value for r in sol.reactions if r.dof == 2)
    expect = 7850.0 * w * t * length * 9.81
    assert abs(ry - expect) < 1e-9 * expect


def test_pressure_and_gravity_plate_matches_oracle(ctx):
    """A jittered CPS4 plate under pressures on its top and right edges and
    a slanted gravity: the device solve against the oracle's, at the plain
    form's bar."""
    m = quad_model(12, 4, 3.0, 1.0)
    m.thickness = 0.02
    m.density = 2700.0
    rng = np.random.default_rng(3)
    ids = m.mesh.node_ids.astype(np.int64) - 1
    inner = ((ids % 13) > 0) & ((ids % 13) < 12) & ((ids // 13) > 0) & ((ids // 13) < 4)
    m.mesh.coords[inner, :2] += rng.uniform(-0.05, 0.05, size=(int(inner.sum()), 2))
    m.steps = [Step(boundary_conditions=[BoundaryCondition([1 + 13 * j for j in range(5)],
                                                           [1, 2])],
                    cloads=[ConcentratedLoad(65, 2, -50.0)],
                    dloads=[DistributedLoad(e, 3, 2.0e5) for e in range(37, 49)] +
                           [DistributedLoad(12, 2, -1.0e5), DistributedLoad(24, 2, -1.0e5)],
                    gravity=(9.81, (0.2, -1.0, 0.0)))]
    sol = solve(m, ctx=ctx)
    ref, _ = oracle.solve(m)
    assert np.linalg.norm(sol.u - ref.u) / np.linalg.norm(ref.u) <= 1e-10
    assert np.max(np.abs(sol.von_mises - ref.von_mises)) <= 1e-8 * np.max(ref.von_mises)
