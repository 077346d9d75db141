"""The oracle against the reference's own golden values and known-answer
tests (CPU only).

Goldens: the stable QA values the reference publishes for its example decks
and bench decks (see tests/golden/make_golden.py for the sources) and the
refinement table of README.md:149-155.  Known-answer tests restate
element.rs:1060-1398, assembly.rs:742-790 and the patch tests of
lib.rs:909-1084.
"""
import math

import numpy as np
import pytest

from oracle import oracle
from solvix_b200.model import (BoundaryCondition, ConcentratedLoad, ElemKind, Element,
                               ElementSet, InvalidModel, Material, Mesh, Model, Node,
                               NoConstraints, NotConverged)
from svx_cases import (E_STEEL, NU_STEEL, REFINEMENT, cantilever_deck, fmt_e3, fmt_mm,
                       fmt_mpa, hex_mesh, load_golden, max_disp, patch_deck, quad_mesh,
                       steel_model)


@pytest.mark.parametrize("name", ["cantilever", "cantilever3d", "plate_hole"])
def test_example_decks_reproduce_published_values(name):
    model, g = load_golden(name)
    sol, flat = oracle.solve(model)
    assert flat.n_nodes == g["nodes"] and flat.n_elem == g["elements"]
    assert sol.iterations == g["iterations"]
    assert fmt_e3(sol.final_residual) == g["residual"]
    assert fmt_mm(max_disp(sol.displacements)) == g["max_disp_mm"]
    assert fmt_mpa(max(0.0, sol.von_mises.max())) == g["max_von_mises_mpa"]
    if "max_nodal_von_mises_mpa" in g:
        assert fmt_mpa(sol.nodal_von_mises.max()) == g["max_nodal_von_mises_mpa"]


@pytest.mark.parametrize("nx,ny,iters,mm", REFINEMENT)
def test_refinement_table(nx, ny, iters, mm):
    sol, _ = oracle.solve(cantilever_deck(nx, ny))
    assert sol.iterations == iters
    assert fmt_mm(max_disp(sol.displacements)) == mm


def test_v01_gate_80x8_deck():
    """docs/qa/v0.1.0-gate.md:160: tip load -111.11111111 N x 9 nodes."""
    m = cantilever_deck(80, 8)
    m.cloads = [ConcentratedLoad(c.node_id, 2, -111.11111111) for c in m.cloads]
    sol, _ = oracle.solve(m)
    assert sol.iterations == 867
    assert fmt_e3(sol.final_residual) == "8.422e-11"
    assert fmt_mpa(sol.von_mises.max()) == "100.344"


def test_patch_cps4_bench_case():
    """docs/qa/v0.2.0-gate.md:51: 14 iterations, 1.000 MPa."""
    sol, _ = oracle.solve(patch_deck())
    assert sol.iterations == 14
    assert fmt_mpa(sol.von_mises.max()) == "1.000"


def _ke(kind, coords, E=1.0, nu=0.25, t=1.0):
    r, ke = oracle.element_stiffness(kind, coords, E, nu, t)
    assert r == 0
    return ke


def test_cps4_stiffness_symmetric_kills_rigid_translation():
    """element.rs:1081-1099."""
    coords = [(0.0, 0.0, 0.0), (2.0, 0.0, 0.0), (2.2, 1.0, 0.0), (0.1, 1.1, 0.0)]
    ke = _ke(1, coords)
    assert np.array_equal(ke, ke.T)  # bitwise mirror (btdb)
    for d in ([1.0, 0.0], [0.0, 1.0]):
        assert np.abs(ke @ np.tile(d, 4)).max() < 1e-12 * np.abs(ke).max()


def test_c3d8_stiffness_symmetric_kills_rigid_translation():
    """element.rs:1135-1157."""
    rng = np.random.default_rng(0)
    base = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                     [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float) * 0.5
    coords = base + rng.uniform(-0.05, 0.05, base.shape)
    ke = _ke(5, coords)
    assert np.array_equal(ke, ke.T)
    for d in np.eye(3):
        assert np.abs(ke @ np.tile(d, 8)).max() < 1e-12 * np.abs(ke).max()
    w = np.linalg.eigvalsh(ke)
    assert (w > -1e-12 * w.max()).all()


def test_c3d8_inverse_jacobian_follows_the_reference():
    """element.rs:446-462 multiplies the cyclic cofactor (which already
    carries its sign) by (-1)^(r+c) again, so J^-1 is exact only when the
    odd off-diagonal cofactors vanish.  For an axis-aligned box rigid
    rotations are zero-energy; for a distorted hex they are not.  The
    oracle (and the CUDA kernels) reproduce the reference's matrix."""
    box = np.array([[0, 0, 0], [2, 0, 0], [2, 1, 0], [0, 1, 0],
                    [0, 0, 1], [2, 0, 1], [2, 1, 1], [0, 1, 1]], float)
    ke = _ke(5, box)
    for w in np.eye(3):
        rot = np.cross(w, box).ravel()
        assert np.abs(ke @ rot).max() < 1e-12 * np.abs(ke).max()
    skew = box + np.random.default_rng(0).uniform(-0.05, 0.05, box.shape)
    ke = _ke(5, skew)
    assert np.abs(ke @ np.cross([0.0, 0.0, 1.0], skew).ravel()).max() > 1e-3 * np.abs(ke).max()


def test_cps3_stiffness_either_orientation():
    """element.rs:1060-1079: CST works for both node orderings."""
    a = _ke(0, [(0, 0, 0), (1, 0, 0), (0, 1, 0)])
    b = _ke(0, [(0, 0, 0), (0, 1, 0), (1, 0, 0)])
    perm = [0, 1, 4, 5, 2, 3]
    assert np.allclose(a, b[np.ix_(perm, perm)], rtol=0, atol=1e-15)


def test_inverted_and_degenerate_elements_are_rejected():
    """element.rs:1120-1133, :1211-1217."""
    inv_quad = [(0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0)]  # clockwise
    r, _ = oracle.element_stiffness(1, inv_quad, 1.0, 0.25, 1.0)
    assert r == 5
    r, _ = oracle.element_stiffness(0, [(0, 0, 0), (1, 1, 0), (2, 2, 0)], 1.0, 0.25, 1.0)
    assert r == 4
    hex_ = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                     [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    r, _ = oracle.element_stiffness(5, hex_[[4, 5, 6, 7, 0, 1, 2, 3]], 1.0, 0.25, 1.0)
    assert r == 5


def test_free_free_assembly_symmetric_and_translation_free():
    """assembly.rs:742-767."""
    for mesh, ndof, d in ((quad_mesh(2, 2, 1.0, 1.0), 2, [1.0, 0.5]),
                          (hex_mesh(2, 2, 2, 1.0, 1.0, 1.0), 3, [1.0, 0.5, -0.25])):
        m = Model(mesh=mesh, materials=[Material("mat", 1.0, 0.25)],
                  elsets=[ElementSet("all", mesh.elem_ids.tolist())],
                  mat_assignments=[("all", "mat")],
                  boundary_conditions=[BoundaryCondition([1], [1, 2])])
        flat, _ = oracle.resolve(m)
        k = oracle.assemble(flat)
        a = k.to_scipy()
        assert abs(a - a.T).max() < 1e-12
        u = np.tile(d, mesh.n_nodes)
        assert np.abs(oracle.spmv(k, u)).max() < 1e-10


def test_threaded_assembly_and_spmv_are_bit_identical():
    """assembly.rs:769-812."""
    m = steel_model(hex_mesh(12, 12, 12, 1.0, 1.0, 1.0))
    m.boundary_conditions = [BoundaryCondition([1], [1, 2, 3])]
    flat, _ = oracle.resolve(m)
    k1 = oracle.assemble(flat, threads=1)
    k8 = oracle.assemble(flat, threads=8)
    assert np.array_equal(k1.row_ptr, k8.row_ptr) and np.array_equal(k1.col_idx, k8.col_idx)
    assert np.array_equal(k1.vals.view(np.int64), k8.vals.view(np.int64))
    big = steel_model(hex_mesh(40, 12, 12, 2.0, 0.1, 0.1))
    big.boundary_conditions = [BoundaryCondition([1], [1, 2, 3])]
    flat, _ = oracle.resolve(big)
    k = oracle.assemble(flat)
    assert k.n > 20000
    s = 0x853C49E6748FEA9B
    u = np.empty(k.n)
    for i in range(k.n):
        s = (s * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
        u[i] = (s >> 11) / float(1 << 53) - 0.5
    a = oracle.spmv(k, u, threads=1)
    b = oracle.spmv(k, u, threads=8)
    assert np.array_equal(a.view(np.int64), b.view(np.int64))


def _fix_left_edge_x(m, nx, ny):
    ids = [j * (nx + 1) + 1 for j in range(ny + 1)]
    m.boundary_conditions += [BoundaryCondition(ids, [1]), BoundaryCondition([1], [2])]


def test_cps4_patch_single_quad():
    """lib.rs:909-950."""
    m = steel_model(quad_mesh(1, 1, 1.0, 1.0))
    _fix_left_edge_x(m, 1, 1)
    sigma = 1e6
    m.cloads = [ConcentratedLoad(2, 1, sigma / 2), ConcentratedLoad(4, 1, sigma / 2)]
    sol, flat = oracle.solve(m)
    assert abs(sol.von_mises[0] - sigma) / sigma < 1e-6
    assert np.all(np.abs(sol.nodal_von_mises - sigma) / sigma < 1e-6)
    ux = sigma / E_STEEL
    assert abs(sol.displacements[1][0] - ux) / ux < 1e-6
    rx = sum(v for r, v in zip(flat.fixed_row, sol.reaction_values) if r % 2 == 0)
    assert abs(rx + sigma) < 1e-6 * sigma
    assert sol.final_residual <= 1e-10


def test_cps3_patch_two_triangles():
    """lib.rs:1011-1084."""
    mesh = Mesh([Node(1, (0, 0, 0)), Node(2, (1, 0, 0)), Node(3, (1, 1, 0)), Node(4, (0, 1, 0))],
                [Element(1, ElemKind.Cps3, [1, 2, 3]), Element(2, ElemKind.Cps3, [1, 3, 4])])
    m = steel_model(mesh)
    m.boundary_conditions = [BoundaryCondition([1, 4], [1]), BoundaryCondition([1], [2])]
    m.cloads = [ConcentratedLoad(2, 1, 5e5), ConcentratedLoad(3, 1, 5e5)]
    sol, _ = oracle.solve(m)
    sigma = 1e6
    assert np.all(np.abs(sol.von_mises - sigma) / sigma < 1e-6)
    assert np.all(np.abs(sol.nodal_von_mises - sigma) / sigma < 1e-6)
    assert abs(sol.displacements[2][1] - (-NU_STEEL * sigma / E_STEEL)) / \
        (NU_STEEL * sigma / E_STEEL) < 1e-6


def test_c3d8_cube_tension_patch():
    """lib.rs:1721-1807: uniform sigma_z on a unit cube."""
    m = steel_model(hex_mesh(1, 1, 1, 1.0, 1.0, 1.0))
    m.boundary_conditions = [BoundaryCondition([1, 2, 3, 4], [3]), BoundaryCondition([1], [1]),
                             BoundaryCondition([1, 2], [2])]
    sigma = 1e6
    m.cloads = [ConcentratedLoad(n, 3, sigma / 4) for n in (5, 6, 7, 8)]
    sol, flat = oracle.solve(m)
    assert np.all(np.abs(sol.von_mises - sigma) / sigma < 1e-6)
    assert np.all(np.abs(sol.nodal_von_mises - sigma) / sigma < 1e-6)
    w = sigma / E_STEEL
    for i in (4, 5, 6, 7):
        assert abs(sol.displacements[i][2] - w) / w < 1e-6
    rz = sum(v for r, v in zip(flat.fixed_row, sol.reaction_values) if r % 3 == 2)
    assert abs(rz + sigma) < 1e-6 * sigma


def test_extrapolation_exact_for_bilinear_field():
    """element.rs:1101-1118: a linear displacement field gives constant
    stress; every nodal value equals the centroid value."""
    m = steel_model(quad_mesh(3, 2, 1.5, 1.0))
    m.boundary_conditions = [BoundaryCondition([1], [1, 2])]
    flat, _ = oracle.resolve(m)
    xy = flat.xyz[:, :2]
    u = np.stack([1e-4 * xy[:, 0] + 2e-5 * xy[:, 1], -3e-5 * xy[:, 0] + 5e-5 * xy[:, 1]],
                 axis=1).ravel()
    vm, vmn, _ = oracle.stress(flat, u)
    assert np.allclose(vm, vm[0], rtol=1e-12) and np.allclose(vmn, vm[0], rtol=1e-12)


def test_reference_error_order_and_texts():
    """lib.rs:596-612, validate (lib.rs:406-436), assembly.rs:143-160."""
    m = steel_model(quad_mesh(2, 1, 2.0, 1.0))
    with pytest.raises(NoConstraints):
        oracle.solve(m)
    m.boundary_conditions = [BoundaryCondition([1, 4], [1, 2])]
    m.cloads = [ConcentratedLoad(3, 2, -1.0)]
    bad = steel_model(quad_mesh(2, 1, 2.0, 1.0))
    bad.boundary_conditions = m.boundary_conditions
    bad.mat_assignments = []
    with pytest.raises(InvalidModel, match=r"^element 1: no material assigned$"):
        oracle.solve(bad)
    bad = steel_model(quad_mesh(2, 1, 2.0, 1.0))
    bad.boundary_conditions = m.boundary_conditions
    bad.cloads = [ConcentratedLoad(99, 1, 1.0)]
    with pytest.raises(InvalidModel, match=r"^load on unknown node 99$"):
        oracle.solve(bad)
    bad.cloads = [ConcentratedLoad(3, 3, 1.0)]
    with pytest.raises(InvalidModel, match=r"^load on node 3 has unsupported dof 3$"):
        oracle.solve(bad)
    bad.cloads = m.cloads
    bad.boundary_conditions = [BoundaryCondition([77], [1])]
    with pytest.raises(InvalidModel, match=r"^boundary condition on unknown node 77$"):
        oracle.solve(bad)
    # an element error beats a load error raised later
    bad.boundary_conditions = m.boundary_conditions
    bad.cloads = [ConcentratedLoad(99, 1, 1.0)]
    bad.materials = [Material("steel", -1.0, 0.3)]
    with pytest.raises(InvalidModel, match=r"^element 1: invalid material constants$"):
        oracle.solve(bad)


def test_budget_exhaustion_is_not_converged():
    m = cantilever_deck(20, 4)
    flat, _ = oracle.resolve(m)
    with pytest.raises(NotConverged) as ei:
        oracle.solve_flat(flat, max_iter=5)
    assert ei.value.iterations == 5 and ei.value.residual > 1e-10


def test_cond_estimate_uses_modified_diagonal():
    """lib.rs:634-644: constrained rows carry diag 1, so min |diag| is 1."""
    model, _ = load_golden("cantilever")
    sol, flat = oracle.solve(model)
    k = oracle.assemble(flat)
    d = k.vals[[np.nonzero(k.col_idx[k.row_ptr[i]:k.row_ptr[i + 1]] == i)[0][0] + k.row_ptr[i]
                for i in range(k.n)]]
    free = np.ones(k.n, bool)
    free[flat.fixed_row] = False
    hi = max(np.abs(d[free]).max(), 1.0)
    assert math.isclose(sol.cond_estimate, hi / 1.0, rel_tol=0, abs_tol=0)
