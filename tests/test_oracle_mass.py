"""The oracle's consistent mass operator (CPU only): element mass matrices
and assemble_mass restated from modal.rs:82-146, 203-271, pinned by the
reference's consistent_mass_totals_match_rho_times_volume
(modal.rs:939-995) and by properties of the assembled matrix: the
stiffness's pattern (the same dof map and triplet construction), the total
mass of a mesh per direction, positive definiteness, the reference's error
texts."""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200.model import (BoundaryCondition, ElemKind, Element, InvalidModel, Mesh,
                               Node)
from svx_cases import hex_mesh, quad_mesh, steel_model

RHO, T = 7850.0, 0.01


def test_consistent_mass_totals_match_rho_times_volume():
    """modal.rs:939-995 for the kinds on this path."""
    _, tri = oracle.element_mass(ElemKind.Cps3, [[0, 0, 0], [1, 0, 0], [0, 1, 0]], RHO, T)
    _, quad = oracle.element_mass(ElemKind.Cps4, [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]],
                                  RHO, T)
    cube = [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1],
            [0, 1, 1]]
    _, hexm = oracle.element_mass(ElemKind.C3d8, cube, RHO, 1.0)
    eps = 1e-9 * RHO
    assert abs(tri[0::2, 0::2].sum() - RHO * T * 0.5) < eps
    assert abs(quad[0::2, 0::2].sum() - RHO * T) < eps
    assert abs(hexm[0::3, 0::3].sum() - RHO) < eps


def test_cps3_closed_form_and_cpe4_equals_cps4():
    _, tri = oracle.element_mass(ElemKind.Cps3, [[0, 0, 0], [2, 0, 0], [0, 1, 0]], RHO, T)
    w = RHO * T * 1.0 / 12.0
    want = np.zeros((6, 6))
    for i in range(3):
        for j in range(3):
            for d in range(2):
                want[2 * i + d, 2 * j + d] = w * (2.0 if i == j else 1.0)
    assert np.array_equal(tri, want)
    xy = [[0, 0, 0], [1.2, 0.1, 0], [1.0, 0.9, 0], [-0.1, 1.1, 0]]
    _, a = oracle.element_mass(ElemKind.Cps4, xy, RHO, T)
    _, b = oracle.element_mass(ElemKind.Cpe4, xy, RHO, T)
    assert np.array_equal(a, b)
    assert np.allclose(a, a.T, rtol=1e-15, atol=0.0)


def test_element_failures_are_the_stiffness_triggers():
    r, _ = oracle.element_mass(ElemKind.Cps3, [[0, 0, 0], [1, 0, 0], [2, 0, 0]], RHO, T)
    assert r != 0
    r, _ = oracle.element_mass(ElemKind.Cps4, [[0, 0, 0], [0, 1, 0], [1, 1, 0], [1, 0, 0]],
                               RHO, T)
    assert r != 0


@pytest.mark.parametrize("case", ["quad", "hex", "mixed_tri_quad"])
def test_assembled_mass_shares_the_stiffness_pattern_and_totals(case):
    if case == "quad":
        mesh, area_or_vol, t = quad_mesh(6, 3, 2.0, 0.5), 2.0 * 0.5, T
    elif case == "hex":
        mesh, area_or_vol, t = hex_mesh(5, 2, 3, 1.0, 0.2, 0.3), 1.0 * 0.2 * 0.3, 1.0
    else:
        q = quad_mesh(4, 2, 1.0, 1.0)
        conn = q.conn.reshape(-1, 4)
        elems = []
        for e, c in enumerate(conn.tolist()):
            if e % 2:
                elems.append(Element(100 + 2 * e, ElemKind.Cps3, [c[0], c[1], c[2]]))
                elems.append(Element(101 + 2 * e, ElemKind.Cps3, [c[0], c[2], c[3]]))
            else:
                elems.append(Element(100 + 2 * e, ElemKind.Cps4, c))
        mesh = Mesh([Node(i, tuple(x)) for i, x in zip(q.node_ids.tolist(), q.coords)], elems)
        area_or_vol, t = 1.0, T
    m = steel_model(mesh, thickness=t)
    m.boundary_conditions = [BoundaryCondition([1], [1, 2])]
    flat, _ = oracle.resolve(m)
    k = oracle.assemble(flat, threads=1)
    mm = oracle.assemble_mass(flat, RHO)
    assert np.array_equal(mm.row_ptr, k.row_ptr) and np.array_equal(mm.col_idx, k.col_idx)
    dense = mm.to_scipy().toarray()
    nd = flat.ndof
    total = RHO * area_or_vol * (t if nd == 2 else 1.0)
    for d in range(nd):
        assert abs(dense[d::nd, d::nd].sum() - total) < 1e-10 * total
        # no coupling between directions
        for e in range(nd):
            if e != d:
                assert not np.any(dense[d::nd, e::nd])
    assert np.allclose(dense, dense.T, rtol=1e-14, atol=0.0)
    assert np.linalg.eigvalsh(dense).min() > 0.0


def test_assembly_error_text():
    mesh = Mesh([Node(1, (0, 0, 0)), Node(2, (1, 0, 0)), Node(3, (2, 0, 0))],
                [Element(9, ElemKind.Cps3, [1, 2, 3])])
    m = steel_model(mesh)
    m.boundary_conditions = [BoundaryCondition([1], [1, 2])]
    flat, _ = oracle.resolve(m)
    with pytest.raises(InvalidModel, match=r"^element 9: degenerate \(zero-area\) triangle$"):
        oracle.assemble_mass(flat, RHO)


def _quad_n(xi, eta):
    s = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], dtype=float)
    n = 0.25 * (1 + xi * s[:, 0]) * (1 + eta * s[:, 1])
    dn = 0.25 * np.stack([s[:, 0] * (1 + eta * s[:, 1]), s[:, 1] * (1 + xi * s[:, 0])])
    return n, dn


def _hex_n(xi, eta, zeta):
    s = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=float)
    a, b, c = 1 + xi * s[:, 0], 1 + eta * s[:, 1], 1 + zeta * s[:, 2]
    n = 0.125 * a * b * c
    dn = 0.125 * np.stack([s[:, 0] * b * c, s[:, 1] * a * c, s[:, 2] * a * b])
    return n, dn


@pytest.mark.parametrize("seed", range(4))
def test_element_mass_matches_an_independent_gauss_integration(seed):
    """rho [t] sum_gp detJ N^T N on randomly distorted elements, computed
    here with numpy, against the oracle's element mass."""
    rng = np.random.Generator(np.random.PCG64(40 + seed))
    g = 1.0 / np.sqrt(3.0)
    quad = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float) + rng.uniform(-0.2, 0.2, (4, 2))
    want = np.zeros((8, 8))
    for xi in (-g, g):
        for eta in (-g, g):
            n, dn = _quad_n(xi, eta)
            detj = np.linalg.det(dn @ quad)
            block = RHO * T * detj * np.outer(n, n)
            want[0::2, 0::2] += block
            want[1::2, 1::2] += block
    _, got = oracle.element_mass(ElemKind.Cps4, np.c_[quad, np.zeros(4)], RHO, T)
    assert np.allclose(got, want, rtol=1e-13, atol=1e-13 * np.abs(want).max())
    hexc = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1],
                     [1, 1, 1], [0, 1, 1]], float) + rng.uniform(-0.15, 0.15, (8, 3))
    want = np.zeros((24, 24))
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                n, dn = _hex_n(xi, eta, zeta)
                detj = np.linalg.det(dn @ hexc)
                block = RHO * detj * np.outer(n, n)
                for d in range(3):
                    want[d::3, d::3] += block
    _, got = oracle.element_mass(ElemKind.C3d8, hexc, RHO, 1.0)
    assert np.allclose(got, want, rtol=1e-13, atol=1e-13 * np.abs(want).max())
