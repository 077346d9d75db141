"""The oracle's restatement of steady heat conduction (heat.rs:52-98),
pinned by the reference's own known-answer tests of that module
(crates/solvix-core/src/heat.rs:529-645, 756-780) and by element-level
identities.  CPU only; this is the checker a conduction operator on the
device will be measured against."""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200.model import ElemKind, InvalidModel, NoConstraints
from svx_cases import hex_mesh, quad_mesh


def thermal_from_mesh(mesh, conductivity, **kw):
    index = {n.id: i for i, n in enumerate(mesh.nodes)}
    xyz = np.array([n.coords for n in mesh.nodes], dtype=np.float64)
    kind = [int(e.kind) for e in mesh.elements]
    conn_ptr = np.zeros(len(mesh.elements) + 1, dtype=np.int64)
    conn_ptr[1:] = np.cumsum([len(e.connectivity) for e in mesh.elements])
    conn = [index[c] for e in mesh.elements for c in e.connectivity]
    return oracle.ThermalModel(xyz, kind, conn_ptr, conn, conductivity,
                               elem_id=[e.id for e in mesh.elements], **kw)


def temps(pairs):
    """[(node indices, temperature), ...] -> the flat constraint arrays."""
    nodes = [i for ids, _ in pairs for i in ids]
    vals = [t for ids, t in pairs for _ in ids]
    return nodes, vals


def test_bar_fixed_temps_linear_gradient_exact():
    # heat.rs:529-558: 8x1 strip 1.0 x 0.1, k = 1, T = 100 left, 0 right
    nx, ny = 8, 1
    mesh = quad_mesh(nx, ny, 1.0, 0.1)
    left = [j * (nx + 1) for j in range(ny + 1)]
    right = [j * (nx + 1) + nx for j in range(ny + 1)]
    tn, tv = temps([(left, 100.0), (right, 0.0)])
    tm = thermal_from_mesh(mesh, 1.0, temp_node=tn, temp_value=tv)
    t, it, res = oracle.solve_thermal(tm)
    assert res <= 1e-10 and it > 0
    exact = 100.0 * (1.0 - tm.xyz[:, 0])
    assert np.max(np.abs(t - exact)) < 1e-8


def test_hex_bar_fixed_temps_linear_gradient_exact():
    # heat.rs:560-593: 6x1x1 hexes over 1.0 x 0.1 x 0.1, k = 5, 20 / 120
    nx, ny, nz = 6, 1, 1
    mesh = hex_mesh(nx, ny, nz, 1.0, 0.1, 0.1)

    def nid(i, j, k):
        return k * (ny + 1) * (nx + 1) + j * (nx + 1) + i

    cold = [nid(0, j, k) for k in range(nz + 1) for j in range(ny + 1)]
    hot = [nid(nx, j, k) for k in range(nz + 1) for j in range(ny + 1)]
    tn, tv = temps([(cold, 20.0), (hot, 120.0)])
    tm = thermal_from_mesh(mesh, 5.0, temp_node=tn, temp_value=tv)
    t, _, _ = oracle.solve_thermal(tm)
    assert np.max(np.abs(t - (20.0 + 100.0 * tm.xyz[:, 0]))) < 1e-8


def test_surface_flux_matches_equivalent_dirichlet():
    # heat.rs:595-645: flux q into the right edge of a k = 2 bar equals
    # T_right = q L / k; both give T(x) = q x / k with T(0) = 0
    nx, ny = 6, 1
    k, q = 2.0, 50.0
    mesh = quad_mesh(nx, ny, 1.0, 0.1)
    left = [j * (nx + 1) for j in range(ny + 1)]
    right = [j * (nx + 1) + nx for j in range(ny + 1)]
    tn, tv = temps([(left, 0.0)])
    fluxed = thermal_from_mesh(mesh, k, temp_node=tn, temp_value=tv,
                               flux_elem=[j * nx + nx - 1 for j in range(ny)],
                               flux_face=[2] * ny, flux_value=[q] * ny)
    tn2, tv2 = temps([(left, 0.0), (right, q / k)])
    fixed = thermal_from_mesh(mesh, k, temp_node=tn2, temp_value=tv2)
    ta, _, _ = oracle.solve_thermal(fluxed)
    tb, _, _ = oracle.solve_thermal(fixed)
    exact = q * fluxed.xyz[:, 0] / k
    assert np.max(np.abs(ta - exact)) < 1e-8 and np.max(np.abs(tb - exact)) < 1e-8


def test_triangles_reproduce_the_linear_gradient():
    # the CPS3 branch (heat.rs:163-182) on the same bar, each quad split
    nx, ny = 8, 2
    quads = quad_mesh(nx, ny, 1.0, 0.2)
    index = {n.id: i for i, n in enumerate(quads.nodes)}
    xyz = np.array([n.coords for n in quads.nodes])
    conn = []
    for e in quads.elements:
        a, b, c, d = (index[x] for x in e.connectivity)
        conn += [a, b, c, a, c, d]
    ne = 2 * len(quads.elements)
    left = [j * (nx + 1) for j in range(ny + 1)]
    right = [j * (nx + 1) + nx for j in range(ny + 1)]
    tn, tv = temps([(left, 100.0), (right, 0.0)])
    tm = oracle.ThermalModel(xyz, [int(ElemKind.Cps3)] * ne, np.arange(ne + 1) * 3, conn, 3.0,
                             temp_node=tn, temp_value=tv)
    t, _, res = oracle.solve_thermal(tm)
    assert res <= 1e-10
    assert np.max(np.abs(t - 100.0 * (1.0 - xyz[:, 0]))) < 1e-8


def test_uniform_source_is_nodally_exact_on_a_strip():
    # a uniform source q with T = 0 at both ends: T(x) = q x (L - x) / (2 k);
    # linear elements with the consistent load (heat.rs:194-203) are exact
    # at the nodes of this one-dimensional field
    nx, ny = 10, 1
    k, q, length = 4.0, 30.0, 2.0
    mesh = quad_mesh(nx, ny, length, 0.1)
    ends = [j * (nx + 1) for j in range(ny + 1)] + [j * (nx + 1) + nx for j in range(ny + 1)]
    tn, tv = temps([(ends, 0.0)])
    tm = thermal_from_mesh(mesh, k, temp_node=tn, temp_value=tv, source=q, thickness=0.5)
    t, _, _ = oracle.solve_thermal(tm)
    x = tm.xyz[:, 0]
    exact = q * x * (length - x) / (2.0 * k)
    assert np.max(np.abs(t - exact)) < 1e-8 * np.max(exact)


@pytest.mark.parametrize("kind,coords", [
    (ElemKind.Cps3, [[0.1, 0.0], [1.3, 0.2], [0.4, 0.9]]),
    (ElemKind.Cps4, [[0.0, 0.0], [1.1, 0.1], [1.3, 1.2], [-0.1, 0.9]]),
    (ElemKind.C3d8, [[0, 0, 0], [1.1, 0, 0.1], [1.2, 1, 0], [0, 1.1, 0], [0, 0.1, 1],
                     [1, 0, 1.2], [1.1, 1.1, 1], [0.1, 1, 1.1]]),
])
def test_conduction_matrix_symmetric_and_kills_constants(kind, coords):
    ke, fe = oracle.conduction_element(int(kind), coords, 2.5, thickness=0.3, source=7.0)
    assert np.allclose(ke, ke.T, rtol=0, atol=1e-14 * np.abs(ke).max())
    # a constant temperature carries no flux
    assert np.max(np.abs(ke.sum(axis=1))) < 1e-12 * np.abs(ke).max()
    assert np.all(np.diag(ke) > 0)
    # the consistent source load integrates q over the element
    assert fe.sum() > 0


def test_thermal_errors():
    # heat.rs:756-780 and the checks of heat.rs:52-79
    mesh = quad_mesh(2, 1, 1.0, 0.1)
    with pytest.raises(NoConstraints):
        oracle.solve_thermal(thermal_from_mesh(mesh, 1.0))
    tm = thermal_from_mesh(mesh, 0.0, temp_node=[0], temp_value=[1.0])
    with pytest.raises(InvalidModel, match="thickness and conductivity must be positive"):
        oracle.solve_thermal(tm)
    beams = oracle.ThermalModel([[0, 0, 0], [0.5, 0, 0], [1, 0, 0]], [int(ElemKind.B31)] * 2,
                                [0, 2, 4], [0, 1, 1, 2], 1.0, temp_node=[0], temp_value=[1.0])
    with pytest.raises(InvalidModel, match="conduction"):
        oracle.solve_thermal(beams)
    bad_face = thermal_from_mesh(mesh, 1.0, temp_node=[0], temp_value=[1.0], flux_elem=[0],
                                 flux_face=[5], flux_value=[1.0])
    with pytest.raises(InvalidModel, match=r"element 1 \(Cps4\) has no face 5"):
        oracle.solve_thermal(bad_face)
