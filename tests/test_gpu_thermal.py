"""Steady heat conduction on the device (svx_solve_thermal_flat) against
the oracle's restatement of heat::solve_thermal (heat.rs:52-98), and the
reference's known-answer cases of heat.rs:529-645 through the device path.

Bars: temperatures within 1e-10 relative of the oracle's (the assembled
values are summed in the same element order; the PCG's reductions differ
in order), exact linear profiles within 1e-8 like the reference's tests,
the same errors with the same texts."""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import abi
from solvix_b200.marshal import ThermalModel
from solvix_b200.model import ElemKind, EmptyMesh, InvalidModel, NoConstraints

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def grid2d(nx, ny, lx, ly, jitter=0.0, tris=False, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    xs, ys = np.meshgrid(np.linspace(0.0, lx, nx + 1), np.linspace(0.0, ly, ny + 1))
    xyz = np.zeros(((nx + 1) * (ny + 1), 3))
    xyz[:, 0] = xs.ravel()
    xyz[:, 1] = ys.ravel()
    inner = (xyz[:, 0] > 0) & (xyz[:, 0] < lx) & (xyz[:, 1] > 0) & (xyz[:, 1] < ly)
    h = min(lx / nx, ly / ny)
    xyz[inner, :2] += rng.uniform(-jitter, jitter, (int(inner.sum()), 2)) * h
    conn, kind = [], []
    for j in range(ny):
        for i in range(nx):
            a = j * (nx + 1) + i
            b, c, d = a + 1, a + nx + 2, a + nx + 1
            if tris:
                conn += [a, b, c, a, c, d]
                kind += [int(ElemKind.Cps3)] * 2
            else:
                conn += [a, b, c, d]
                kind += [int(ElemKind.Cps4)]
    nn = 3 if tris else 4
    return xyz, kind, np.arange(len(kind) + 1) * nn, conn


def hex_grid(nx, ny, nz, lx, ly, lz):
    def nid(i, j, k):
        return k * (ny + 1) * (nx + 1) + j * (nx + 1) + i
    xyz = np.array([(lx * i / nx, ly * j / ny, lz * k / nz) for k in range(nz + 1)
                    for j in range(ny + 1) for i in range(nx + 1)])
    conn = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                conn += [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                         nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1),
                         nid(i, j + 1, k + 1)]
    ne = nx * ny * nz
    return xyz, [int(ElemKind.C3d8)] * ne, np.arange(ne + 1) * 8, conn, nid


def plate_case(tris, seed):
    nx, ny = 24, 8
    xyz, kind, cp, conn = grid2d(nx, ny, 3.0, 1.0, jitter=0.2, tris=tris, seed=seed)
    left = [j * (nx + 1) for j in range(ny + 1)]
    per = 2 if tris else 1
    # heat flows in through the right edge of the last column of cells:
    # edge 2 (b -> c) of a quad (a, b, c, d) or of its first triangle (a, b, c)
    right_cells = [j * nx + nx - 1 for j in range(ny)]
    if tris:
        fe, ff = [per * c for c in right_cells], [2] * ny
    else:
        fe, ff = right_cells, [2] * ny
    return ThermalModel(xyz, kind, cp, conn, 3.5, thickness=0.02, source=120.0,
                        temp_node=left + [left[0]], temp_value=[10.0] * len(left) + [15.0],
                        flux_elem=fe, flux_face=ff, flux_value=[40.0] * ny)


@pytest.mark.parametrize("tris", [False, True])
def test_plate_with_source_flux_and_temperatures_matches_oracle(ctx, tris):
    tm = plate_case(tris, seed=5)
    t, it, res = ctx.solve_thermal(tm)
    t_o, it_o, res_o = oracle.solve_thermal(tm)
    assert res <= 1e-10
    assert rel(t, t_o) <= 1e-10
    assert abs(it - it_o) <= max(3, it_o // 10)
    # the later constraint on node 0 wins (heat.rs:367-375); prescribed
    # values come out of the PCG like the free ones, to its tolerance
    assert abs(t[0] - 15.0) <= 1e-8 * 15.0


def test_hex_block_with_source_matches_oracle(ctx):
    xyz, kind, cp, conn, nid = hex_grid(12, 4, 3, 1.2, 0.4, 0.3)
    cold = [nid(0, j, k) for k in range(4) for j in range(5)]
    hot = [nid(12, j, k) for k in range(4) for j in range(5)]
    tm = ThermalModel(xyz, kind, cp, conn, 45.0, source=2.0e4, temp_node=cold + hot,
                      temp_value=[20.0] * len(cold) + [80.0] * len(hot))
    t, _, res = ctx.solve_thermal(tm)
    t_o, _, _ = oracle.solve_thermal(tm)
    assert res <= 1e-10 and rel(t, t_o) <= 1e-10


def test_known_answer_cases_of_the_reference(ctx):
    # heat.rs:529-558 (quad bar), 560-593 (hex bar), 595-645 (flux)
    xyz, kind, cp, conn = grid2d(8, 1, 1.0, 0.1)
    left, right = [0, 9], [8, 17]
    tm = ThermalModel(xyz, kind, cp, conn, 1.0, temp_node=left + right,
                      temp_value=[100.0, 100.0, 0.0, 0.0])
    t, it, res = ctx.solve_thermal(tm)
    assert res <= 1e-10 and it > 0
    assert np.max(np.abs(t - 100.0 * (1.0 - xyz[:, 0]))) < 1e-8
    hx, hk, hcp, hconn, nid = hex_grid(6, 1, 1, 1.0, 0.1, 0.1)
    cold = [nid(0, j, k) for k in range(2) for j in range(2)]
    hot = [nid(6, j, k) for k in range(2) for j in range(2)]
    tm = ThermalModel(hx, hk, hcp, hconn, 5.0, temp_node=cold + hot,
                      temp_value=[20.0] * 4 + [120.0] * 4)
    t, _, _ = ctx.solve_thermal(tm)
    assert np.max(np.abs(t - (20.0 + 100.0 * hx[:, 0]))) < 1e-8
    xyz, kind, cp, conn = grid2d(6, 1, 1.0, 0.1)
    tm = ThermalModel(xyz, kind, cp, conn, 2.0, temp_node=[0, 7], temp_value=[0.0, 0.0],
                      flux_elem=[5], flux_face=[2], flux_value=[50.0])
    t, _, _ = ctx.solve_thermal(tm)
    assert np.max(np.abs(t - 50.0 * xyz[:, 0] / 2.0)) < 1e-8


def test_errors_follow_the_reference(ctx):
    xyz, kind, cp, conn = grid2d(2, 1, 1.0, 0.1)
    with pytest.raises(NoConstraints):
        ctx.solve_thermal(ThermalModel(xyz, kind, cp, conn, 1.0))
    with pytest.raises(EmptyMesh):
        ctx.solve_thermal(ThermalModel(np.zeros((0, 3)), [], [0], [], 1.0, temp_node=[],
                                       temp_value=[]))
    with pytest.raises(InvalidModel, match="thickness and conductivity must be positive"):
        ctx.solve_thermal(ThermalModel(xyz, kind, cp, conn, -1.0, temp_node=[0],
                                       temp_value=[1.0]))
    with pytest.raises(InvalidModel, match=r"element 2 \(Cps4\) has no face 7"):
        ctx.solve_thermal(ThermalModel(xyz, kind, cp, conn, 1.0, temp_node=[0],
                                       temp_value=[1.0], flux_elem=[1], flux_face=[7],
                                       flux_value=[1.0]))
    inside_out = np.array(conn).reshape(-1, 4)
    inside_out[1] = inside_out[1][::-1]
    with pytest.raises(InvalidModel, match="element 2: non-positive Jacobian"):
        ctx.solve_thermal(ThermalModel(xyz, kind, cp, inside_out.ravel(), 1.0, temp_node=[0],
                                       temp_value=[1.0]))
    with pytest.raises(ValueError):
        ctx.solve_thermal(ThermalModel(xyz, kind, cp, conn, 1.0, temp_node=[99],
                                       temp_value=[1.0]))
    assert abi.SVX_OK == 0
