"""Seeded synthetic workloads (flat models) for the benchmark configurations.

No public dataset exists for this path; every workload is generated from a
fixed seed (``numpy.random.Generator(PCG64(seed))``) with the shapes, sizes
and value distributions of the configurations it stands for:

* ``cantilever_cps4``  2D CPS4 plane-stress cantilever (default 200 x 20,
  10 m x 1 m, interior jitter +-0.15 h, t = 0.01, E = 210e9, nu = 0.3, x = 0
  clamped in dofs 1-2, -1000 N in dof 2 at the top-right node; seed 1);
* ``cantilever_c3d8``  3D C3D8 cantilever (default 160 x 16 x 16 over
  2.0 x 0.2 x 0.2 m, interior jitter +-0.1 h, E = 70e9, nu = 0.33, x = 0
  face clamped, -5 kN in z spread over the x = L face nodes; seed 2), with
  an optional per-element log-uniform E (the 480 x 48 x 48 heterogeneous
  case, E = 10^U(9, 11), nu = 0.3; seed 3);
* ``plate_batch``      uneven 2D plates (nx ~ U{10..160}, ny ~ U{4..40},
  h = 1, CPS4 or CPS3 with a per-quad split diagonal, E = 10^U(9, log10 3e11),
  nu ~ U(0.15, 0.45), t ~ U(0.001, 0.05), left edge clamped, one CLOAD of
  U(100, 1e4) N at a random right-edge node, random dof and sign; seed 4);
* ``request_stream``   70 % plates as above and 30 % C3D8 cantilevers
  (nx ~ U{20..120}, ny = nz ~ U{4..16}, E = 70e9, nu = 0.33, tip load
  U(1e3, 1e4) N) with Poisson arrival times (seed 5).

Node numbering follows the reference's structured builders (row-major, x
fastest; C3D8 bottom face counter-clockwise then top,
crates/solvix-core/src/assembly.rs:554-624).
"""
from __future__ import annotations

import numpy as np

from . import abi
from .marshal import FlatModel


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _quad_connectivity(nx: int, ny: int) -> np.ndarray:
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    n0 = j * (nx + 1) + i
    return np.stack([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1], axis=-1).reshape(-1, 4)


def _hex_connectivity(nx: int, ny: int, nz: int) -> np.ndarray:
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    sx, sxy = nx + 1, (nx + 1) * (ny + 1)
    n0 = k * sxy + j * sx + i
    c = np.stack([n0, n0 + 1, n0 + sx + 1, n0 + sx,
                  n0 + sxy, n0 + sxy + 1, n0 + sxy + sx + 1, n0 + sxy + sx], axis=-1)
    return c.reshape(-1, 8)


def cantilever_cps4(nx: int = 200, ny: int = 20, length: float = 10.0, height: float = 1.0,
                    jitter: float = 0.15, thickness: float = 0.01, E: float = 210e9,
                    nu: float = 0.3, load: float = -1000.0, seed: int = 1) -> FlatModel:
    rng = _rng(seed)
    hx, hy = length / nx, height / ny
    j, i = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    x = (i * hx).astype(np.float64).ravel()
    y = (j * hy).astype(np.float64).ravel()
    interior = ((i > 0) & (i < nx) & (j > 0) & (j < ny)).ravel()
    dx = rng.uniform(-jitter, jitter, size=x.shape) * hx
    dy = rng.uniform(-jitter, jitter, size=y.shape) * hy
    x = np.where(interior, x + dx, x)
    y = np.where(interior, y + dy, y)
    xyz = np.stack([x, y, np.zeros_like(x)], axis=1)
    conn = _quad_connectivity(nx, ny)
    n_nodes = xyz.shape[0]
    root = np.arange(ny + 1) * (nx + 1)
    fixed = np.stack([root * 2, root * 2 + 1], axis=1).ravel()
    f = np.zeros(n_nodes * 2)
    tip = ny * (nx + 1) + nx
    f[tip * 2 + 1] = load
    return FlatModel(xyz=xyz, kind=np.full(conn.shape[0], abi.SVX_CPS4, np.uint8),
                     conn_ptr=np.arange(conn.shape[0] + 1, dtype=np.int64) * 4,
                     conn=conn.ravel(), youngs=E, poisson=nu, thickness=thickness, ndof=2,
                     fixed_row=fixed, f=f,
                     node_id=np.arange(1, n_nodes + 1, dtype=np.uint32),
                     elem_id=np.arange(1, conn.shape[0] + 1, dtype=np.uint32))


def cantilever_c3d8(nx: int = 160, ny: int = 16, nz: int = 16, lx: float = 2.0,
                    ly: float = 0.2, lz: float = 0.2, jitter: float = 0.1, E=70e9,
                    nu: float = 0.33, total_load: float = -5000.0, load_dof: int = 3,
                    hetero_E: tuple | None = None, seed: int = 2) -> FlatModel:
    """hetero_E = (log10 lo, log10 hi) draws a per-element log-uniform E."""
    rng = _rng(seed)
    hx, hy, hz = lx / nx, ly / ny, lz / nz
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1),
                          indexing="ij")
    pts = [(i * hx).ravel().astype(np.float64), (j * hy).ravel().astype(np.float64),
           (k * hz).ravel().astype(np.float64)]
    interior = ((i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)).ravel()
    for a, h in enumerate((hx, hy, hz)):
        d = rng.uniform(-jitter, jitter, size=pts[a].shape) * h
        pts[a] = np.where(interior, pts[a] + d, pts[a])
    xyz = np.stack(pts, axis=1)
    conn = _hex_connectivity(nx, ny, nz)
    n_elem = conn.shape[0]
    n_nodes = xyz.shape[0]
    if hetero_E is not None:
        youngs = 10.0 ** rng.uniform(hetero_E[0], hetero_E[1], size=n_elem)
    else:
        youngs = np.full(n_elem, float(E))
    root = (i == 0).ravel().nonzero()[0]
    fixed = np.stack([root * 3, root * 3 + 1, root * 3 + 2], axis=1).ravel()
    tip = (i == nx).ravel().nonzero()[0]
    f = np.zeros(n_nodes * 3)
    f[tip * 3 + (load_dof - 1)] = total_load / tip.shape[0]
    return FlatModel(xyz=xyz, kind=np.full(n_elem, abi.SVX_C3D8, np.uint8),
                     conn_ptr=np.arange(n_elem + 1, dtype=np.int64) * 8, conn=conn.ravel(),
                     youngs=youngs, poisson=nu, thickness=1.0, ndof=3, fixed_row=fixed, f=f,
                     node_id=np.arange(1, n_nodes + 1, dtype=np.uint32),
                     elem_id=np.arange(1, n_elem + 1, dtype=np.uint32))


def heterogeneous_c3d8(nx: int = 480, ny: int = 48, nz: int = 48, seed: int = 3) -> FlatModel:
    """The precision case: 480 x 48 x 48 C3D8, E = 10^U(9, 11) per element,
    nu = 0.3, clamp and -5 kN tip load as the 160 x 16 x 16 case."""
    return cantilever_c3d8(nx, ny, nz, hetero_E=(9.0, 11.0), nu=0.3, seed=seed)


def plate(rng: np.random.Generator, nx: int | None = None, ny: int | None = None) -> FlatModel:
    """One model of the 2D plate distribution."""
    nx = int(rng.integers(10, 161)) if nx is None else nx
    ny = int(rng.integers(4, 41)) if ny is None else ny
    tri = bool(rng.random() < 0.5)
    E = 10.0 ** rng.uniform(9.0, np.log10(3e11))
    nu = rng.uniform(0.15, 0.45)
    t = rng.uniform(0.001, 0.05)
    j, i = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    xyz = np.stack([i.ravel().astype(np.float64), j.ravel().astype(np.float64),
                    np.zeros(i.size)], axis=1)
    quads = _quad_connectivity(nx, ny)
    if tri:
        diag = rng.random(quads.shape[0]) < 0.5  # split along 0-2 or 1-3
        t1 = np.where(diag[:, None], quads[:, [0, 1, 2]], quads[:, [0, 1, 3]])
        t2 = np.where(diag[:, None], quads[:, [0, 2, 3]], quads[:, [1, 2, 3]])
        conn = np.stack([t1, t2], axis=1).reshape(-1, 3)
        kind, nn = abi.SVX_CPS3, 3
    else:
        conn, kind, nn = quads, abi.SVX_CPS4, 4
    n_nodes = xyz.shape[0]
    root = np.arange(ny + 1) * (nx + 1)
    fixed = np.stack([root * 2, root * 2 + 1], axis=1).ravel()
    f = np.zeros(n_nodes * 2)
    node = int(rng.integers(0, ny + 1)) * (nx + 1) + nx
    dof = int(rng.integers(0, 2))
    sign = 1.0 if rng.random() < 0.5 else -1.0
    f[node * 2 + dof] = sign * rng.uniform(100.0, 1e4)
    n_elem = conn.shape[0]
    return FlatModel(xyz=xyz, kind=np.full(n_elem, kind, np.uint8),
                     conn_ptr=np.arange(n_elem + 1, dtype=np.int64) * nn, conn=conn.ravel(),
                     youngs=E, poisson=nu, thickness=t, ndof=2, fixed_row=fixed, f=f,
                     node_id=np.arange(1, n_nodes + 1, dtype=np.uint32),
                     elem_id=np.arange(1, n_elem + 1, dtype=np.uint32))


def plate_batch(count: int = 4096, seed: int = 4) -> list:
    rng = _rng(seed)
    return [plate(rng) for _ in range(count)]


def small_cantilever_c3d8(rng: np.random.Generator) -> FlatModel:
    """One C3D8 request of the serving mix."""
    nx = int(rng.integers(20, 121))
    nyz = int(rng.integers(4, 17))
    load = -rng.uniform(1e3, 1e4)
    return cantilever_c3d8(nx, nyz, nyz, lx=nx / nyz * 0.1, ly=0.1, lz=0.1, jitter=0.0,
                           E=70e9, nu=0.33, total_load=load, seed=int(rng.integers(1 << 31)))


def request_stream(count: int = 20000, rate_per_s: float = 100.0, seed: int = 5):
    """[(arrival_s, FlatModel)] with Poisson arrivals.  The models do not
    depend on the rate (the unit-rate gaps are drawn first and scaled)."""
    rng = _rng(seed)
    t = np.cumsum(rng.exponential(1.0, size=count)) / rate_per_s
    out = []
    for k in range(count):
        m = plate(rng) if rng.random() < 0.7 else small_cantilever_c3d8(rng)
        out.append((float(t[k]), m))
    return out
