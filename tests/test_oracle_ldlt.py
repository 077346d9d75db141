"""The oracle's restatement of the reference's direct path (CPU only).

ldl.rs (reverse Cuthill-McKee ordering, elimination tree, up-looking LDLT,
its solve and the D-based condition estimate) and the Method dispatch of
lib.rs:664-686 (Pcg, Ldlt, Auto = PCG with the direct fallback when PCG
returns NotConverged).  Pinned by the reference's own tests: ldl.rs:293-434
and lib.rs:909-1084, 1721-1807 (patch tests run through both methods),
lib.rs:1862-1937 (the slender column whose PCG stalls).  A second, pure
Python restatement of ldl.rs below cross-checks the C++ one bit for bit on
small systems.
"""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200.model import (BoundaryCondition, ConcentratedLoad, ElemKind, Element,
                               ElementSet, InvalidModel, Material, Mesh, Model, Node,
                               NotConverged)
from svx_cases import (E_STEEL, NU_STEEL, fmt_mm, fmt_mpa, hex_cantilever, hex_mesh,
                       load_golden, max_disp, quad_mesh, steel_model)


# ---------------------------------------------------------------- helpers
def csr_from_rows(rows):
    """ldl.rs:314-330."""
    row_ptr, col, val = [0], [], []
    for r in rows:
        for c, v in r:
            col.append(c)
            val.append(v)
        row_ptr.append(len(col))
    k = oracle.Csr.__new__(oracle.Csr)
    k.n, k.nnz = len(rows), len(col)
    k.row_ptr = np.array(row_ptr, dtype=np.int64)
    k.col_idx = np.array(col, dtype=np.int64)
    k.vals = np.array(val, dtype=np.float64)
    k.f = np.zeros(k.n)
    return k


def grid_csr(nx, ny):
    """ldl.rs:286-291: K of model_with_mesh(quad_mesh(nx, ny, 1, 1)),
    E = 1, nu = 0.25 (assembly.rs:697-722), before Dirichlet."""
    mesh = quad_mesh(nx, ny, 1.0, 1.0)
    m = Model(mesh=mesh, thickness=1.0, materials=[Material("mat", 1.0, 0.25)],
              elsets=[ElementSet("all", mesh.elem_ids.tolist())],
              mat_assignments=[("all", "mat")],
              boundary_conditions=[BoundaryCondition([1], [1, 2])])
    flat, _ = oracle.resolve(m)
    return oracle.assemble(flat, threads=1)


def bandwidth(k):
    """ldl.rs:276-284."""
    rows = np.repeat(np.arange(k.n), np.diff(k.row_ptr))
    return int(np.max(np.abs(rows - k.col_idx)))


def permuted(k, perm):
    invp = np.empty_like(perm)
    invp[perm] = np.arange(k.n)
    rows = [sorted((int(perm[k.col_idx[p]]), float(k.vals[p]))
                   for p in range(k.row_ptr[old], k.row_ptr[old + 1])) for old in invp]
    return csr_from_rows(rows), invp


def modified_system(model):
    """The Dirichlet-modified K and f that the reference factorizes."""
    flat, _ = oracle.resolve(model)
    k = oracle.assemble(flat, threads=1)
    f = flat.f.copy()
    oracle.apply_dirichlet(k, f, flat.fixed_row)
    return k, f, flat


# ------------------------------------------- pure-Python restatement of ldl.rs
def py_rcm(k):
    n = k.n
    deg = np.diff(k.row_ptr)
    visited = [False] * n
    order = []
    while len(order) < n:
        start = min((i for i in range(n) if not visited[i]), key=lambda i: deg[i])
        visited[start] = True
        queue, head = [start], 0
        while head < len(queue):
            u = queue[head]
            head += 1
            order.append(u)
            for idx in range(k.row_ptr[u], k.row_ptr[u + 1]):
                v = int(k.col_idx[idx])
                if not visited[v]:
                    visited[v] = True
                    queue.append(v)
    perm = np.empty(n, dtype=np.int64)
    for new, old in enumerate(reversed(order)):
        perm[old] = new
    return perm


def py_ldlt(k, b):
    """ldl.rs:144-251 line by line; returns (x, d, nnz_l)."""
    n = k.n
    perm = py_rcm(k)
    a, invp = permuted(k, perm)
    parent, ancestor = [-1] * n, [-1] * n
    for i in range(n):
        for p in range(a.row_ptr[i], a.row_ptr[i + 1]):
            node = int(a.col_idx[p])
            while node < i:
                nxt = ancestor[node]
                ancestor[node] = i
                if nxt == -1:
                    parent[node] = i
                    break
                node = nxt
    lp, lc, lv, d = [0], [], [], [0.0] * n
    x = [0.0] * n
    seen = [-1] * n
    for i in range(n):
        pattern = []
        seen[i] = i
        for p in range(a.row_ptr[i], a.row_ptr[i + 1]):
            node = int(a.col_idx[p])
            while node < i and seen[node] != i:
                pattern.append(node)
                seen[node] = i
                if parent[node] == -1:
                    break
                node = parent[node]
        pattern.sort()
        aii = 0.0
        for p in range(a.row_ptr[i], a.row_ptr[i + 1]):
            c = int(a.col_idx[p])
            x[c] = float(a.vals[p])
            if c == i:
                aii = float(a.vals[p])
        for kk in pattern:
            w = x[kk]
            for p in range(lp[kk], lp[kk + 1]):
                w -= lv[p] * x[lc[p]]
            x[kk] = w
            lik = w / d[kk]
            aii -= lik * w
            lc.append(kk)
            lv.append(lik)
        lp.append(len(lc))
        for kk in pattern:
            x[kk] = 0.0
        for p in range(a.row_ptr[i], a.row_ptr[i + 1]):
            x[int(a.col_idx[p])] = 0.0
        d[i] = aii
    y = [float(b[invp[i]]) for i in range(n)]
    for i in range(n):
        s = y[i]
        for p in range(lp[i], lp[i + 1]):
            s -= lv[p] * y[lc[p]]
        y[i] = s
    y = [yi / di for yi, di in zip(y, d)]
    for i in reversed(range(n)):
        xi = y[i]
        for p in range(lp[i], lp[i + 1]):
            y[lc[p]] -= lv[p] * xi
    out = np.zeros(n)
    out[invp] = y
    return out, np.array(d), len(lv)


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


# ------------------------------------------------------------------ ldl.rs
def test_rcm_is_a_valid_permutation_that_cuts_bandwidth():
    """ldl.rs:293-312."""
    k = grid_csr(20, 5)
    perm = oracle.rcm(k)
    assert np.array_equal(np.sort(perm), np.arange(k.n))
    reordered, _ = permuted(k, perm)
    assert bandwidth(reordered) < bandwidth(k)


def test_factorize_and_solve_small_spd_system():
    """ldl.rs:332-348."""
    k = csr_from_rows([[(0, 4.0), (1, 1.0)], [(0, 1.0), (1, 3.0), (2, 1.0)],
                       [(1, 1.0), (2, 2.0)]])
    b = np.array([1.0, 2.0, 3.0])
    r = oracle.ldlt(k, b)
    ku = oracle.spmv(k, r.u, threads=1)
    assert np.all(np.abs(ku - b) < 1e-12)
    assert r.cond > 1.0


def test_factorize_rejects_singular_matrix():
    """ldl.rs:350-359: the second pivot of [1 1; 1 1] is exactly zero."""
    k = csr_from_rows([[(0, 1.0), (1, 1.0)], [(0, 1.0), (1, 1.0)]])
    with pytest.raises(InvalidModel, match=r"^stiffness matrix is not positive definite "
                                           r"\(pivot near-zero at equation 1\)$"):
        oracle.ldlt(k, np.ones(2))


def test_negative_pivot_text():
    k = csr_from_rows([[(0, 1.0), (1, 2.0)], [(0, 2.0), (1, 1.0)]])
    with pytest.raises(InvalidModel, match=r"\(pivot negative at equation 1\)$"):
        oracle.ldlt(k, np.ones(2))


def test_fill_and_3d_cantilever():
    """ldl.rs:361-434: hex cantilever 40x4x4; direct residual < 1e-8, then
    both public methods (Auto at the PCG bar, Ldlt one decade looser)."""
    m = hex_cantilever(40, 4, 4)
    k, f, _ = modified_system(m)
    r = oracle.ldlt(k, f)
    assert r.residual < 1e-8
    assert r.nnz_l > k.nnz // 2
    for method, tol in (("auto", 1e-10), ("ldlt", 1e-8)):
        sol, _ = oracle.solve(m, method=method)
        assert sol.final_residual <= tol
    auto, _ = oracle.solve(m, method="auto")
    direct, _ = oracle.solve(m, method="ldlt")
    assert auto.solver_method == "pcg" and auto.iterations > 0
    assert direct.solver_method == "ldlt" and direct.iterations == 0
    assert direct.cond_estimate == r.cond
    rel = np.linalg.norm(direct.u - auto.u) / np.linalg.norm(auto.u)
    assert rel < 1e-8


@pytest.mark.parametrize("case", ["grid", "hex", "dangling_free"])
def test_cxx_restatement_matches_python_restatement_bitwise(case):
    if case == "grid":
        m = steel_model(quad_mesh(7, 3, 2.0, 0.5))
        m.boundary_conditions = [BoundaryCondition([1, 9, 17, 25], [1, 2])]
        m.cloads = [ConcentratedLoad(32, 2, -1000.0), ConcentratedLoad(16, 1, 300.0)]
    elif case == "hex":
        m = hex_cantilever(5, 2, 2)
    else:
        # a mesh in two pieces (two RCM components) joined by nothing
        mesh = quad_mesh(3, 2, 1.0, 1.0)
        nodes = list(zip(mesh.node_ids.tolist(), map(tuple, mesh.coords)))
        off = len(nodes)
        extra = [Node(off + i + 1, (5.0 + x, y, 0.0)) for i, (_, (x, y, _z)) in
                 enumerate(nodes)]
        conn = mesh.conn.reshape(-1, 4)
        elems = [Element(i + 1, ElemKind.Cps4, conn[i].tolist()) for i in range(len(conn))]
        elems += [Element(len(conn) + i + 1, ElemKind.Cps4, (conn[i] + off).tolist())
                  for i in range(len(conn))]
        mesh2 = Mesh([Node(i, c) for i, c in nodes] + extra, elems)
        m = steel_model(mesh2)
        m.boundary_conditions = [BoundaryCondition([1, 5, 9, off + 1, off + 5, off + 9],
                                                   [1, 2])]
        m.cloads = [ConcentratedLoad(12, 2, -10.0), ConcentratedLoad(off + 12, 1, 7.0)]
    k, f, _ = modified_system(m)
    assert np.array_equal(oracle.rcm(k), py_rcm(k))
    r = oracle.ldlt(k, f, threads=1)
    x, d, nnz_l = py_ldlt(k, f)
    assert r.nnz_l == nnz_l
    assert np.array_equal(bits(r.d), bits(d))
    assert np.array_equal(bits(r.u), bits(x))


def test_dangling_node_is_a_near_zero_pivot_on_the_direct_path_only():
    """A node used by no element keeps a zero diagonal (assembly.rs:299-302):
    Jacobi-PCG skips it (inv_diag 0, solver.rs:101-105) while the direct
    path rejects it; RCM starts at the degree-1 rows, so they come last."""
    mesh = quad_mesh(4, 2, 2.0, 1.0)
    nodes = [Node(i, tuple(c)) for i, c in zip(mesh.node_ids.tolist(), mesh.coords)]
    nodes.append(Node(99, (9.0, 9.0, 0.0)))
    conn = mesh.conn.reshape(-1, 4)
    elems = [Element(i + 1, ElemKind.Cps4, conn[i].tolist()) for i in range(len(conn))]
    m = steel_model(Mesh(nodes, elems))
    m.boundary_conditions = [BoundaryCondition([1, 6, 11], [1, 2])]
    m.cloads = [ConcentratedLoad(15, 2, -100.0)]
    sol, _ = oracle.solve(m, method="auto")
    assert sol.solver_method == "pcg"
    n = 2 * len(nodes)
    with pytest.raises(InvalidModel, match=rf"\(pivot near-zero at equation {n - 2}\)$"):
        oracle.solve(m, method="ldlt")


# ------------------------------------------------------------------ lib.rs
def _fix_left_edge_x(m, nx, ny):
    ids = [j * (nx + 1) + 1 for j in range(ny + 1)]
    m.boundary_conditions += [BoundaryCondition(ids, [1]), BoundaryCondition([1], [2])]


@pytest.mark.parametrize("method", ["auto", "ldlt"])
def test_patch_tests_through_both_methods(method):
    """lib.rs:907-950 (BOTH_METHODS), 1011-1084, 1721-1807."""
    sigma = 1e6
    m = steel_model(quad_mesh(1, 1, 1.0, 1.0))
    _fix_left_edge_x(m, 1, 1)
    m.cloads = [ConcentratedLoad(2, 1, sigma / 2), ConcentratedLoad(4, 1, sigma / 2)]
    sol, flat = oracle.solve(m, method=method)
    assert sol.solver_method == ("ldlt" if method == "ldlt" else "pcg")
    assert abs(sol.von_mises[0] - sigma) / sigma < 1e-6
    assert np.all(np.abs(sol.nodal_von_mises - sigma) / sigma < 1e-6)
    ux = sigma / E_STEEL
    assert abs(sol.displacements[1][0] - ux) / ux < 1e-6
    rx = sum(v for r, v in zip(flat.fixed_row, sol.reaction_values) if r % 2 == 0)
    assert abs(rx + sigma) < 1e-6 * sigma
    assert sol.final_residual <= 1e-10

    mesh = Mesh([Node(1, (0, 0, 0)), Node(2, (1, 0, 0)), Node(3, (1, 1, 0)), Node(4, (0, 1, 0))],
                [Element(1, ElemKind.Cps3, [1, 2, 3]), Element(2, ElemKind.Cps3, [1, 3, 4])])
    m = steel_model(mesh)
    m.boundary_conditions = [BoundaryCondition([1, 4], [1]), BoundaryCondition([1], [2])]
    m.cloads = [ConcentratedLoad(2, 1, 5e5), ConcentratedLoad(3, 1, 5e5)]
    sol, _ = oracle.solve(m, method=method)
    assert np.all(np.abs(sol.von_mises - sigma) / sigma < 1e-6)
    assert abs(sol.displacements[2][1] - (-NU_STEEL * sigma / E_STEEL)) / \
        (NU_STEEL * sigma / E_STEEL) < 1e-6

    m = steel_model(hex_mesh(1, 1, 1, 1.0, 1.0, 1.0))
    m.boundary_conditions = [BoundaryCondition([1, 2, 3, 4], [3]), BoundaryCondition([1], [1]),
                             BoundaryCondition([1, 2], [2])]
    m.cloads = [ConcentratedLoad(n, 3, sigma / 4) for n in (5, 6, 7, 8)]
    sol, flat = oracle.solve(m, method=method)
    assert np.all(np.abs(sol.von_mises - sigma) / sigma < 1e-6)
    w = sigma / E_STEEL
    for i in (4, 5, 6, 7):
        assert abs(sol.displacements[i][2] - w) / w < 1e-6
    rz = sum(v for r, v in zip(flat.fixed_row, sol.reaction_values) if r % 3 == 2)
    assert abs(rz + sigma) < 1e-6 * sigma


def slender_column():
    """lib.rs:1862-1901: a 1 x 40 CPS4 column of aspect 1000."""
    nx, ny, w, length = 1, 40, 1e-3, 1.0
    m = steel_model(quad_mesh(nx, ny, w, length))
    m.boundary_conditions = [BoundaryCondition([1, 2], [2]), BoundaryCondition([1], [1])]
    top_left, top_right = ny * (nx + 1) + 1, (ny + 1) * (nx + 1)
    p = 1000.0
    m.cloads = [ConcentratedLoad(top_left, 2, p / 2), ConcentratedLoad(top_right, 2, p / 2)]
    return m, p, p * length / (E_STEEL * w), (top_left, top_right)


def test_slender_column_pcg_budget_exhaustion_falls_back_to_ldlt():
    """lib.rs:1862-1937."""
    m, p, stretch, tops = slender_column()
    with pytest.raises(NotConverged):
        oracle.solve(m, method="pcg")
    for method in ("auto", "ldlt"):
        sol, flat = oracle.solve(m, method=method)
        assert sol.solver_method == "ldlt" and sol.iterations == 0
        for nid in tops:
            uy = sol.displacements[nid - 1][1]
            assert abs(uy - stretch) / stretch < 1e-6
        ry = sum(v for r, v in zip(flat.fixed_row, sol.reaction_values) if r % 2 == 1)
        assert abs(ry + p) < 1e-6 * p
        assert sol.cond_estimate > 1e4


@pytest.mark.parametrize("name", ["cantilever", "cantilever3d", "plate_hole"])
def test_example_decks_through_the_direct_path(name):
    """The direct solution of the example decks prints the same published
    max displacement and von Mises as the PCG one (docs/examples.md)."""
    model, g = load_golden(name)
    sol, _ = oracle.solve(model, method="ldlt")
    assert sol.solver_method == "ldlt" and sol.final_residual <= 1e-8
    assert fmt_mm(max_disp(sol.displacements)) == g["max_disp_mm"]
    assert fmt_mpa(max(0.0, sol.von_mises.max())) == g["max_von_mises_mpa"]


@pytest.mark.parametrize("seed", range(6))
def test_ldlt_agrees_with_a_dense_factorization_in_the_same_order(seed):
    """Random sparse SPD systems: the oracle's u solves the system like a
    dense solve, and its D is the squared diagonal of the dense Cholesky
    factor of the RCM-permuted matrix (so the condition estimate is the
    same), independently of the reference's own tests."""
    import scipy.sparse as sp
    rng = np.random.Generator(np.random.PCG64(100 + seed))
    n = int(rng.integers(20, 120))
    a = sp.random(n, n, density=min(1.0, 6.0 / n), random_state=int(rng.integers(1 << 30)))
    a = a + a.T
    a = a + sp.diags(np.abs(a).sum(axis=1).A1 + rng.uniform(0.5, 2.0, n))
    a = sp.csr_matrix(a)
    a.sort_indices()
    k = csr_from_rows([[(int(c), float(v)) for c, v in
                        zip(a.indices[a.indptr[r]:a.indptr[r + 1]],
                            a.data[a.indptr[r]:a.indptr[r + 1]])] for r in range(n)])
    b = rng.normal(size=n)
    r = oracle.ldlt(k, b, threads=1)
    dense = a.toarray()
    want = np.linalg.solve(dense, b)
    assert np.linalg.norm(r.u - want) <= 1e-12 * np.linalg.norm(want)
    perm = oracle.rcm(k)
    invp = np.empty_like(perm)
    invp[perm] = np.arange(n)
    chol = np.linalg.cholesky(dense[np.ix_(invp, invp)])
    d_dense = np.diag(chol) ** 2
    assert np.allclose(r.d, d_dense, rtol=1e-12, atol=0.0)
    assert abs(r.cond - d_dense.max() / d_dense.min()) <= 1e-12 * r.cond
