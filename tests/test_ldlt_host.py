"""The direct path's host side (no GPU): the product's reverse Cuthill-McKee
ordering (svx_order_rcm) is the reference's (ldl.rs:27-60, restated by the
oracle) permutation for permutation, its half-bandwidth is the pattern's in
that order, and the ABI carries the method option and its outputs."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle
from solvix_b200 import abi
from svx_cases import hex_cantilever, quad_mesh, steel_model
from test_oracle_ldlt import csr_from_rows, grid_csr, modified_system, slender_column
from solvix_b200.model import BoundaryCondition, ConcentratedLoad, ElemKind, Element, Mesh, Node


def product_rcm(k):
    lib = abi.load()
    perm = np.zeros(k.n, dtype=np.int32)
    bw = C.c_int64(-1)
    rp = np.ascontiguousarray(k.row_ptr, dtype=np.int64)
    ci = np.ascontiguousarray(k.col_idx, dtype=np.int32)
    st = lib.svx_order_rcm(k.n, abi.ptr(rp, C.c_int64), abi.ptr(ci, C.c_int32),
                           abi.ptr(perm, C.c_int32), C.byref(bw))
    assert st == abi.SVX_OK
    return perm, int(bw.value)


def pattern(a):
    """Oracle-shaped CSR of a scipy matrix's pattern (sorted columns)."""
    a = sp.csr_matrix(a)
    a.sort_indices()
    k = csr_from_rows([[(int(c), 1.0) for c in a.indices[a.indptr[r]:a.indptr[r + 1]]]
                       for r in range(a.shape[0])])
    return k


def dangling_model():
    mesh = quad_mesh(4, 2, 2.0, 1.0)
    nodes = [Node(i, tuple(c)) for i, c in zip(mesh.node_ids.tolist(), mesh.coords)]
    nodes += [Node(99, (9.0, 9.0, 0.0)), Node(98, (8.0, 9.0, 0.0))]
    conn = mesh.conn.reshape(-1, 4)
    elems = [Element(i + 1, ElemKind.Cps4, conn[i].tolist()) for i in range(len(conn))]
    m = steel_model(Mesh(nodes, elems))
    m.boundary_conditions = [BoundaryCondition([1, 6, 11], [1, 2])]
    m.cloads = [ConcentratedLoad(15, 2, -100.0)]
    return m


def cases():
    yield "grid 20x5", grid_csr(20, 5)
    yield "slender column", modified_system(slender_column()[0])[0]
    yield "hex 40x4x4", modified_system(hex_cantilever(40, 4, 4))[0]
    yield "hex 7x5x3", modified_system(hex_cantilever(7, 5, 3))[0]
    yield "dangling nodes", modified_system(dangling_model())[0]
    rng = np.random.Generator(np.random.PCG64(3))
    for n, dens in ((1, 1.0), (2, 1.0), (50, 0.05), (400, 0.004), (300, 0.0)):
        a = sp.random(n, n, density=dens, random_state=int(rng.integers(1 << 30)), format="csr")
        a = (a + a.T + sp.identity(n)).tocsr()
        yield f"random {n}", pattern(a)


@pytest.mark.parametrize("name,k", list(cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_rcm_is_the_reference_permutation(name, k):
    perm, bw = product_rcm(k)
    want = oracle.rcm(k)
    assert np.array_equal(perm, want), name
    rows = np.repeat(np.arange(k.n), np.diff(k.row_ptr))
    assert bw == (int(np.max(np.abs(want[rows] - want[k.col_idx]))) if k.nnz else 0)


def test_rcm_rejects_bad_patterns():
    lib = abi.load()
    perm = np.zeros(2, dtype=np.int32)
    bw = C.c_int64(0)
    rp = np.array([0, 1, 2], dtype=np.int64)
    ci = np.array([0, 5], dtype=np.int32)
    assert lib.svx_order_rcm(2, abi.ptr(rp, C.c_int64), abi.ptr(ci, C.c_int32),
                             abi.ptr(perm, C.c_int32), C.byref(bw)) == abi.SVX_BAD_ARGUMENT
    rp = np.array([0, 2, 1], dtype=np.int64)
    ci = np.array([0, 1], dtype=np.int32)
    assert lib.svx_order_rcm(2, abi.ptr(rp, C.c_int64), abi.ptr(ci, C.c_int32),
                             abi.ptr(perm, C.c_int32), C.byref(bw)) == abi.SVX_BAD_ARGUMENT
    assert lib.svx_order_rcm(0, None, None, None, None) == abi.SVX_OK


def test_method_option_and_direct_outputs_in_the_abi():
    opts = abi.default_opts()
    assert opts.method == abi.SVX_METHOD_PCG
    names = [f for f, _ in abi.SvxSolution._fields_]
    assert names[-3:] == ["solver_method", "factor_bandwidth", "ms_factor"]
    assert (abi.SVX_METHOD_PCG, abi.SVX_METHOD_LDLT, abi.SVX_METHOD_AUTO) == (0, 1, 2)
