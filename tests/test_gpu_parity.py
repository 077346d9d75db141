"""Parity of the CUDA path against the oracle, through the C ABI (GPU).

Bars (as stated by the reference's own tests and the path's contract):
* CSR pattern (row_ptr, col_idx): bit-exact.
* K values: bit-exact against the oracle summing duplicates in the same
  fixed order (element ascending); within 1e-14 of the row scale against
  the reference's own (unstable-sort) order.
* Element stresses / reactions for the same u: bit-exact.
* Displacements: ||u - u_oracle|| / ||u_oracle|| <= 1e-10 (plain FP64);
  <= 1e-8 for the mixed-precision form.
* von Mises fields: max |vm - vm_oracle| <= 1e-8 * max |vm_oracle|.
"""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import abi, solve, workloads
from solvix_b200.marshal import FlatModel
from solvix_b200.model import (BoundaryCondition, ConcentratedLoad, ElemKind, Element,
                               InvalidModel, Mesh, Node, NotConverged)
from svx_cases import (fmt_e3, fmt_mm, fmt_mpa, hex_cantilever, load_golden, max_disp,
                       patch_deck, quad_mesh, steel_model)

pytestmark = pytest.mark.gpu

U_TOL = 1e-10
VM_TOL = 1e-8


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def vm_rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def same_bits(a, b):
    """Bitwise equality up to the sign of zero."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return bool(np.all((bits(a) == bits(b)) | ((a == 0) & (b == 0))))


# ------------------------------------------------------------------ meshes
def mixed_plate():
    """CPS3 and CPS4 in one model (plate generator, triangle branch + quads)."""
    rng = np.random.Generator(np.random.PCG64(11))
    tri = workloads.plate(rng, nx=7, ny=4)
    while tri.kind[0] != abi.SVX_CPS3:
        tri = workloads.plate(rng, nx=7, ny=4)
    return tri


def orphan_and_collapsed():
    """A quad mesh with one node used by no element and one collapsed quad
    (a repeated node) - the pattern's edge cases."""
    flat = workloads.cantilever_cps4(6, 3, length=3.0, height=1.5, jitter=0.0, seed=3)
    xyz = np.vstack([flat.xyz, [[9.0, 9.0, 0.0]]])  # orphan node, index n
    n_nodes = xyz.shape[0]
    conn = flat.conn.reshape(-1, 4).copy()
    # collapse the first element's third node onto its fourth (triangle-shaped
    # quad); the dropped corner stays in use by the neighbouring elements
    conn[0, 2] = conn[0, 3]
    f = np.zeros(n_nodes * 2)
    f[: flat.f.shape[0]] = flat.f
    return FlatModel(xyz=xyz, kind=flat.kind, conn_ptr=flat.conn_ptr, conn=conn.ravel(),
                     youngs=flat.youngs, poisson=flat.poisson, thickness=flat.thickness, ndof=2,
                     fixed_row=np.concatenate([flat.fixed_row, [2 * (n_nodes - 1),
                                                               2 * (n_nodes - 1) + 1]]), f=f)


CASES = {
    "cps4_jitter": lambda: workloads.cantilever_cps4(24, 6, length=2.4, height=0.6, seed=5),
    "c3d8_jitter": lambda: workloads.cantilever_c3d8(10, 3, 4, lx=1.0, ly=0.3, lz=0.4, seed=6),
    "c3d8_hetero": lambda: workloads.cantilever_c3d8(12, 4, 4, lx=1.2, ly=0.4, lz=0.4,
                                                     hetero_E=(9.0, 11.0), nu=0.3, seed=3),
    "mixed_cps3_cps4": mixed_plate,
    "orphan_collapsed": orphan_and_collapsed,
}


@pytest.fixture(params=sorted(CASES))
def case(request):
    return CASES[request.param]()


def test_pattern_and_values_bit_exact(ctx, case):
    op = ctx.assemble(case, keep_original=True)
    rp, ci, v = op.csr(which=1)
    oracle.set_sort_mode(1)
    k = oracle.assemble(case)
    assert np.array_equal(rp, k.row_ptr)
    assert np.array_equal(ci.astype(np.int64), k.col_idx)
    assert same_bits(v, k.vals)
    # against the reference's own duplicate order: last-bit differences only
    oracle.set_sort_mode(0)
    kr = oracle.assemble(case)
    scale = np.repeat(np.maximum.reduceat(np.abs(kr.vals), kr.row_ptr[:-1]),
                      np.diff(kr.row_ptr))
    scale = np.where(scale > 0, scale, 1.0)  # rows of an unreferenced node are all 0
    assert np.max(np.abs(v - kr.vals) / scale) <= 1e-14


def test_dirichlet_diagonal_and_spmv(ctx, case):
    op = ctx.assemble(case)
    rp, ci, v = op.csr(which=0)
    f_mod, inv_d = op.vectors(which=0)
    oracle.set_sort_mode(1)
    k = oracle.assemble(case)
    f = case.f.copy()
    oracle.apply_dirichlet(k, f, case.fixed_row)
    assert same_bits(v, k.vals) and same_bits(f_mod, f)
    d = np.array([k.vals[k.row_ptr[i] + np.nonzero(k.col_idx[k.row_ptr[i]:k.row_ptr[i + 1]]
                                                   == i)[0][0]] for i in range(k.n)])
    inv_ref = np.where(d == 0.0, 0.0, 1.0 / np.where(d == 0.0, 1.0, d))
    assert same_bits(inv_d, inv_ref)
    x = np.random.default_rng(1).standard_normal(k.n)
    y = op.spmv(x)
    y_ref = oracle.spmv(k, x)
    row_scale = np.abs(k.to_scipy()) @ np.abs(x) + 1e-300
    assert np.max(np.abs(y - y_ref) / row_scale) <= 1e-14


def test_solve_matches_oracle(ctx, case):
    sol = ctx.solve_flat(case)
    ref = oracle.solve_flat(case)
    assert rel(sol.u, ref.u) <= U_TOL
    assert vm_rel(sol.von_mises, ref.von_mises) <= VM_TOL
    assert vm_rel(sol.nodal_von_mises, ref.nodal_von_mises) <= VM_TOL
    assert np.max(np.abs(sol.reaction_values - ref.reaction_values)) <= \
        1e-8 * max(1.0, np.max(np.abs(ref.reaction_values)))
    assert sol.cond_estimate == pytest.approx(ref.cond_estimate, rel=1e-14)
    assert sol.final_residual <= 1e-10
    assert abs(sol.iterations - ref.iterations) <= max(3, ref.iterations // 10)


def test_stress_recovery_bit_exact_for_the_same_u(ctx, case):
    ref = oracle.solve_flat(case)
    op = ctx.assemble(case)
    op.set_solution(ref.u)
    vm, vmn, react, disp = op.stress()
    vm_o, vmn_o, react_o = oracle.stress(case, ref.u)
    assert same_bits(vm, vm_o) and same_bits(vmn, vmn_o)
    assert same_bits(disp.ravel()[: 3 * case.n_nodes],
                     ref.displacements.ravel())
    oracle.set_sort_mode(1)
    _, _, react_s = oracle.stress(case, ref.u)
    assert same_bits(react, react_s)
    assert np.max(np.abs(react - react_o)) <= 1e-9 * max(1.0, np.max(np.abs(react_o)))


@pytest.mark.parametrize("name", ["cantilever", "cantilever3d", "plate_hole"])
def test_reference_decks_through_the_public_api(ctx, name):
    model, g = load_golden(name)
    sol = solve(model, ctx=ctx)
    ref, _ = oracle.solve(model)
    assert rel(sol.u, ref.u) <= U_TOL
    assert fmt_mm(max_disp(sol.displacements)) == g["max_disp_mm"]
    assert fmt_mpa(sol.von_mises.max()) == g["max_von_mises_mpa"]
    if "max_nodal_von_mises_mpa" in g:
        assert fmt_mpa(sol.nodal_von_mises.max()) == g["max_nodal_von_mises_mpa"]
    assert abs(sol.iterations - g["iterations"]) <= max(3, g["iterations"] // 10)
    assert fmt_e3(sol.cond_estimate) == fmt_e3(ref.cond_estimate)
    assert sol.solver_method == "pcg"
    assert len(sol.reactions) == sum(len(b.node_ids) * len(b.dofs)
                                     for b in model.boundary_conditions)


def test_patch_deck(ctx):
    sol = solve(patch_deck(), ctx=ctx)
    assert fmt_mpa(sol.von_mises.max()) == "1.000"


def test_reaction_balance_and_bitwise_symmetry(ctx):
    """lib.rs:1121-1128: sum of reactions = -applied load; Ke is mirrored
    bitwise and summed in the same order on both sides, so K = K^T exactly."""
    m = hex_cantilever(20, 4, 4)
    sol = solve(m, ctx=ctx)
    ry = sum(r.value for r in sol.reactions if r.dof == 2)
    assert abs(ry - 10000.0) < 1e-6 * 10000.0
    flat, _ = oracle.resolve(m)
    op = ctx.assemble(flat, keep_original=True)
    rp, ci, v = op.csr(which=1)
    import scipy.sparse as sp
    a = sp.csr_matrix((v, ci, rp), shape=(op.n, op.n))
    assert (a != a.T).nnz == 0


def test_element_errors_and_precedence(ctx):
    # inverted hex (top and bottom faces swapped)
    m = steel_model(Mesh(
        [Node(i + 1, c) for i, c in enumerate(
            [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1),
             (0, 1, 1)])],
        [Element(9, ElemKind.C3d8, [5, 6, 7, 8, 1, 2, 3, 4])]))
    m.boundary_conditions = [BoundaryCondition([1, 2, 3, 4], [1, 2, 3])]
    m.cloads = [ConcentratedLoad(7, 3, 1.0)]
    with pytest.raises(InvalidModel, match=r"^element 9: non-positive Jacobian determinant at "
                                           r"a Gauss point$"):
        solve(m, ctx=ctx)
    # degenerate triangle before a material error on a later element
    mesh = Mesh([Node(1, (0, 0, 0)), Node(2, (1, 0, 0)), Node(3, (2, 0, 0)), Node(4, (1, 1, 0))],
                [Element(1, ElemKind.Cps3, [1, 2, 4]), Element(2, ElemKind.Cps3, [1, 2, 3]),
                 Element(3, ElemKind.Cps3, [2, 3, 4])])
    m = steel_model(mesh)
    m.elsets[0].element_ids = [1, 2]
    m.boundary_conditions = [BoundaryCondition([1], [1, 2])]
    m.cloads = [ConcentratedLoad(4, 1, 1.0)]
    with pytest.raises(InvalidModel, match=r"^element 2: degenerate \(zero-area\) triangle$"):
        solve(m, ctx=ctx)
    # an unsupported kind is rejected, not solved another way
    mesh = Mesh([Node(i + 1, (float(i % 3), float(i // 3), 0.0)) for i in range(9)],
                [Element(4, ElemKind.Cps8, [1, 3, 9, 7, 2, 6, 8, 4])])
    m = steel_model(mesh)
    m.boundary_conditions = [BoundaryCondition([1], [1, 2])]
    with pytest.raises(InvalidModel, match=r"^element 4: element kind CPS8 is outside"):
        solve(m, ctx=ctx)


def test_budget_exhaustion_surfaces_not_converged(ctx):
    flat = workloads.cantilever_cps4(40, 4, length=2.0, height=0.1, jitter=0.0)
    with pytest.raises(NotConverged) as ei:
        ctx.solve_flat(flat, max_iter=7)
    assert ei.value.iterations == 7 and ei.value.residual > 1e-10
    st, _u, it, res = oracle.pcg(_modified(flat), _fmod(flat), max_iter=7)
    assert it == 7 and abs(res - ei.value.residual) <= 1e-6 * res


def _modified(flat):
    k = oracle.assemble(flat)
    f = flat.f.copy()
    oracle.apply_dirichlet(k, f, flat.fixed_row)
    return k


def _fmod(flat):
    k = oracle.assemble(flat)
    f = flat.f.copy()
    oracle.apply_dirichlet(k, f, flat.fixed_row)
    return f


def test_zero_load_returns_zero_without_iterating(ctx):
    flat = workloads.cantilever_cps4(8, 2, jitter=0.0)
    flat.f[:] = 0.0
    sol = ctx.solve_flat(flat)
    assert sol.iterations == 0 and not sol.u.any() and sol.final_residual == 0.0


def test_runs_are_bitwise_deterministic(ctx):
    flat = workloads.cantilever_c3d8(16, 4, 4, lx=1.6, ly=0.4, lz=0.4, seed=9)
    a = ctx.solve_flat(flat)
    b = ctx.solve_flat(flat)
    assert np.array_equal(bits(a.u), bits(b.u)) and a.iterations == b.iterations
    assert np.array_equal(bits(a.von_mises), bits(b.von_mises))


@pytest.mark.parametrize("precision", [abi.SVX_FP64, abi.SVX_MIXED])
def test_shared_and_global_adjacency_agree_bitwise(ctx, monkeypatch, precision):
    """The persistent kernels with each block's adjacency in shared memory
    (the default at these sizes) and in global memory (SVX_SHARED_ADJ_MAX=0
    when the context is created) do the same arithmetic in the same order."""
    from solvix_b200 import Context
    flats = [workloads.cantilever_c3d8(16, 4, 4, lx=1.6, ly=0.4, lz=0.4, seed=9),
             workloads.cantilever_cps4(60, 8, seed=3)]
    monkeypatch.setenv("SVX_SHARED_ADJ_MAX", "0")
    with Context(0) as plain_ctx:
        monkeypatch.delenv("SVX_SHARED_ADJ_MAX")
        for flat in flats:
            a = ctx.solve_flat(flat, precision=precision)
            b = plain_ctx.solve_flat(flat, precision=precision)
            assert a.iterations == b.iterations
            assert np.array_equal(bits(a.u), bits(b.u))
            assert np.array_equal(bits(a.von_mises), bits(b.von_mises))


def test_mixed_precision_meets_1e8(ctx):
    flat = workloads.cantilever_c3d8(24, 4, 4, lx=1.2, ly=0.2, lz=0.2, seed=2)
    ref = oracle.solve_flat(flat)
    sol = ctx.solve_flat(flat, precision=abi.SVX_MIXED)
    assert rel(sol.u, ref.u) <= 1e-8
    assert sol.solver_method == "pcg-mixed" and sol.outer_iterations >= 1
    assert vm_rel(sol.von_mises, ref.von_mises) <= 1e-7


def test_full_size_cantilever_c3d8_properties(ctx):
    """The 160 x 16 x 16 case at full size: pattern and values bit-exact
    against the oracle's assembly, and the solve's true residual and
    reaction balance (size-independent properties)."""
    flat = workloads.cantilever_c3d8()
    op = ctx.assemble(flat, keep_original=True)
    assert op.nnz == 10393929
    rp, ci, v = op.csr(which=1)
    oracle.set_sort_mode(1)
    k = oracle.assemble(flat)
    assert np.array_equal(rp, k.row_ptr) and np.array_equal(ci.astype(np.int64), k.col_idx)
    assert same_bits(v, k.vals)
    u, it, res, cond = op.solve()
    assert res <= 1e-10
    rk, ck, vk = op.csr(which=0)
    import scipy.sparse as sp
    a = sp.csr_matrix((vk, ck, rk), shape=(op.n, op.n))
    f_mod, _ = op.vectors(which=0)
    true_res = np.linalg.norm(f_mod - a @ u) / np.linalg.norm(f_mod)
    assert true_res <= 1e-9
    vm, vmn, react, _ = op.stress()
    assert abs(react[2::3].sum() - 5000.0) <= 1e-6 * 5000.0


def test_large_system_graph_path_fp64_mixed_and_defect(ctx):
    """Above 50M nonzeros (and whenever K exceeds L2) the solve iterates
    the standalone kernels in a CUDA graph (FP64); the mixed form and the
    defect correction's inner solves stream the difference-form FP32
    operator there too.  Host-checked properties at 657k DOF: the true
    residual of each solution through the CSR on the host, and both FP32
    forms against FP64 within their bar.  The stopping rule is the
    reference's, on the recursive residual (solver.rs:108-123); on this
    100x-contrast model the FP64 recursion drifts from the true residual by
    a factor of about 30 over ~5,000 iterations, hence the 1e-8 bar on the
    true residual."""
    flat = workloads.heterogeneous_c3d8(200, 32, 32, seed=7)
    op = ctx.assemble(flat)
    assert op.nnz > 50_000_000
    rk, ck, vk = op.csr(which=0)
    import scipy.sparse as sp
    a = sp.csr_matrix((vk, ck, rk), shape=(op.n, op.n))
    f_mod, _ = op.vectors(which=0)
    u64, it64, res64, _ = op.solve()
    assert res64 <= 1e-10
    assert np.linalg.norm(f_mod - a @ u64) / np.linalg.norm(f_mod) <= 1e-8
    um, itm, resm, _ = op.solve(precision=abi.SVX_MIXED)
    assert resm <= 1e-10
    assert np.linalg.norm(f_mod - a @ um) / np.linalg.norm(f_mod) <= 1e-8
    assert rel(um, u64) <= 1e-8
    # the defect correction: FP32 inner solves (the quad-layout FP32 SpMV on
    # FP32 vectors) inside FP64 corrections, with its iteration split
    ud, itd, resd, _ = op.solve(precision=abi.SVX_MIXED_DEFECT)
    assert resd <= 1e-10
    assert np.linalg.norm(f_mod - a @ ud) / np.linalg.norm(f_mod) <= 1e-8
    assert rel(ud, u64) <= 1e-8
    assert op.last_outer_iterations >= 2
    assert 0 < op.last_fp32_iterations <= itd
    op.free()
