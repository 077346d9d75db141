"""The consistent-mass operator on the device (svx_assemble_mass) against the
oracle's restatement of assemble_mass (crates/solvix-core/src/modal.rs:
82-146, 203-271), through the C ABI (GPU).

Bars: the CSR pattern is the stiffness's (bit-exact); values bit-exact
against the oracle summing the triplets in element order, within 1e-14 of
the row scale against the reference's own (unstable-sort) order; the
reference's mass-totals test (modal.rs:939-990) holds per element kind;
M x agrees with the exported CSR's product; errors carry the reference's
texts for the first failing element."""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import abi, workloads
from solvix_b200.marshal import FlatModel
from solvix_b200.model import InvalidModel

pytestmark = pytest.mark.gpu

RHO = 7850.0


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def same_bits(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return bool(np.all((bits(a) == bits(b)) | ((a == 0) & (b == 0))))


def mixed_plate():
    rng = np.random.Generator(np.random.PCG64(11))
    tri = workloads.plate(rng, nx=9, ny=5)
    while tri.kind[0] != abi.SVX_CPS3:
        tri = workloads.plate(rng, nx=9, ny=5)
    return tri


CASES = {
    "cps4_jitter": lambda: workloads.cantilever_cps4(24, 6, length=2.4, height=0.6, seed=5),
    "cps3_plate": mixed_plate,
    "c3d8_jitter": lambda: workloads.cantilever_c3d8(10, 3, 4, lx=1.0, ly=0.3, lz=0.4, seed=6),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_mass_pattern_and_values_match_the_oracle(ctx, name):
    flat = CASES[name]()
    op = ctx.assemble_mass(flat, RHO)
    stiff = ctx.assemble(flat)
    try:
        rp, ci, v = op.csr(which=0)
        srp, sci, _ = stiff.csr(which=0)
        # the stiffness's pattern, zeros and diagonals included
        assert np.array_equal(rp, srp) and np.array_equal(ci, sci)
        oracle.set_sort_mode(1)
        m = oracle.assemble_mass(flat, RHO)
        assert np.array_equal(rp, m.row_ptr)
        assert np.array_equal(ci.astype(np.int64), m.col_idx)
        assert same_bits(v, m.vals)
        oracle.set_sort_mode(0)
        mr = oracle.assemble_mass(flat, RHO)
        scale = np.repeat(np.maximum.reduceat(np.abs(mr.vals), mr.row_ptr[:-1]),
                          np.diff(mr.row_ptr))
        scale = np.where(scale > 0, scale, 1.0)
        assert np.max(np.abs(v - mr.vals) / scale) <= 1e-14
        # M x on the device against the exported matrix
        import scipy.sparse as sp
        a = sp.csr_matrix((v, ci, rp), shape=(op.n, op.n))
        x = np.random.default_rng(2).standard_normal(op.n)
        y = op.spmv(x)
        assert np.max(np.abs(y - a @ x)) <= 1e-13 * (np.abs(a) @ np.abs(x)).max()
        # a rigid translation along each direction carries the whole mass
        nd = flat.ndof
        for d in range(nd):
            e = np.zeros(op.n)
            e[d::nd] = 1.0
            total = e @ (a @ e)
            assert total == pytest.approx(float(np.sum(op.spmv(e)[d::nd])), rel=1e-12)
    finally:
        op.free()
        stiff.free()


def _one_element(kind, coords, ndof, thickness=1.0):
    n = len(coords)
    xyz = np.zeros((n, 3))
    xyz[:, :len(coords[0])] = coords
    return FlatModel(xyz=xyz, kind=np.array([kind], dtype=np.uint8),
                     conn_ptr=np.array([0, n], dtype=np.int64),
                     conn=np.arange(n, dtype=np.int32), youngs=np.array([1.0]),
                     poisson=np.array([0.3]), thickness=thickness, ndof=ndof,
                     fixed_row=np.zeros(0, dtype=np.int64), f=np.zeros(n * ndof))


def test_consistent_mass_totals_match_rho_times_volume(ctx):
    """modal.rs:939-990: per dof, the mass matrix sums to rho * volume (a
    rigid unit translation in one dof carries the element's whole mass)."""
    t = 0.01
    cases = [
        (abi.SVX_CPS3, [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]], 2, RHO * t * 0.5),
        (abi.SVX_CPS4, [[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]], 2, RHO * t),
        (abi.SVX_C3D8, [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.0], [0.0, 1.0, 0.0],
                        [0.0, 0.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 1.0], [0.0, 1.0, 1.0]],
         3, RHO),
    ]
    for kind, coords, nd, expect in cases:
        flat = _one_element(kind, coords, nd, thickness=t)
        op = ctx.assemble_mass(flat, RHO)
        try:
            e = np.zeros(op.n)
            e[0::nd] = 1.0
            total = float(e @ op.spmv(e))
            assert abs(total - expect) < 1e-9 * RHO, (kind, total, expect)
        finally:
            op.free()


def test_mass_errors_follow_the_reference(ctx):
    # an inverted hex (top and bottom faces swapped)
    hexc = [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1],
            [0, 1, 1]]
    inverted = _one_element(abi.SVX_C3D8, [hexc[i] for i in (4, 5, 6, 7, 0, 1, 2, 3)], 3)
    inverted.elem_id = np.array([9], dtype=np.uint32)
    with pytest.raises(InvalidModel, match=r"^element 9: non-positive Jacobian determinant at "
                                           r"a Gauss point$"):
        ctx.assemble_mass(inverted, RHO)
    # a zero-area triangle
    flat = _one_element(abi.SVX_CPS3, [[0.0, 0.0], [1.0, 0.0], [2.0, 0.0]], 2)
    flat.elem_id = np.array([2], dtype=np.uint32)
    with pytest.raises(InvalidModel, match=r"^element 2: degenerate \(zero-area\) triangle$"):
        ctx.assemble_mass(flat, RHO)
    # a mass operator is not solved; a negative density is refused
    ok = _one_element(abi.SVX_CPS4, [[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]], 2)
    op = ctx.assemble_mass(ok, RHO)
    try:
        with pytest.raises(ValueError, match="consistent mass"):
            op.solve()
    finally:
        op.free()
    with pytest.raises(ValueError, match="density"):
        ctx.assemble_mass(ok, -1.0)
