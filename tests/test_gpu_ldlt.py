"""The direct path on the device (SVX_METHOD_LDLT / SVX_METHOD_AUTO) against
the oracle's restatement of the reference's (ldl.rs, lib.rs:645-686).

Bars.  The device factorizes in the reference's RCM order but sums in another
order, so D and u agree with the oracle's to rounding amplified by the
conditioning: u within 1e-8 relative (the bar of the precision, batched and
served forms), within 1e-6 on the slender column (condition estimate
3.5e12, where the reference's own bar is 1e-6 against the analytical
stretch), and the D-based condition estimate within 1e-6 relative.
Residuals meet the reference's direct bar (1e-8); a failed pivot gives the
reference's message and equation.
"""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import abi, solve, solve_with_method
from solvix_b200.model import InvalidModel, Method
from svx_cases import (E_STEEL, NU_STEEL, fmt_mm, fmt_mpa, hex_cantilever, hex_mesh,
                       load_golden, max_disp, quad_mesh, steel_model)
from test_ldlt_host import dangling_model
from test_oracle_ldlt import modified_system, slender_column
from solvix_b200.model import BoundaryCondition, ConcentratedLoad, ElemKind, Element, Mesh, Node

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def direct_oracle(model):
    k, f, _ = modified_system(model)
    return oracle.ldlt(k, f)


def test_slender_column_falls_back_to_the_device_factorization(ctx):
    """lib.rs:1862-1937 through the device: PCG alone stalls, Auto and Ldlt
    give the direct solution."""
    m, p, stretch, tops = slender_column()
    ref = direct_oracle(m)
    for method in (Method.Auto, Method.Ldlt):
        sol = solve_with_method(m, method, ctx=ctx)
        assert sol.solver_method == "ldlt" and sol.iterations == 0
        for nid in tops:
            uy = sol.displacements[nid - 1][1]
            assert abs(uy - stretch) / stretch < 1e-6
        ry = sum(r.value for r in sol.reactions if r.dof == 2)
        assert abs(ry + p) < 1e-6 * p
        assert sol.cond_estimate > 1e4
        assert abs(sol.cond_estimate - ref.cond) <= 1e-6 * ref.cond
        assert sol.final_residual <= 1e-8
        assert rel(sol.u, ref.u) <= 1e-6


@pytest.mark.parametrize("dims", [(40, 4, 4), (6, 2, 2), (16, 8, 8)])
def test_hex_cantilevers_match_the_oracle(ctx, dims):
    """ldl.rs:361-434 (40x4x4) and wider bands (more tiles per step)."""
    m = hex_cantilever(*dims)
    ref = direct_oracle(m)
    sol = solve_with_method(m, Method.Ldlt, ctx=ctx)
    assert sol.solver_method == "ldlt" and sol.iterations == 0
    assert sol.final_residual <= 1e-8
    assert rel(sol.u, ref.u) <= 1e-8
    assert abs(sol.cond_estimate - ref.cond) <= 1e-6 * ref.cond
    pcg = solve_with_method(m, Method.Auto, ctx=ctx)
    assert pcg.solver_method == "pcg" and pcg.iterations > 0
    assert rel(sol.u, pcg.u) <= 1e-8


def test_patch_tests_through_the_direct_path(ctx):
    """lib.rs:907-950, 1011-1084, 1721-1807 with Method::Ldlt."""
    sigma = 1e6
    m = steel_model(quad_mesh(1, 1, 1.0, 1.0))
    m.boundary_conditions = [BoundaryCondition([1, 3], [1]), BoundaryCondition([1], [2])]
    m.cloads = [ConcentratedLoad(2, 1, sigma / 2), ConcentratedLoad(4, 1, sigma / 2)]
    sol = solve_with_method(m, Method.Ldlt, ctx=ctx)
    assert abs(sol.von_mises[0] - sigma) / sigma < 1e-6
    assert abs(sol.displacements[1][0] - sigma / E_STEEL) / (sigma / E_STEEL) < 1e-6
    assert sol.final_residual <= 1e-10

    mesh = Mesh([Node(1, (0, 0, 0)), Node(2, (1, 0, 0)), Node(3, (1, 1, 0)), Node(4, (0, 1, 0))],
                [Element(1, ElemKind.Cps3, [1, 2, 3]), Element(2, ElemKind.Cps3, [1, 3, 4])])
    m = steel_model(mesh)
    m.boundary_conditions = [BoundaryCondition([1, 4], [1]), BoundaryCondition([1], [2])]
    m.cloads = [ConcentratedLoad(2, 1, 5e5), ConcentratedLoad(3, 1, 5e5)]
    sol = solve_with_method(m, Method.Ldlt, ctx=ctx)
    assert np.all(np.abs(sol.von_mises - sigma) / sigma < 1e-6)
    assert abs(sol.displacements[2][1] + NU_STEEL * sigma / E_STEEL) / \
        (NU_STEEL * sigma / E_STEEL) < 1e-6

    m = steel_model(hex_mesh(1, 1, 1, 1.0, 1.0, 1.0))
    m.boundary_conditions = [BoundaryCondition([1, 2, 3, 4], [3]), BoundaryCondition([1], [1]),
                             BoundaryCondition([1, 2], [2])]
    m.cloads = [ConcentratedLoad(n, 3, sigma / 4) for n in (5, 6, 7, 8)]
    sol = solve_with_method(m, Method.Ldlt, ctx=ctx)
    assert np.all(np.abs(sol.von_mises - sigma) / sigma < 1e-6)
    rz = sum(r.value for r in sol.reactions if r.dof == 3)
    assert abs(rz + sigma) < 1e-6 * sigma


def test_failed_pivot_text_and_auto_on_a_dangling_node(ctx):
    """A node no element uses: the direct path fails with the reference's
    message at the reference's equation; Auto keeps the converged PCG."""
    m = dangling_model()
    k, f, _ = modified_system(m)
    with pytest.raises(InvalidModel) as want:
        oracle.ldlt(k, f)
    with pytest.raises(InvalidModel) as got:
        solve_with_method(m, Method.Ldlt, ctx=ctx)
    assert str(got.value) == str(want.value)
    assert "pivot near-zero at equation" in str(got.value)
    sol = solve(m, ctx=ctx)
    assert sol.solver_method == "pcg"


@pytest.mark.parametrize("name", ["cantilever", "cantilever3d", "plate_hole"])
def test_example_decks_through_the_direct_path(ctx, name):
    model, g = load_golden(name)
    sol = solve_with_method(model, Method.Ldlt, ctx=ctx)
    ref = direct_oracle(model)
    assert sol.solver_method == "ldlt" and sol.final_residual <= 1e-8
    assert rel(sol.u, ref.u) <= 1e-8
    assert fmt_mm(max_disp(sol.displacements)) == g["max_disp_mm"]
    assert fmt_mpa(sol.von_mises.max()) == g["max_von_mises_mpa"]


def test_flat_api_method_option(ctx):
    """svx_solve_flat with opts.method: a PCG budget of 7 iterations makes
    Auto fall back; the direct outputs are reported."""
    from solvix_b200 import workloads
    flat = workloads.cantilever_cps4(40, 4, length=2.0, height=0.1, jitter=0.0)
    sol = ctx.solve_flat(flat, max_iter=7, method=abi.SVX_METHOD_AUTO)
    assert sol.solver_method == "ldlt" and sol.iterations == 0
    ref = oracle.solve_flat(flat, method="ldlt")
    assert ref.solver_method == "ldlt"
    assert rel(sol.u, ref.u) <= 1e-8
    assert abs(sol.cond_estimate - ref.cond_estimate) <= 1e-6 * ref.cond_estimate


def test_band_wider_than_the_grid(ctx):
    """A band of more tiles than the substitution kernel has blocks (174
    tiles against one block per SM, 148 on a B200): every block takes
    several tiles of a block row.  The 24 x 36 x 36 hex cantilever (102,675
    DOF, RCM half-bandwidth 5,549 rows) is too large for the oracle's serial
    LDL^T, so the direct solution is checked against the device's FP64 PCG
    and by its own residual."""
    import torch

    from solvix_b200 import workloads
    flat = workloads.cantilever_c3d8(24, 36, 36)
    sol = ctx.solve_flat(flat, method=abi.SVX_METHOD_LDLT)
    assert sol.solver_method == "ldlt" and sol.iterations == 0
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert sol.factor_bandwidth == 5549 and (sol.factor_bandwidth + 31) // 32 > sms - 1
    assert sol.final_residual <= 1e-8
    pcg = ctx.solve_flat(flat)
    assert rel(sol.u, pcg.u) <= 1e-8
    assert np.max(np.abs(sol.von_mises - pcg.von_mises)) <= 1e-7 * np.max(np.abs(pcg.von_mises))
