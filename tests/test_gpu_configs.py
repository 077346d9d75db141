"""Parity at the sizes the path's bars are quoted on, through the C ABI (GPU).

The plain form's bar is the reference's FP64 CPU path on the same model to
a relative displacement error of 1e-10, with the von Mises field matched;
the mixed and batched forms' bar is 1e-8.  The small-case parity tests
(test_gpu_parity.py) prove it on models of a few thousand DOF; these tests
prove it on the configurations themselves:

* the 200 x 20 CPS4 cantilever (8,442 DOF, jittered, t = 0.01 m);
* the 160 x 16 x 16 C3D8 cantilever (139,587 DOF, 10.4M nonzeros);
* the 4,096-plate mix (CPS4 / CPS3, nx 10..160, ny 4..40) solved as one
  batch in FP64 and mixed, 64 seeded members checked against the oracle;
* the heterogeneous C3D8 model (per-element E over 1e9..1e11) on the
  CUDA-graph iteration form that the 480 x 48 x 48 model runs on, at
  160 x 16 x 16 where the oracle solves it in seconds, FP64 and mixed.

Both solvers stop at ||r|| / ||f|| <= 1e-10 and sum their dot products in
different orders, so their iteration counts differ by a few percent; at
this tolerance each solution is within ~1e-12 of the converged one (the
oracle's own solution at 1e-10 is 3e-13 from its 1e-14 solution on the
160 x 16 x 16 cantilever), so the 1e-10 bar holds with margin.
"""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import Context, abi, workloads

pytestmark = pytest.mark.gpu

U_TOL = 1e-10      # plain FP64 against the oracle
MIXED_TOL = 1e-8   # mixed and batched forms
VM_TOL = 1e-8      # von Mises fields, relative to their maximum


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def vm_rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _check_plain(sol, ref, it_slack=0.1):
    assert rel(sol.u, ref.u) <= U_TOL
    assert vm_rel(sol.von_mises, ref.von_mises) <= VM_TOL
    assert vm_rel(sol.nodal_von_mises, ref.nodal_von_mises) <= VM_TOL
    assert np.max(np.abs(sol.reaction_values - ref.reaction_values)) <= \
        1e-8 * max(1.0, np.max(np.abs(ref.reaction_values)))
    assert sol.cond_estimate == pytest.approx(ref.cond_estimate, rel=1e-14)
    assert sol.final_residual <= 1e-10
    assert abs(sol.iterations - ref.iterations) <= max(3, int(it_slack * ref.iterations))


def test_cps4_cantilever_200x20_matches_oracle(ctx):
    flat = workloads.cantilever_cps4()
    assert flat.n_dof == 8442 and flat.n_elem == 4000
    sol = ctx.solve_flat(flat)
    ref = oracle.solve_flat(flat)
    _check_plain(sol, ref)
    # the tip load of -1000 N in y is carried by the clamped edge
    ry = sol.reaction_values[flat.fixed_row % 2 == 1].sum()
    assert abs(ry - 1000.0) <= 1e-6 * 1000.0


def test_c3d8_cantilever_160x16x16_matches_oracle(ctx):
    flat = workloads.cantilever_c3d8(160, 16, 16)
    assert flat.n_dof == 139587
    sol = ctx.solve_flat(flat)
    ref = oracle.solve_flat(flat)
    _check_plain(sol, ref)
    rz = sol.reaction_values[flat.fixed_row % 3 == 2].sum()
    assert abs(rz - 5000.0) <= 1e-6 * 5000.0


@pytest.fixture(scope="module")
def plate_mix():
    flats = workloads.plate_batch(4096, seed=4)
    rng = np.random.default_rng(2024)
    sample = sorted(int(k) for k in rng.choice(len(flats), 64, replace=False))
    # the sample reaches both element kinds and the mix's size range
    kinds = {int(flats[k].kind[0]) for k in sample}
    assert kinds == {abi.SVX_CPS3, abi.SVX_CPS4}
    refs = {k: oracle.solve_flat(flats[k]) for k in sample}
    return flats, sample, refs


@pytest.mark.parametrize("precision,tol", [(abi.SVX_FP64, U_TOL), (abi.SVX_MIXED, MIXED_TOL)])
def test_plate_mix_4096_batched_matches_oracle(ctx, plate_mix, precision, tol):
    flats, sample, refs = plate_mix
    out, st = ctx.solve_batch(flats, precision=precision)
    assert st["not_converged"] == 0
    assert all(o["status"] == abi.SVX_OK for o in out)
    for k in sample:
        ref = refs[k]
        assert rel(out[k]["u"], ref.u) <= tol, k
        assert vm_rel(out[k]["von_mises"], ref.von_mises) <= (VM_TOL if tol == U_TOL else 1e-7)
        assert out[k]["cond_estimate"] == pytest.approx(ref.cond_estimate, rel=1e-14)
        if precision == abi.SVX_FP64:
            assert abs(out[k]["iterations"] - ref.iterations) <= max(3, ref.iterations // 10)


@pytest.fixture(scope="module")
def hetero_160():
    flat = workloads.heterogeneous_c3d8(160, 16, 16, seed=3)
    return flat, oracle.solve_flat(flat)


@pytest.fixture(scope="module")
def graph_ctx():
    """A context whose solves iterate in the CUDA-graph form at any size
    (SVX_GRAPH_MIN_NNZ=0 when the context is created)."""
    import os
    old = os.environ.get("SVX_GRAPH_MIN_NNZ")
    os.environ["SVX_GRAPH_MIN_NNZ"] = "0"
    try:
        c = Context(0)
    finally:
        if old is None:
            del os.environ["SVX_GRAPH_MIN_NNZ"]
        else:
            os.environ["SVX_GRAPH_MIN_NNZ"] = old
    yield c
    c.close()


def test_heterogeneous_c3d8_graph_form_fp64_matches_oracle(graph_ctx, hetero_160):
    flat, ref = hetero_160
    sol = graph_ctx.solve_flat(flat)
    # on a 100x-contrast model CG's iteration count is more sensitive to
    # the order of its dot-product sums than on the uniform cantilevers
    _check_plain(sol, ref, it_slack=0.25)


def test_heterogeneous_c3d8_graph_form_mixed_matches_oracle(graph_ctx, hetero_160):
    flat, ref = hetero_160
    sol = graph_ctx.solve_flat(flat, precision=abi.SVX_MIXED)
    assert sol.solver_method == "pcg-mixed"
    assert rel(sol.u, ref.u) <= MIXED_TOL
    assert vm_rel(sol.von_mises, ref.von_mises) <= 1e-7
    assert sol.final_residual <= 1e-10


def test_heterogeneous_c3d8_defect_correction_matches_oracle(graph_ctx, hetero_160):
    """FP32 inner PCG (FP32 K, vectors, preconditioner; FP64 dots) to 1e-5
    inside FP64 defect correction, on the graph form."""
    flat, ref = hetero_160
    sol = graph_ctx.solve_flat(flat, precision=abi.SVX_MIXED_DEFECT)
    assert sol.solver_method == "pcg-defect"
    assert sol.final_residual <= 1e-10
    assert sol.outer_iterations >= 2
    assert 0 < sol.fp32_iterations <= sol.iterations
    assert rel(sol.u, ref.u) <= MIXED_TOL
    assert vm_rel(sol.von_mises, ref.von_mises) <= 1e-7


def test_heterogeneous_c3d8_persistent_form_matches_oracle(ctx, hetero_160):
    flat, ref = hetero_160
    sol = ctx.solve_flat(flat)
    _check_plain(sol, ref, it_slack=0.25)
    mixed = ctx.solve_flat(flat, precision=abi.SVX_MIXED)
    assert rel(mixed.u, ref.u) <= MIXED_TOL
