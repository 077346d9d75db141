"""The allocation-free PCG entry point (svx_pcg_solve_noalloc) against the
allocating solve, through the C ABI (GPU).

svx_pcg_solve_noalloc serves callers that cannot let a library allocate
device memory (an application owning the device-memory budget through its
own arena, or a latency-bounded loop that cannot absorb cudaMalloc's
synchronisation).  It takes a device-resident CSR system and keeps its work
vectors in one static device array, so two calls in a row must both
reproduce the allocating path's result even though the second call starts
from the first call's leftover scratch contents.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from solvix_b200 import abi, workloads
from solvix_b200.core import Context

pytestmark = pytest.mark.gpu

U_TOL = 1e-10  # the plain FP64 displacement bar of the parity tests


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_pcg_matches_the_allocating_solve_on_two_calls():
    import torch

    lib = abi.load()
    ctx = Context(0)
    op = None
    try:
        flat = workloads.cantilever_c3d8(24, 6, 6, lx=1.2, ly=0.3, lz=0.3, seed=8)
        op = ctx.assemble(flat)
        rp, ci, vals = op.csr(which=0)       # the PCG operator (after Dirichlet)
        f, _ = op.vectors(which=0)
        u_ref, it_ref, res_ref, _ = op.solve()
        dev = torch.device("cuda:0")
        d_rp = torch.from_numpy(rp.astype(np.int32)).to(dev)
        d_ci = torch.from_numpy(ci.astype(np.int32)).to(dev)
        d_vals = torch.from_numpy(vals).to(dev)
        d_f = torch.from_numpy(f).to(dev)
        for _call in range(2):
            d_u = torch.full((op.n,), float("nan"), dtype=torch.float64, device=dev)
            it = C.c_int64(-1)
            res = C.c_double(-1.0)
            torch.cuda.synchronize()
            st = lib.svx_pcg_solve_noalloc(op.n, d_rp.data_ptr(), d_ci.data_ptr(),
                                           d_vals.data_ptr(), d_f.data_ptr(), 1e-10, 0,
                                           d_u.data_ptr(), C.byref(it), C.byref(res), None)
            assert st == abi.SVX_OK
            u = d_u.cpu().numpy()
            assert rel(u, u_ref) <= U_TOL
            # same stopping rule; the reduction order may differ from the
            # allocating path's, so the count is compared like the parity tests
            assert abs(it.value - it_ref) <= max(3, it_ref // 10)
            assert res.value <= 1e-10
        # a system larger than the static scratch is refused before any work
        it = C.c_int64(-1)
        st = lib.svx_pcg_solve_noalloc(abi.SVX_NOALLOC_MAX_DOF + 1, d_rp.data_ptr(),
                                       d_ci.data_ptr(), d_vals.data_ptr(), d_f.data_ptr(), 1e-10,
                                       0, d_u.data_ptr(), C.byref(it), None, None)
        assert st == abi.SVX_BAD_ARGUMENT and it.value == -1
    finally:
        if op is not None:
            op.free()
        ctx.close()
