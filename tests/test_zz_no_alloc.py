"""The allocation-free PCG entry point (svx_pcg_solve_noalloc) against the
allocating solve and the oracle, through the C ABI (GPU).

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

from oracle import oracle
from solvix_b200 import abi, workloads
from solvix_b200.core import Context

pytestmark = pytest.mark.gpu

U_TOL = 1e-10  # the plain FP64 displacement bar of the parity tests


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class _System:
    """The PCG operator of a small C3D8 cantilever as a device CSR, with the
    allocating solve's and the oracle's solutions of it."""

    def __init__(self, ctx):
        import torch

        flat = workloads.cantilever_c3d8(24, 6, 6, lx=1.2, ly=0.3, lz=0.3, seed=8)
        op = ctx.assemble(flat)
        try:
            rp, ci, vals = op.csr(which=0)   # the PCG operator (after Dirichlet)
            f, _ = op.vectors(which=0)
            self.u_ref, self.it_ref, _, _ = op.solve()
            self.n = op.n
        finally:
            op.free()
        self.u_oracle = oracle.solve_flat(flat).u
        dev = torch.device("cuda:0")
        self.rp = torch.from_numpy(rp.astype(np.int32)).to(dev)
        self.ci = torch.from_numpy(ci.astype(np.int32)).to(dev)
        self.vals = torch.from_numpy(vals).to(dev)
        self.f = torch.from_numpy(f).to(dev)
        self.dev = dev

    def solve(self, lib, tol=1e-10, max_iter=0, stream=None):
        import torch
        d_u = torch.full((self.n,), float("nan"), dtype=torch.float64, device=self.dev)
        it = C.c_int64(-1)
        res = C.c_double(-1.0)
        torch.cuda.synchronize()
        st = lib.svx_pcg_solve_noalloc(self.n, self.rp.data_ptr(), self.ci.data_ptr(),
                                       self.vals.data_ptr(), self.f.data_ptr(), tol, max_iter,
                                       d_u.data_ptr(), C.byref(it), C.byref(res), stream)
        return st, d_u.cpu().numpy(), it.value, res.value


def test_noalloc_pcg_matches_the_allocating_solve_on_two_calls():
    lib = abi.load()
    with Context(0) as ctx:
        sysm = _System(ctx)
    for _call in range(2):
        st, u, it, res = sysm.solve(lib)
        assert st == abi.SVX_OK
        assert rel(u, sysm.u_ref) <= U_TOL
        assert rel(u, sysm.u_oracle) <= U_TOL
        # same stopping rule; the reduction order differs from the allocating
        # path's, so the count is compared like the parity tests do
        assert abs(it - sysm.it_ref) <= max(3, sysm.it_ref // 10)
        assert res <= 1e-10


def test_noalloc_pcg_on_a_caller_stream_after_a_stopped_call():
    """A call stopped by max_iter leaves its iterate and scalars in the
    shared array; the next call on a caller's own stream still converges to
    the oracle's solution."""
    import torch

    lib = abi.load()
    with Context(0) as ctx:
        sysm = _System(ctx)
    st, _u, it, res = sysm.solve(lib, max_iter=3)
    assert st == abi.SVX_NOT_CONVERGED and it == 3 and res > 1e-10
    s = torch.cuda.Stream(device=sysm.dev)
    st, u, it, res = sysm.solve(lib, stream=C.c_void_p(s.cuda_stream))
    assert st == abi.SVX_OK and res <= 1e-10
    assert rel(u, sysm.u_oracle) <= U_TOL


def test_noalloc_pcg_refuses_bad_arguments_before_any_work():
    lib = abi.load()
    with Context(0) as ctx:
        sysm = _System(ctx)
    it = C.c_int64(-1)
    # a system larger than the static scratch
    st = lib.svx_pcg_solve_noalloc(abi.SVX_NOALLOC_MAX_DOF + 1, sysm.rp.data_ptr(),
                                   sysm.ci.data_ptr(), sysm.vals.data_ptr(), sysm.f.data_ptr(),
                                   1e-10, 0, sysm.f.data_ptr(), C.byref(it), None, None)
    assert st == abi.SVX_BAD_ARGUMENT and it.value == -1
    # a negative or NaN tolerance
    for tol in (-1.0, float("nan")):
        st, _u, it2, _r = sysm.solve(lib, tol=tol)
        assert st == abi.SVX_BAD_ARGUMENT and it2 == -1
