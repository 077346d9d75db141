"""Host-side API over the C ABI: contexts, operators and the solve entry
points that mirror solvix-core's ``solve`` / ``solve_with_method``
(crates/solvix-core/src/lib.rs:556-590).

Every compute call goes through ``libsolvix_b200.so``; when the library or
the CUDA device is unavailable the calls raise (there is no CPU path).
"""
from __future__ import annotations

import ctypes as C
import threading
import weakref
from typing import Optional

import numpy as np

from . import abi
from .marshal import FlatModel, ThermalModel, model_desc
from .model import (DeviceError, EmptyMesh, InvalidModel, Method, Model, NoConstraints,
                    NotConverged, Reaction, SolveError, Solution)


def _raise(status: int, err: abi.SvxError | None, what: str = ""):
    msg = err.message.decode(errors="replace") if err is not None else what
    if status == abi.SVX_INVALID_MODEL:
        raise InvalidModel(msg, reason=int(err.reason) if err is not None else 0,
                           elem_index=int(err.elem_index) if err is not None else -1)
    if status == abi.SVX_NOT_CONVERGED:
        raise NotConverged(int(err.iterations), float(err.residual))
    if status == abi.SVX_NO_CONSTRAINTS:
        raise NoConstraints("no constraints")
    if status == abi.SVX_EMPTY_MESH:
        raise EmptyMesh("empty mesh")
    if status == abi.SVX_BAD_ARGUMENT:
        raise ValueError(msg or "bad argument")
    raise DeviceError(msg or f"status {status}")


class Context:
    """One device context: a CUDA stream and a caching device allocator."""

    def __init__(self, device: int = 0):
        self.lib = abi.load()
        h = C.c_void_p()
        st = self.lib.svx_ctx_create(int(device), C.byref(h))
        if st != abi.SVX_OK:
            buf = C.create_string_buffer(512)
            self.lib.svx_last_error(None, buf, 512)
            raise DeviceError(buf.value.decode() or f"svx_ctx_create failed ({st})")
        self.handle = h
        self.device = device
        self._ops = weakref.WeakSet()

    @property
    def stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        return int(self.lib.svx_ctx_stream(self.handle) or 0)

    def close(self):
        """Free every live operator of this context, then the context."""
        if getattr(self, "handle", None):
            for op in list(getattr(self, "_ops", ())):
                op.free()
            self.lib.svx_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------
    def assemble(self, flat: FlatModel, keep_original: bool = False) -> "Operator":
        s = flat.as_struct()
        h = C.c_void_p()
        err = abi.SvxError()
        flags = abi.SVX_KEEP_ORIGINAL if keep_original else 0
        st = self.lib.svx_assemble(self.handle, C.byref(s), flags, C.byref(h), C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)
        op = Operator(self, h, flat)
        self._ops.add(op)
        return op

    def assemble_mass(self, flat: FlatModel, density: float) -> "Operator":
        """The consistent mass matrix of the flat model (svx_assemble_mass,
        modal.rs:203-271) as an operator: ``csr()`` exports it and
        ``spmv(x)`` returns M x."""
        s = flat.as_struct()
        h = C.c_void_p()
        err = abi.SvxError()
        st = self.lib.svx_assemble_mass(self.handle, C.byref(s), float(density), C.byref(h),
                                        C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)
        op = Operator(self, h, flat)
        self._ops.add(op)
        return op

    def solve_thermal(self, tm: ThermalModel, tol: float = 1e-10, max_iter: int = 0,
                      check_every: int = 0):
        """Steady conduction on the device (svx_solve_thermal_flat, the
        reference's heat::solve_thermal); returns (temperatures, iterations,
        residual) or raises the reference's SolveError."""
        t = np.zeros(tm.n_nodes)
        it = C.c_int64(0)
        res = C.c_double(0.0)
        err = abi.SvxError()
        opts = abi.default_opts(tol=tol, max_iter=max_iter, check_every=check_every)
        s = tm.as_struct()
        st = self.lib.svx_solve_thermal_flat(self.handle, C.byref(s), C.byref(opts),
                                             abi.ptr(t, C.c_double), C.byref(it), C.byref(res),
                                             C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)
        return t, int(it.value), float(res.value)

    def solve_flat(self, flat: FlatModel, tol: float = 1e-10, max_iter: int = 0,
                   precision: int = abi.SVX_FP64, inner_tol: float = 1e-5,
                   want_stress: bool = True, check_every: int = 0,
                   method: int = abi.SVX_METHOD_PCG) -> Solution:
        """method: abi.SVX_METHOD_PCG (default), SVX_METHOD_LDLT (the direct
        path on the device) or SVX_METHOD_AUTO (PCG, then the direct path
        when it does not converge), lib.rs:664-686."""
        out = _SolutionBuffers(flat.n_nodes, flat.ndof, flat.n_elem, flat.fixed_row.shape[0])
        opts = abi.default_opts(tol=tol, max_iter=max_iter, precision=precision,
                                inner_tol=inner_tol, want_stress=int(want_stress),
                                check_every=check_every, method=int(method))
        err = abi.SvxError()
        s = flat.as_struct()
        st = self.lib.svx_solve_flat(self.handle, C.byref(s), C.byref(opts),
                                     C.byref(out.struct), C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)
        return out.solution(flat, precision)

    def solve_batch(self, flats, tol: float = 1e-10, max_iter: int = 0, want_u: bool = True,
                    want_stress: bool = True, precision: int = abi.SVX_FP64):
        """Solve many independent FlatModels (equal ndof) in one batched launch.

        Returns (list of per-model dicts with u / von_mises / iterations /
        residual / converged / status / cond_estimate / nnz, stats dict).
        A model rejected on its own (bad element, no constraints, ...) has
        ``status`` set to that error code and does not affect the others.
        """
        flats = list(flats)
        count = len(flats)
        raw = (abi.SvxFlatModelRaw * count)(*[f.raw_fields() for f in flats])
        structs = C.cast(raw, C.POINTER(abi.SvxFlatModel))
        us = [np.zeros(f.n_dof) if want_u else None for f in flats]
        vms = [np.zeros(f.n_elem) if want_stress else None for f in flats]
        u_ptrs = (abi.c_double_p * count)(*[abi.ptr(a, C.c_double) for a in us])
        vm_ptrs = (abi.c_double_p * count)(*[abi.ptr(a, C.c_double) for a in vms])
        results = (abi.SvxBatchResult * count)()
        stats = abi.SvxBatchStats()
        opts = abi.default_opts(tol=tol, max_iter=max_iter, want_stress=int(want_stress),
                                precision=precision)
        err = abi.SvxError()
        st = self.lib.svx_batch_solve(self.handle, count, structs, C.byref(opts),
                                      u_ptrs if want_u else None,
                                      vm_ptrs if want_stress else None, results,
                                      C.byref(stats), C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)
        out = [{"u": us[k], "von_mises": vms[k], "iterations": int(results[k].iterations),
                "residual": float(results[k].residual),
                "converged": results[k].status == abi.SVX_OK,
                "status": int(results[k].status), "reason": int(results[k].reason),
                "elem_index": int(results[k].elem_index),
                "cond_estimate": float(results[k].cond_estimate),
                "nnz": int(results[k].nnz)} for k in range(count)]
        st_d = {name: getattr(stats, name) for name, _ in abi.SvxBatchStats._fields_}
        return out, st_d

    def solve_model(self, model: Model, tol: float = 1e-10, precision: int = abi.SVX_FP64,
                    inner_tol: float = 1e-5, method: int = abi.SVX_METHOD_AUTO) -> Solution:
        """The reference-shaped path: resolve ids / sets on the host (C++),
        then assemble, solve and recover stresses on the device."""
        desc, keep = model_desc(model)
        res = C.c_void_p()
        err = abi.SvxError()
        st = self.lib.svx_resolve(C.byref(desc), C.byref(res), C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)
        try:
            flat_s = self.lib.svx_resolved_flat(res).contents
            n_nodes, ndof = int(flat_s.n_nodes), int(flat_s.ndof)
            out = _SolutionBuffers(n_nodes, ndof, int(flat_s.n_elem), int(flat_s.n_fixed))
            opts = abi.default_opts(tol=tol, precision=precision, inner_tol=inner_tol,
                                    method=int(method))
            st = self.lib.svx_solve_resolved(self.handle, res, C.byref(opts),
                                             C.byref(out.struct), C.byref(err))
            if st != abi.SVX_OK:
                _raise(st, err)
            rows = np.ctypeslib.as_array(flat_s.fixed_row, shape=(int(flat_s.n_fixed),)).copy() \
                if flat_s.n_fixed else np.zeros(0, np.int64)
            node_ids = np.ctypeslib.as_array(flat_s.node_id, shape=(n_nodes,)).copy()
        finally:
            self.lib.svx_resolved_free(res)
        return out.solution_from(rows, node_ids, ndof, precision)


class _SolutionBuffers:
    def __init__(self, n_nodes, ndof, n_elem, n_fixed):
        self.u = np.zeros(n_nodes * ndof)
        self.disp = np.zeros((n_nodes, 3))
        self.vm = np.zeros(n_elem)
        self.vm_node = np.zeros(n_nodes)
        self.react = np.zeros(n_fixed)
        s = abi.SvxSolution()
        s.u = abi.ptr(self.u, C.c_double)
        s.displacements = abi.ptr(self.disp, C.c_double)
        s.von_mises = abi.ptr(self.vm, C.c_double)
        s.nodal_von_mises = abi.ptr(self.vm_node, C.c_double)
        s.reactions = abi.ptr(self.react, C.c_double)
        self.struct = s

    def solution_from(self, rows, node_ids, ndof, precision) -> Solution:
        s = self.struct
        reactions = [Reaction(int(node_ids[r // ndof]), int(r % ndof) + 1, float(v))
                     for r, v in zip(rows.tolist(), self.react.tolist())] \
            if rows.shape[0] <= 200000 else []
        return Solution(
            displacements=self.disp, von_mises=self.vm, nodal_von_mises=self.vm_node,
            reactions=reactions, iterations=int(s.iterations),
            final_residual=float(s.final_residual),
            solver_method="ldlt" if s.solver_method == abi.SVX_METHOD_LDLT else
            "pcg" if precision == abi.SVX_FP64 else
            "pcg-mixed" if precision == abi.SVX_MIXED else "pcg-defect",
            cond_estimate=float(s.cond_estimate), u=self.u, reaction_values=self.react,
            outer_iterations=int(s.outer_iterations), ms_assemble=float(s.ms_assemble),
            ms_solve=float(s.ms_solve), ms_stress=float(s.ms_stress),
            factor_bandwidth=int(s.factor_bandwidth), ms_factor=float(s.ms_factor),
            fp32_iterations=int(s.fp32_iterations))

    def solution(self, flat: FlatModel, precision) -> Solution:
        node_ids = flat.node_id if flat.node_id is not None else \
            np.arange(1, flat.n_nodes + 1, dtype=np.uint32)
        return self.solution_from(flat.fixed_row, node_ids, flat.ndof, precision)


class Operator:
    """An assembled system resident on the device (svx_op_t)."""

    def __init__(self, ctx: Context, handle, flat: FlatModel):
        self.ctx = ctx
        self.lib = ctx.lib
        self.handle = handle
        self.flat = flat
        n = C.c_int64()
        nnz = C.c_int64()
        self.lib.svx_op_dims(handle, C.byref(n), C.byref(nnz))
        self.n, self.nnz = int(n.value), int(nnz.value)
        # iteration split of the last solve: FP32-operator iterations and
        # outer steps (corrections or true-residual checks)
        self.last_fp32_iterations = 0
        self.last_outer_iterations = 0

    def free(self):
        if getattr(self, "handle", None):
            if getattr(self.ctx, "handle", None):
                self.lib.svx_op_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def csr(self, which: int = 0):
        rp = np.zeros(self.n + 1, dtype=np.int64)
        ci = np.zeros(self.nnz, dtype=np.int32)
        v = np.zeros(self.nnz)
        st = self.lib.svx_op_get_csr(self.handle, int(which), abi.ptr(rp, C.c_int64),
                                     abi.ptr(ci, C.c_int32), abi.ptr(v, C.c_double))
        if st != abi.SVX_OK:
            _raise(st, None, "svx_op_get_csr failed")
        return rp, ci, v

    def vectors(self, which: int = 0):
        f = np.zeros(self.n)
        d = np.zeros(self.n)
        st = self.lib.svx_op_get_vectors(self.handle, int(which), abi.ptr(f, C.c_double),
                                         abi.ptr(d, C.c_double))
        if st != abi.SVX_OK:
            _raise(st, None, "svx_op_get_vectors failed")
        return f, d

    def spmv(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.n)
        st = self.lib.svx_op_spmv(self.handle, abi.ptr(x, C.c_double), abi.ptr(y, C.c_double))
        if st != abi.SVX_OK:
            _raise(st, None, "svx_op_spmv failed")
        return y

    def set_solution(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        st = self.lib.svx_op_set_solution(self.handle, abi.ptr(u, C.c_double))
        if st != abi.SVX_OK:
            _raise(st, None, "svx_op_set_solution failed")

    def time_kernels(self, reps: int = 50):
        """(FP64 spmv_node_dot, update, p_update, FP32 difference-form
        spmv_node_dot) average device ms per launch."""
        ms = np.zeros(4)
        st = self.lib.svx_op_time_kernels(self.handle, int(reps), abi.ptr(ms, C.c_double))
        if st != abi.SVX_OK:
            _raise(st, None, "svx_op_time_kernels failed")
        return ms

    def reassemble(self):
        """Re-run K1-K4 from the device-resident model (no host traffic)."""
        err = abi.SvxError()
        st = self.lib.svx_op_reassemble(self.handle, C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)

    def solve_device(self, tol=1e-10, max_iter=0, precision=abi.SVX_FP64, inner_tol=1e-5,
                     want_stress=True, check_every=0):
        """Solve (and recover stresses) leaving every result on the device;
        returns (iterations, residual, ms_solve, ms_stress, ms_assemble) with
        ms_assemble the device time of the operator's last assembly."""
        sol = abi.SvxSolution()
        opts = abi.default_opts(tol=tol, max_iter=max_iter, precision=precision,
                                inner_tol=inner_tol, check_every=check_every,
                                want_stress=int(want_stress))
        err = abi.SvxError()
        st = self.lib.svx_op_solve(self.handle, C.byref(opts), C.byref(sol), C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)
        self.last_fp32_iterations = int(sol.fp32_iterations)
        self.last_outer_iterations = int(sol.outer_iterations)
        return int(sol.iterations), float(sol.final_residual), float(sol.ms_solve), \
            float(sol.ms_stress), float(sol.ms_assemble)

    def solve(self, tol=1e-10, max_iter=0, precision=abi.SVX_FP64, inner_tol=1e-5,
              check_every=0, method=abi.SVX_METHOD_PCG):
        u = np.zeros(self.n)
        sol = abi.SvxSolution()
        sol.u = abi.ptr(u, C.c_double)
        opts = abi.default_opts(tol=tol, max_iter=max_iter, precision=precision,
                                inner_tol=inner_tol, check_every=check_every, want_stress=0,
                                method=int(method))
        err = abi.SvxError()
        st = self.lib.svx_op_solve(self.handle, C.byref(opts), C.byref(sol), C.byref(err))
        if st != abi.SVX_OK:
            _raise(st, err)
        self.last_fp32_iterations = int(sol.fp32_iterations)
        self.last_outer_iterations = int(sol.outer_iterations)
        return u, int(sol.iterations), float(sol.final_residual), float(sol.cond_estimate)

    def stress(self):
        fl = self.flat
        out = _SolutionBuffers(fl.n_nodes, fl.ndof, fl.n_elem, fl.fixed_row.shape[0])
        st = self.lib.svx_op_stress(self.handle, C.byref(out.struct))
        if st != abi.SVX_OK:
            _raise(st, None, "svx_op_stress failed")
        return out.vm, out.vm_node, out.react, out.disp


_default = {}
_default_lock = threading.Lock()


def default_context(device: int = 0) -> Context:
    with _default_lock:
        ctx = _default.get(device)
        if ctx is None:
            ctx = Context(device)
            _default[device] = ctx
        return ctx


def solve_with_method(model: Model, method: Method = Method.Auto,
                      ctx: Optional[Context] = None) -> Solution:
    """Linear-static solve of a reference-shaped model on the GPU
    (lib.rs:586-716): ``Method.Pcg`` runs the FP64 Jacobi-PCG and surfaces a
    budget overrun as ``NotConverged``; ``Method.Ldlt`` runs the direct path
    (RCM-ordered band LDLT on the device); ``Method.Auto`` runs the PCG and
    falls back to the direct path when it does not converge."""
    code = {Method.Auto: abi.SVX_METHOD_AUTO, Method.Pcg: abi.SVX_METHOD_PCG,
            Method.Ldlt: abi.SVX_METHOD_LDLT}[method]
    return (ctx or default_context()).solve_model(model, method=code)


def solve(model: Model, ctx: Optional[Context] = None) -> Solution:
    """solvix_core::solve for linear-static models (lib.rs:556-581)."""
    if model.steps and model.steps[-1].nlgeom:
        raise InvalidModel("NLGEOM steps are outside the linear-static GPU path")
    return solve_with_method(model, Method.Auto, ctx)
