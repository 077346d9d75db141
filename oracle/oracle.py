"""CPU oracle bindings (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/libsvx_oracle.so`` (the C++ restatement of the reference's
element / assembly / solver / stress arithmetic) and restates the reference's
host-side model handling in plain Python:

* ``Model::load_state``            crates/solvix-core/src/lib.rs:388-403
* ``solve_with_thermal`` checks    lib.rs:596-612 (NoConstraints, validate, thickness)
* ``Model::validate``              lib.rs:406-436
* ``ndof_per_node``                lib.rs:725-752
* ``Mesh::node_index``             lib.rs:106-108 (first node with the id)
* ``Model::material_for_element``  lib.rs:357-367
* CLOAD loop of ``assemble_with``  crates/solvix-core/src/assembly.rs:365-380
* ``edge_pressure_forces``         assembly.rs:382, :393-452
* ``gravity_forces``               assembly.rs:383, :458-539 (plane kinds)
* ``constrained_dofs``             crates/solvix-core/src/solver.rs:15-41

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from solvix_b200 import abi  # noqa: E402  (struct layouts only)
from solvix_b200.marshal import FlatModel, ThermalModel  # noqa: E402
from solvix_b200.model import (ElemKind, EmptyMesh, InvalidModel, Model,  # noqa: E402
                               NoConstraints, NotConverged, SolveError)

LIB_PATH = os.path.join(HERE, "libsvx_oracle.so")


class OracleCsr(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("nnz", C.c_int64),
        ("row_ptr", abi.c_int64_p),
        ("col_idx", abi.c_int64_p),
        ("vals", abi.c_double_p),
        ("f", abi.c_double_p),
    ]


_SIG = {
    "svx_oracle_set_sort_mode": (None, [C.c_int]),
    "svx_oracle_element_stiffness": (C.c_int, [C.c_int, abi.c_double_p, C.c_double, C.c_double,
                                               C.c_double, abi.c_double_p]),
    "svx_oracle_assemble": (C.c_int, [C.POINTER(abi.SvxFlatModel), C.c_int,
                                      C.POINTER(OracleCsr), C.POINTER(abi.SvxError)]),
    "svx_oracle_csr_free": (None, [C.POINTER(OracleCsr)]),
    "svx_oracle_spmv": (None, [C.POINTER(OracleCsr), abi.c_double_p, abi.c_double_p, C.c_int]),
    "svx_oracle_apply_dirichlet": (None, [C.POINTER(OracleCsr), abi.c_double_p, abi.c_int64_p,
                                          C.c_int64]),
    "svx_oracle_pcg": (C.c_int, [C.POINTER(OracleCsr), abi.c_double_p, C.c_double, C.c_int64,
                                 C.c_int, abi.c_double_p, abi.c_int64_p, abi.c_double_p]),
    "svx_oracle_solve": (C.c_int, [C.POINTER(abi.SvxFlatModel), C.c_int, C.c_double, C.c_int64,
                                   C.POINTER(abi.SvxSolution), C.POINTER(abi.SvxError)]),
    "svx_oracle_solve_method": (C.c_int, [C.POINTER(abi.SvxFlatModel), C.c_int, C.c_double,
                                          C.c_int64, C.c_int, C.POINTER(abi.SvxSolution),
                                          C.POINTER(C.c_int), C.POINTER(abi.SvxError)]),
    "svx_oracle_rcm": (None, [C.POINTER(OracleCsr), abi.c_int64_p]),
    "svx_oracle_element_mass": (C.c_int, [C.c_int, abi.c_double_p, C.c_double, C.c_double,
                                          abi.c_double_p]),
    "svx_oracle_assemble_mass": (C.c_int, [C.POINTER(abi.SvxFlatModel), C.c_double,
                                           C.POINTER(OracleCsr), C.POINTER(abi.SvxError)]),
    "svx_oracle_ldlt": (C.c_int, [C.POINTER(OracleCsr), abi.c_double_p, C.c_int, abi.c_double_p,
                                  abi.c_double_p, abi.c_double_p, abi.c_double_p, abi.c_int64_p,
                                  C.POINTER(abi.SvxError)]),
    "svx_oracle_stress": (C.c_int, [C.POINTER(abi.SvxFlatModel), abi.c_double_p, C.c_int,
                                    abi.c_double_p, abi.c_double_p, abi.c_double_p,
                                    C.POINTER(abi.SvxError)]),
    "svx_oracle_solve_thermal": (C.c_int, [C.POINTER(abi.SvxThermalModel), C.c_int,
                                           C.c_double, abi.c_double_p, abi.c_int64_p,
                                           abi.c_double_p, C.POINTER(abi.SvxError)]),
    "svx_oracle_conduction_element": (C.c_int, [C.c_int, abi.c_double_p, C.c_double,
                                                C.c_double, C.c_int, C.c_double,
                                                abi.c_double_p, abi.c_double_p]),
}

_lib = None


def build(force: bool = False) -> str:
    """Compile libsvx_oracle.so with the Makefile beside this file."""
    src = os.path.join(HERE, "svx_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "libsvx_oracle.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = abi.bind(C.CDLL(LIB_PATH), _SIG)
    return _lib


def set_sort_mode(mode: int) -> None:
    """0: the reference's unstable row sort (default); 1: stable, the
    triplet-stream order the CUDA assembly sums in."""
    lib().svx_oracle_set_sort_mode(int(mode))


def default_threads() -> int:
    """min(8, cores), the reference's worker_threads (assembly.rs:17-21)."""
    return max(1, min(8, os.cpu_count() or 1))


# ----------------------------------------------------------------- host logic
class Pending:
    """An error the reference raises after the element loop (CLOAD, BC)."""

    def __init__(self, err: SolveError):
        self.err = err


def ndof_per_node(kinds) -> int:
    """lib.rs:725-752."""
    ks = set(int(k) for k in np.unique(np.asarray(kinds)))
    plane = bool(ks & {0, 1, 2, 3, 4})
    solid = bool(ks & {5, 6})
    beam = 7 in ks
    if beam and (plane or solid):
        raise InvalidModel("mixed beam and continuum elements (v1: B31-only models)")
    if beam:
        return 3
    if plane and solid:
        raise InvalidModel("mixed dimensionality")
    return 3 if solid else 2


_KIND_DEBUG = {ElemKind.Cps3: "Cps3", ElemKind.Cps4: "Cps4", ElemKind.Cps8: "Cps8",
               ElemKind.Cpe4: "Cpe4", ElemKind.Cpe8: "Cpe8", ElemKind.C3d8: "C3d8",
               ElemKind.C3d4: "C3d4", ElemKind.B31: "B31"}


def _edge_pressure(model, dloads, first_index, ndof, f):
    """edge_pressure_forces (assembly.rs:393-452): pressure * thickness *
    edge length, half to each end node, along the inward normal."""
    mesh = model.mesh
    ids = mesh.elem_ids.tolist()
    for dl in dloads:
        try:
            e = ids.index(int(dl.element_id))
        except ValueError:
            return Pending(InvalidModel(f"distributed load on unknown element {dl.element_id}"))
        kind = ElemKind(int(mesh.elem_kinds[e]))
        if kind == ElemKind.Cps3:
            max_face = 3
        elif kind in (ElemKind.Cps4, ElemKind.Cpe4):
            max_face = 4
        else:
            return Pending(InvalidModel(
                f"edge pressure on element {dl.element_id} ({_KIND_DEBUG[kind]}) unsupported "
                "(linear quad/tri edges only)"))
        if dl.face == 0 or dl.face > max_face:
            return Pending(InvalidModel(
                f"element {dl.element_id} ({_KIND_DEBUG[kind]}) has no face {dl.face}"))
        a = int(mesh.conn_ptr[e])
        nn = int(mesh.conn_ptr[e + 1]) - a
        ia = first_index[int(mesh.conn[a + dl.face - 1])]
        ib = first_index[int(mesh.conn[a + dl.face % nn])]
        pa = (float(mesh.coords[ia][0]), float(mesh.coords[ia][1]))
        pb = (float(mesh.coords[ib][0]), float(mesh.coords[ib][1]))
        d = (pb[0] - pa[0], pb[1] - pa[1])
        length = math.sqrt(d[0] * d[0] + d[1] * d[1])
        if length == 0.0:
            return Pending(InvalidModel(f"zero-length pressure edge on element {dl.element_id}"))
        n_in = (-d[1] / length, d[0] / length)
        fmag = float(dl.magnitude) * float(model.thickness) * length / 2.0
        for i in (ia, ib):
            f[i * ndof] += fmag * n_in[0]
            f[i * ndof + 1] += fmag * n_in[1]
    return None


def _gravity(model, gravity, first_index, ndof, f):
    """gravity_forces (assembly.rs:458-539) for CPS3 (thirds) and CPS4 /
    CPE4 (quarters); solids are rejected; the kinds the device path does
    not assemble (CPS8, CPE8, B31) are left out, their element error wins."""
    if gravity is None:
        return None
    g, direction = float(gravity[0]), gravity[1]
    dir2 = (float(direction[0]), float(direction[1]))
    if dir2 == (0.0, 0.0):
        return Pending(InvalidModel("gravity direction has no in-plane component"))
    mesh = model.mesh
    rho, t = float(model.density), float(model.thickness)
    for e in range(mesh.n_elements):
        kind = ElemKind(int(mesh.elem_kinds[e]))
        a, b = int(mesh.conn_ptr[e]), int(mesh.conn_ptr[e + 1])
        idx = [first_index[int(nid)] for nid in mesh.conn[a:b].tolist()]
        p = [(float(mesh.coords[i][0]), float(mesh.coords[i][1])) for i in idx]
        if kind == ElemKind.Cps3:
            cross = (p[1][0] - p[0][0]) * (p[2][1] - p[0][1]) - \
                (p[1][1] - p[0][1]) * (p[2][0] - p[0][0])
            per = [rho * t * abs(cross) / 2.0 * g / 3.0] * 3
        elif kind in (ElemKind.Cps4, ElemKind.Cpe4):
            shoelace = 0.0
            for k in range(4):
                pa, pb = p[k], p[(k + 1) % 4]
                shoelace += pa[0] * pb[1] - pb[0] * pa[1]
            per = [rho * t * abs(shoelace) / 2.0 * g / 4.0] * 4
        elif kind in (ElemKind.C3d8, ElemKind.C3d4):
            return Pending(InvalidModel(
                "gravity on solid elements unsupported (plane and beam only)"))
        else:
            continue
        for i, w in zip(idx, per):
            f[i * ndof] += w * dir2[0]
            f[i * ndof + 1] += w * dir2[1]
    return None


def resolve(model: Model):
    """Reference-shaped model -> (FlatModel, pending error or None).

    Raises the SolveError the reference raises before assembly.
    """
    bcs, cloads, dloads, gravity = model.load_state()
    mesh = model.mesh
    if len(bcs) == 0:
        raise NoConstraints("no constraints")
    # validate (lib.rs:406-436), mapped to InvalidModel("{:?}")
    if mesh.n_nodes == 0 or mesh.n_elements == 0:
        raise InvalidModel("EmptyMesh")
    if len(model.materials) == 0:
        raise InvalidModel("NoMaterial")
    first_index = {}
    for i, nid in enumerate(mesh.node_ids.tolist()):
        first_index.setdefault(nid, i)
    kinds = mesh.elem_kinds
    conn_ids = mesh.conn.tolist()
    for e in range(mesh.n_elements):
        a, b = int(mesh.conn_ptr[e]), int(mesh.conn_ptr[e + 1])
        if b - a != ElemKind(int(kinds[e])).node_count():
            raise InvalidModel(f"MalformedElement({int(mesh.elem_ids[e])})")
        for nid in conn_ids[a:b]:
            if nid not in first_index:
                raise InvalidModel(f"UnknownNode({nid})")
    t = float(model.thickness)
    if t <= 0.0 or t != t:
        raise InvalidModel("thickness must be positive")
    ndof = ndof_per_node(kinds)
    conn = np.array([first_index[nid] for nid in conn_ids], dtype=np.int32)
    # material_for_element (lib.rs:357-367)
    set_by_name = {}
    for s in model.elsets:
        set_by_name.setdefault(s.name, s)
    mat_by_name = {}
    for m in model.materials:
        mat_by_name.setdefault(m.name, m)
    decided = {}
    for set_name, mat_name in model.mat_assignments:
        s = set_by_name.get(set_name)
        if s is None:
            continue
        for eid in np.asarray(s.element_ids).tolist():
            if eid not in decided:
                decided[eid] = mat_by_name.get(mat_name)
    n_elem = mesh.n_elements
    E = np.zeros(n_elem)
    nu = np.zeros(n_elem)
    nomat = np.zeros(n_elem, dtype=np.uint8)
    for e, eid in enumerate(mesh.elem_ids.tolist()):
        m = decided.get(eid)
        if m is None:
            nomat[e] = 1
        else:
            E[e] = m.youngs_modulus
            nu[e] = m.poisson_ratio
    n = mesh.n_nodes * ndof
    f = np.zeros(n)
    pending = None
    # CLOAD loop (assembly.rs:365-380)
    for cl in cloads:
        if cl.dof == 0 or cl.dof > ndof:
            pending = Pending(InvalidModel(
                f"load on node {cl.node_id} has unsupported dof {cl.dof}"))
            break
        idx = first_index.get(int(cl.node_id))
        if idx is None:
            pending = Pending(InvalidModel(f"load on unknown node {cl.node_id}"))
            break
        f[idx * ndof + cl.dof - 1] += cl.value
    if pending is None:
        pending = _edge_pressure(model, dloads, first_index, ndof, f)
    if pending is None:
        pending = _gravity(model, gravity, first_index, ndof, f)
    rows = []
    if pending is None:
        # constrained_dofs (solver.rs:15-41)
        for bc in bcs:
            for nid in bc.node_ids:
                idx = first_index.get(int(nid))
                if idx is None:
                    pending = Pending(InvalidModel(
                        f"boundary condition on unknown node {nid}"))
                    break
                for dof in bc.dofs:
                    if dof == 0 or dof > ndof:
                        pending = Pending(InvalidModel(
                            f"boundary condition on node {nid} has unsupported dof {dof}"))
                        break
                    rows.append(idx * ndof + dof - 1)
                if pending:
                    break
            if pending:
                break
    flat = FlatModel(xyz=mesh.coords, kind=kinds, conn_ptr=mesh.conn_ptr, conn=conn,
                     youngs=E, poisson=nu, thickness=t, ndof=ndof,
                     fixed_row=np.array(rows, dtype=np.int64), f=f,
                     node_id=mesh.node_ids, elem_id=mesh.elem_ids, no_material=nomat)
    return flat, pending


# ----------------------------------------------------------------- numerics
def element_stiffness(kind: int, coords, E: float, nu: float, t: float = 1.0):
    coords = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).reshape(-1, 3))
    N = {0: 6, 1: 8, 5: 24}[int(kind)]
    ke = np.zeros((N, N))
    r = lib().svx_oracle_element_stiffness(int(kind), abi.ptr(coords, C.c_double), E, nu, t,
                                           abi.ptr(ke, C.c_double))
    return r, ke


class Csr:
    """Host CSR copied out of the oracle."""

    def __init__(self, c: OracleCsr):
        n, nnz = int(c.n), int(c.nnz)
        self.n, self.nnz = n, nnz
        self.row_ptr = np.ctypeslib.as_array(c.row_ptr, shape=(n + 1,)).copy()
        self.col_idx = np.ctypeslib.as_array(c.col_idx, shape=(nnz,)).copy() if nnz else \
            np.zeros(0, np.int64)
        self.vals = np.ctypeslib.as_array(c.vals, shape=(nnz,)).copy() if nnz else np.zeros(0)
        self.f = np.ctypeslib.as_array(c.f, shape=(n,)).copy() if n else np.zeros(0)

    def struct(self):
        s = OracleCsr()
        s.n, s.nnz = self.n, self.nnz
        s.row_ptr = abi.ptr(self.row_ptr, C.c_int64)
        s.col_idx = abi.ptr(self.col_idx, C.c_int64)
        s.vals = abi.ptr(self.vals, C.c_double)
        s.f = abi.ptr(self.f, C.c_double)
        return s

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.vals, self.col_idx, self.row_ptr), shape=(self.n, self.n))


def _raise_err(err: abi.SvxError):
    code = err.code
    msg = err.message.decode()
    if code == abi.SVX_INVALID_MODEL:
        raise InvalidModel(msg, reason=err.reason, elem_index=err.elem_index)
    if code == abi.SVX_NOT_CONVERGED:
        raise NotConverged(int(err.iterations), float(err.residual))
    if code == abi.SVX_NO_CONSTRAINTS:
        raise NoConstraints(msg)
    if code == abi.SVX_EMPTY_MESH:
        raise EmptyMesh(msg)
    raise SolveError(msg)


def assemble(flat: FlatModel, threads: int | None = None) -> Csr:
    s = flat.as_struct()
    out = OracleCsr()
    err = abi.SvxError()
    st = lib().svx_oracle_assemble(C.byref(s), threads or default_threads(), C.byref(out),
                                   C.byref(err))
    if st != abi.SVX_OK:
        _raise_err(err)
    try:
        return Csr(out)
    finally:
        lib().svx_oracle_csr_free(C.byref(out))


def spmv(k: Csr, x, threads: int | None = None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(k.n)
    s = k.struct()
    lib().svx_oracle_spmv(C.byref(s), abi.ptr(x, C.c_double), abi.ptr(y, C.c_double),
                          threads or default_threads())
    return y


def apply_dirichlet(k: Csr, f, rows):
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    s = k.struct()
    lib().svx_oracle_apply_dirichlet(C.byref(s), abi.ptr(f, C.c_double),
                                     abi.ptr(rows, C.c_int64), rows.shape[0])


def pcg(k: Csr, f, tol=1e-10, max_iter=1000, threads: int | None = None):
    """Returns (status, u, iterations, residual)."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    u = np.zeros(k.n)
    it = C.c_int64(0)
    res = C.c_double(0.0)
    s = k.struct()
    st = lib().svx_oracle_pcg(C.byref(s), abi.ptr(f, C.c_double), tol, max_iter,
                              threads or default_threads(), abi.ptr(u, C.c_double),
                              C.byref(it), C.byref(res))
    return st, u, int(it.value), float(res.value)


def element_mass(kind: int, coords, rho: float, t: float = 1.0):
    """Consistent mass of one element (modal.rs:82-146); returns (reason, me)."""
    coords = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).reshape(-1, 3))
    N = {0: 6, 1: 8, 3: 8, 5: 24}[int(kind)]
    me = np.zeros((N, N))
    r = lib().svx_oracle_element_mass(int(kind), abi.ptr(coords, C.c_double), float(rho),
                                      float(t), abi.ptr(me, C.c_double))
    return r, me


def assemble_mass(flat: FlatModel, rho: float) -> Csr:
    """assemble_mass (modal.rs:203-271) on a flat model; raises
    InvalidModel with the reference's text for a failing element."""
    s = flat.as_struct()
    out = OracleCsr()
    err = abi.SvxError()
    st = lib().svx_oracle_assemble_mass(C.byref(s), float(rho), C.byref(out), C.byref(err))
    if st != abi.SVX_OK:
        _raise_err(err)
    try:
        return Csr(out)
    finally:
        lib().svx_oracle_csr_free(C.byref(out))


def rcm(k: Csr):
    """Reverse Cuthill-McKee permutation, old -> new (ldl.rs:27-60)."""
    perm = np.zeros(k.n, dtype=np.int64)
    s = k.struct()
    lib().svx_oracle_rcm(C.byref(s), abi.ptr(perm, C.c_int64))
    return perm


class LdltResult:
    def __init__(self, u, residual, cond, d, nnz_l):
        self.u, self.residual, self.cond, self.d, self.nnz_l = u, residual, cond, d, nnz_l


def ldlt(k: Csr, f, threads: int | None = None) -> LdltResult:
    """Factorize the (Dirichlet-modified) k and solve k u = f as the
    reference's direct path (ldl.rs:144-265, lib.rs:645-663); raises
    InvalidModel with the reference's pivot message."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    u = np.zeros(k.n)
    d = np.zeros(k.n)
    res = C.c_double(0.0)
    cond = C.c_double(0.0)
    nnz_l = C.c_int64(0)
    err = abi.SvxError()
    s = k.struct()
    st = lib().svx_oracle_ldlt(C.byref(s), abi.ptr(f, C.c_double), threads or default_threads(),
                               abi.ptr(u, C.c_double), C.byref(res), C.byref(cond),
                               abi.ptr(d, C.c_double), C.byref(nnz_l), C.byref(err))
    if st != abi.SVX_OK:
        _raise_err(err)
    return LdltResult(u, float(res.value), float(cond.value), d, int(nnz_l.value))


METHODS = {"pcg": 0, "ldlt": 1, "auto": 2}


class OracleSolution:
    def __init__(self, flat: FlatModel):
        n = flat.n_dof
        self.u = np.zeros(n)
        self.displacements = np.zeros((flat.n_nodes, 3))
        self.von_mises = np.zeros(flat.n_elem)
        self.nodal_von_mises = np.zeros(flat.n_nodes)
        self.reaction_values = np.zeros(flat.fixed_row.shape[0])
        self.iterations = 0
        self.final_residual = 0.0
        self.cond_estimate = 0.0
        self.solver_method = "pcg"


def solve_flat(flat: FlatModel, tol=1e-10, max_iter=0, threads: int | None = None,
               method: str = "pcg"):
    """Full linear-static pipeline on a flat model with the reference's
    Method ("pcg", "ldlt" or "auto", lib.rs:664-686); raises SolveError."""
    out = OracleSolution(flat)
    sol = abi.SvxSolution()
    sol.u = abi.ptr(out.u, C.c_double)
    sol.displacements = abi.ptr(out.displacements, C.c_double)
    sol.von_mises = abi.ptr(out.von_mises, C.c_double)
    sol.nodal_von_mises = abi.ptr(out.nodal_von_mises, C.c_double)
    sol.reactions = abi.ptr(out.reaction_values, C.c_double)
    err = abi.SvxError()
    s = flat.as_struct()
    used = C.c_int(0)
    st = lib().svx_oracle_solve_method(C.byref(s), threads or default_threads(), tol, max_iter,
                                       METHODS[method], C.byref(sol), C.byref(used),
                                       C.byref(err))
    if st != abi.SVX_OK:
        _raise_err(err)
    out.solver_method = "ldlt" if used.value == 1 else "pcg"
    out.iterations = int(sol.iterations)
    out.final_residual = float(sol.final_residual)
    out.cond_estimate = float(sol.cond_estimate)
    return out


def stress(flat: FlatModel, u, threads: int | None = None):
    """(von Mises per element, per node, reactions) for a given u."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    vm = np.zeros(flat.n_elem)
    vmn = np.zeros(flat.n_nodes)
    re = np.zeros(flat.fixed_row.shape[0])
    err = abi.SvxError()
    s = flat.as_struct()
    st = lib().svx_oracle_stress(C.byref(s), abi.ptr(u, C.c_double), threads or default_threads(),
                                 abi.ptr(vm, C.c_double), abi.ptr(vmn, C.c_double),
                                 abi.ptr(re, C.c_double), C.byref(err))
    if st != abi.SVX_OK:
        _raise_err(err)
    return vm, vmn, re


def solve(model: Model, tol=1e-10, threads: int | None = None, method: str = "pcg"):
    """Reference-order solve of a reference-shaped model (Method::Pcg by
    default; "ldlt" and "auto" as in lib.rs:664-686)."""
    flat, pending = resolve(model)
    if pending is not None:
        # Element failures come first (assembly runs before the CLOAD loop).
        assemble(flat, threads)
        raise pending.err
    return solve_flat(flat, tol=tol, threads=threads, method=method), flat


# ------------------------------------------------------------------ thermal
def solve_thermal(tm: ThermalModel, tol=1e-10, threads: int | None = None):
    """heat::solve_thermal restated; returns (temperatures, iterations,
    residual) or raises the reference's SolveError."""
    t = np.zeros(tm.n_nodes)
    it = C.c_int64(0)
    res = C.c_double(0.0)
    err = abi.SvxError()
    s = tm.as_struct()
    st = lib().svx_oracle_solve_thermal(C.byref(s), default_threads() if threads is None
                                        else int(threads), float(tol), abi.ptr(t, C.c_double),
                                        C.byref(it), C.byref(res), C.byref(err))
    if st != abi.SVX_OK:
        _raise_err(err)
    return t, int(it.value), float(res.value)


def conduction_element(kind: int, coords, conductivity: float, thickness: float = 1.0,
                       source=None):
    """One element's conduction matrix and heat-source load (heat.rs:149-296)."""
    nn = {int(ElemKind.Cps3): 3, int(ElemKind.Cps4): 4, int(ElemKind.Cpe4): 4,
          int(ElemKind.C3d8): 8}[int(kind)]
    c = np.zeros((nn, 3))
    xy = np.asarray(coords, dtype=np.float64).reshape(nn, -1)
    c[:, :xy.shape[1]] = xy
    c = np.ascontiguousarray(c)
    ke = np.zeros(nn * nn)
    fe = np.zeros(nn)
    r = lib().svx_oracle_conduction_element(int(kind), abi.ptr(c, C.c_double), float(conductivity),
                                            float(thickness), int(source is not None),
                                            float(source or 0.0), abi.ptr(ke, C.c_double),
                                            abi.ptr(fe, C.c_double))
    if r:
        raise InvalidModel(f"reason {r}")
    return ke.reshape(nn, nn), fe
