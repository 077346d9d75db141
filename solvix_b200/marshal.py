"""Marshalling between the Python model mirror and the C ABI structs.

``FlatModel`` is the index-resolved model of ``svx_flat_model_t``; it is what
the synthetic generators build directly for very large meshes.
``model_desc`` packs a reference-shaped :class:`~solvix_b200.model.Model`
(ids, element sets, assignments, BCs by node id) into ``svx_model_desc_t``.
Both return the ctypes struct together with the numpy arrays it points into;
the caller keeps that pair alive for the duration of the call.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import abi
from .model import Model


@dataclass
class FlatModel:
    xyz: np.ndarray               # float64 [n_nodes, 3]
    kind: np.ndarray              # uint8 [n_elem]
    conn_ptr: np.ndarray          # int64 [n_elem + 1]
    conn: np.ndarray              # int32 node indices
    youngs: np.ndarray            # float64 [n_elem]
    poisson: np.ndarray           # float64 [n_elem]
    thickness: float
    ndof: int
    fixed_row: np.ndarray         # int64 constrained rows (BC order)
    f: np.ndarray                 # float64 [n_nodes * ndof]
    node_id: Optional[np.ndarray] = None   # uint32
    elem_id: Optional[np.ndarray] = None   # uint32
    no_material: Optional[np.ndarray] = None  # uint8

    def __post_init__(self):
        self.xyz = np.ascontiguousarray(np.asarray(self.xyz, dtype=np.float64).reshape(-1, 3))
        self.kind = np.ascontiguousarray(self.kind, dtype=np.uint8)
        self.conn_ptr = np.ascontiguousarray(self.conn_ptr, dtype=np.int64)
        self.conn = np.ascontiguousarray(self.conn, dtype=np.int32)
        n_elem = self.kind.shape[0]
        self.youngs = np.ascontiguousarray(np.broadcast_to(
            np.asarray(self.youngs, dtype=np.float64), (n_elem,)))
        self.poisson = np.ascontiguousarray(np.broadcast_to(
            np.asarray(self.poisson, dtype=np.float64), (n_elem,)))
        self.fixed_row = np.ascontiguousarray(self.fixed_row, dtype=np.int64)
        self.f = np.ascontiguousarray(self.f, dtype=np.float64)
        if self.node_id is not None:
            self.node_id = np.ascontiguousarray(self.node_id, dtype=np.uint32)
        if self.elem_id is not None:
            self.elem_id = np.ascontiguousarray(self.elem_id, dtype=np.uint32)
        if self.no_material is not None:
            self.no_material = np.ascontiguousarray(self.no_material, dtype=np.uint8)

    @property
    def n_nodes(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def n_elem(self) -> int:
        return int(self.kind.shape[0])

    @property
    def n_dof(self) -> int:
        return self.n_nodes * self.ndof

    def nbytes(self) -> int:
        """Host bytes of the arrays the C ABI copies in."""
        arrs = [self.xyz, self.kind, self.conn_ptr, self.conn, self.youngs, self.poisson,
                self.fixed_row, self.f]
        arrs += [a for a in (self.node_id, self.elem_id, self.no_material) if a is not None]
        return int(sum(a.nbytes for a in arrs))

    def as_struct(self) -> abi.SvxFlatModel:
        s = abi.SvxFlatModel()
        s.n_nodes = self.n_nodes
        s.xyz = abi.ptr(self.xyz, C.c_double)
        s.node_id = abi.ptr(self.node_id, C.c_uint32)
        s.n_elem = self.n_elem
        s.kind = abi.ptr(self.kind, C.c_uint8)
        s.conn_ptr = abi.ptr(self.conn_ptr, C.c_int64)
        s.conn = abi.ptr(self.conn, C.c_int32)
        s.youngs = abi.ptr(self.youngs, C.c_double)
        s.poisson = abi.ptr(self.poisson, C.c_double)
        s.no_material = abi.ptr(self.no_material, C.c_uint8)
        s.elem_id = abi.ptr(self.elem_id, C.c_uint32)
        s.thickness = float(self.thickness)
        s.ndof = int(self.ndof)
        s.n_fixed = int(self.fixed_row.shape[0])
        s.fixed_row = abi.ptr(self.fixed_row, C.c_int64)
        s.f = abi.ptr(self.f, C.c_double)
        return s

    def raw_fields(self) -> tuple:
        """The svx_flat_model_t fields with integer addresses, in field order
        (for abi.SvxFlatModelRaw)."""
        def addr(a):
            return None if a is None else a.__array_interface__["data"][0]
        return (self.n_nodes, addr(self.xyz), addr(self.node_id), self.n_elem, addr(self.kind),
                addr(self.conn_ptr), addr(self.conn), addr(self.youngs), addr(self.poisson),
                addr(self.no_material), addr(self.elem_id), float(self.thickness),
                int(self.ndof), int(self.fixed_row.shape[0]), addr(self.fixed_row),
                addr(self.f))

    @classmethod
    def from_struct(cls, s: abi.SvxFlatModel) -> "FlatModel":
        """Copy a library-owned svx_flat_model_t into numpy arrays."""
        n, m = int(s.n_nodes), int(s.n_elem)

        def arr(p, count, dt):
            if not p or count == 0:
                return np.zeros(count, dtype=dt) if p else None
            return np.ctypeslib.as_array(p, shape=(count,)).astype(dt, copy=True)

        conn_ptr = arr(s.conn_ptr, m + 1, np.int64)
        n_conn = int(conn_ptr[-1]) if conn_ptr is not None and m > 0 else 0
        return cls(
            xyz=arr(s.xyz, 3 * n, np.float64).reshape(-1, 3),
            kind=arr(s.kind, m, np.uint8),
            conn_ptr=conn_ptr,
            conn=arr(s.conn, n_conn, np.int32) if n_conn else np.zeros(0, np.int32),
            youngs=arr(s.youngs, m, np.float64),
            poisson=arr(s.poisson, m, np.float64),
            thickness=float(s.thickness),
            ndof=int(s.ndof),
            fixed_row=arr(s.fixed_row, int(s.n_fixed), np.int64)
            if s.n_fixed else np.zeros(0, np.int64),
            f=arr(s.f, n * int(s.ndof), np.float64),
            node_id=arr(s.node_id, n, np.uint32),
            elem_id=arr(s.elem_id, m, np.uint32),
            no_material=arr(s.no_material, m, np.uint8),
        )


def _cstr_array(names):
    raw = [n.encode("utf-8") for n in names]
    arr = (C.c_char_p * max(1, len(raw)))(*raw)
    return arr, raw


def model_desc(model: Model):
    """Pack a Model (after ``load_state``) into ``svx_model_desc_t``.

    Returns ``(desc, keepalive)``.
    """
    bcs, cloads, dloads, gravity = model.load_state()
    mesh = model.mesh
    keep = []

    d = abi.SvxModelDesc()
    d.n_nodes = mesh.n_nodes
    node_ids = np.ascontiguousarray(mesh.node_ids, dtype=np.uint32)
    coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    keep += [node_ids, coords]
    d.node_ids = abi.ptr(node_ids, C.c_uint32)
    d.node_coords = abi.ptr(coords, C.c_double)

    d.n_elems = mesh.n_elements
    ek = [np.ascontiguousarray(mesh.elem_ids, dtype=np.uint32),
          np.ascontiguousarray(mesh.elem_kinds, dtype=np.uint8),
          np.ascontiguousarray(mesh.conn_ptr, dtype=np.int64),
          np.ascontiguousarray(mesh.conn, dtype=np.uint32)]
    keep += ek
    d.elem_ids = abi.ptr(ek[0], C.c_uint32)
    d.elem_kinds = abi.ptr(ek[1], C.c_uint8)
    d.elem_conn_ptr = abi.ptr(ek[2], C.c_int64)
    d.elem_conn = abi.ptr(ek[3], C.c_uint32)

    mats = list(model.materials)
    d.n_materials = len(mats)
    mnames, raw = _cstr_array([m.name for m in mats])
    e_arr = np.array([m.youngs_modulus for m in mats] or [0.0], dtype=np.float64)
    nu_arr = np.array([m.poisson_ratio for m in mats] or [0.0], dtype=np.float64)
    keep += [mnames, raw, e_arr, nu_arr]
    d.material_names = C.cast(mnames, abi.c_char_pp)
    d.youngs_modulus = abi.ptr(e_arr, C.c_double)
    d.poisson_ratio = abi.ptr(nu_arr, C.c_double)

    sets = list(model.elsets)
    d.n_elsets = len(sets)
    snames, raw = _cstr_array([s.name for s in sets])
    sptr = np.zeros(len(sets) + 1, dtype=np.int64)
    parts = [np.asarray(s.element_ids, dtype=np.uint32).ravel() for s in sets]
    if parts:
        np.cumsum([p.shape[0] for p in parts], out=sptr[1:])
    sids = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(1, np.uint32),
                                dtype=np.uint32)
    keep += [snames, raw, sptr, sids]
    d.elset_names = C.cast(snames, abi.c_char_pp)
    d.elset_ptr = abi.ptr(sptr, C.c_int64)
    d.elset_elem_ids = abi.ptr(sids, C.c_uint32)

    asg = list(model.mat_assignments)
    d.n_assignments = len(asg)
    a_set, raw1 = _cstr_array([a[0] for a in asg])
    a_mat, raw2 = _cstr_array([a[1] for a in asg])
    keep += [a_set, raw1, a_mat, raw2]
    d.assign_elset = C.cast(a_set, abi.c_char_pp)
    d.assign_material = C.cast(a_mat, abi.c_char_pp)

    d.thickness = float(model.thickness)

    d.n_bcs = len(bcs)
    bn_ptr = np.zeros(len(bcs) + 1, dtype=np.int64)
    bd_ptr = np.zeros(len(bcs) + 1, dtype=np.int64)
    bn = [np.asarray(b.node_ids, dtype=np.uint32).ravel() for b in bcs]
    bd = [np.asarray(b.dofs, dtype=np.int64).ravel() for b in bcs]
    if bcs:
        np.cumsum([x.shape[0] for x in bn], out=bn_ptr[1:])
        np.cumsum([x.shape[0] for x in bd], out=bd_ptr[1:])
    bn_all = np.ascontiguousarray(np.concatenate(bn) if bn else np.zeros(1, np.uint32),
                                  dtype=np.uint32)
    bd_all = np.ascontiguousarray(np.concatenate(bd) if bd else np.zeros(1, np.int64),
                                  dtype=np.int64)
    keep += [bn_ptr, bd_ptr, bn_all, bd_all]
    d.bc_node_ptr = abi.ptr(bn_ptr, C.c_int64)
    d.bc_node_ids = abi.ptr(bn_all, C.c_uint32)
    d.bc_dof_ptr = abi.ptr(bd_ptr, C.c_int64)
    d.bc_dofs = abi.ptr(bd_all, C.c_int64)

    d.n_cloads = len(cloads)
    cn = np.array([c.node_id for c in cloads] or [0], dtype=np.uint32)
    cd = np.array([c.dof for c in cloads] or [0], dtype=np.int64)
    cv = np.array([c.value for c in cloads] or [0.0], dtype=np.float64)
    keep += [cn, cd, cv]
    d.cload_node_ids = abi.ptr(cn, C.c_uint32)
    d.cload_dofs = abi.ptr(cd, C.c_int64)
    d.cload_values = abi.ptr(cv, C.c_double)

    d.density = float(model.density)
    d.n_dloads = len(dloads)
    de = np.array([x.element_id for x in dloads] or [0], dtype=np.uint32)
    df = np.array([x.face for x in dloads] or [0], dtype=np.int64)
    dv = np.array([x.magnitude for x in dloads] or [0.0], dtype=np.float64)
    keep += [de, df, dv]
    d.dload_elem_ids = abi.ptr(de, C.c_uint32)
    d.dload_faces = abi.ptr(df, C.c_int64)
    d.dload_values = abi.ptr(dv, C.c_double)
    d.has_gravity = 1 if gravity is not None else 0
    if gravity is not None:
        g, direction = gravity
        d.gravity_magnitude = float(g)
        for k in range(3):
            d.gravity_dir[k] = float(direction[k])
    return d, keep


class ThermalModel:
    """Flat steady-conduction model (svx_thermal_model_t): what
    heat::solve_thermal (heat.rs:52-98) reads from a Model and its last
    Step, with 0-based node indices, temperature constraints in order (a
    later one for the same node wins) and plane-edge heat fluxes by element
    index and 1-based face."""

    def __init__(self, xyz, kind, conn_ptr, conn, conductivity, thickness=1.0, elem_id=None,
                 source=None, temp_node=(), temp_value=(), flux_elem=(), flux_face=(),
                 flux_value=()):
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self.kind = np.ascontiguousarray(kind, dtype=np.uint8)
        self.conn_ptr = np.ascontiguousarray(conn_ptr, dtype=np.int64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32)
        self.elem_id = None if elem_id is None else np.ascontiguousarray(elem_id, dtype=np.uint32)
        self.conductivity = float(conductivity)
        self.thickness = float(thickness)
        self.source = source
        self.temp_node = np.ascontiguousarray(temp_node, dtype=np.int64)
        self.temp_value = np.ascontiguousarray(temp_value, dtype=np.float64)
        self.flux_elem = np.ascontiguousarray(flux_elem, dtype=np.int64)
        self.flux_face = np.ascontiguousarray(flux_face, dtype=np.int32)
        self.flux_value = np.ascontiguousarray(flux_value, dtype=np.float64)

    @property
    def n_nodes(self) -> int:
        return self.xyz.shape[0]

    def as_struct(self) -> abi.SvxThermalModel:
        """The C view of this model (valid while the model is alive)."""
        def p(a, t):
            return a.ctypes.data_as(C.POINTER(t)) if a is not None and a.size else None
        return abi.SvxThermalModel(
            self.n_nodes, p(self.xyz, C.c_double), self.kind.shape[0], p(self.kind, C.c_uint8),
            p(self.conn_ptr, C.c_int64), p(self.conn, C.c_int32), p(self.elem_id, C.c_uint32),
            self.thickness, self.conductivity, int(self.source is not None),
            float(self.source or 0.0), self.temp_node.shape[0], p(self.temp_node, C.c_int64),
            p(self.temp_value, C.c_double), self.flux_elem.shape[0], p(self.flux_elem, C.c_int64),
            p(self.flux_face, C.c_int32), p(self.flux_value, C.c_double))
