"""Abaqus .inp decks of the linear-static path through svx_inp_parse: the
reference's parse_inp (crates/solvix-io/src/parser.rs) for the keywords
such decks use, returning the Python mirror of its Model (with the BCs and
loads of Model::load_state) and its ParseReport warnings.  A deck that
uses keywords outside that set raises ``UnsupportedDeck``: parse it with
the reference's own parser."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .model import (BoundaryCondition, ConcentratedLoad, DistributedLoad, ElemKind, Element,
                    ElementSet, Material, Mesh, Model, Node, Step)


class ParseError(Exception):
    """The reference's ParseError: a 1-based line and a message."""

    def __init__(self, line: int, message: str):
        super().__init__(f"line {line}: {message}")
        self.line = line
        self.message = message


class UnsupportedDeck(Exception):
    """The deck needs the reference's parser (keywords outside this reader)."""


def _strs(p, n):
    return [p[i].decode() for i in range(n)]


def parse_inp(text: str):
    """Returns (Model, warnings, steps read) or raises ParseError /
    UnsupportedDeck."""
    lib = abi.load()
    raw = text.encode()
    h = C.c_void_p()
    err = abi.SvxError()
    st = lib.svx_inp_parse(raw, len(raw), C.byref(h), C.byref(err))
    if st == abi.SVX_PARSE_ERROR:
        raise ParseError(int(err.elem_index), err.message.decode())
    if st == abi.SVX_UNSUPPORTED:
        raise UnsupportedDeck(err.message.decode())
    if st != abi.SVX_OK:
        raise ValueError(err.message.decode())
    try:
        d = lib.svx_inp_model(h).contents
        nn, ne = int(d.n_nodes), int(d.n_elems)
        ids = np.ctypeslib.as_array(d.node_ids, shape=(nn,)).copy() if nn else []
        xyz = np.ctypeslib.as_array(d.node_coords, shape=(3 * nn,)).reshape(nn, 3).copy() \
            if nn else np.zeros((0, 3))
        nodes = [Node(int(ids[i]), tuple(float(v) for v in xyz[i])) for i in range(nn)]
        ptr = [int(d.elem_conn_ptr[i]) for i in range(ne + 1)]
        elems = [Element(int(d.elem_ids[e]), ElemKind(int(d.elem_kinds[e])),
                         [int(d.elem_conn[q]) for q in range(ptr[e], ptr[e + 1])])
                 for e in range(ne)]
        mats = [Material(n, float(d.youngs_modulus[i]), float(d.poisson_ratio[i]))
                for i, n in enumerate(_strs(d.material_names, int(d.n_materials)))]
        names = _strs(d.elset_names, int(d.n_elsets))
        sets = [ElementSet(n, [int(d.elset_elem_ids[q])
                               for q in range(int(d.elset_ptr[i]), int(d.elset_ptr[i + 1]))])
                for i, n in enumerate(names)]
        na = int(d.n_assignments)
        assign = list(zip(_strs(d.assign_elset, na), _strs(d.assign_material, na)))
        def span(ptr, b):
            return range(int(ptr[b]), int(ptr[b + 1]))
        bcs = [BoundaryCondition([int(d.bc_node_ids[q]) for q in span(d.bc_node_ptr, b)],
                                 [int(d.bc_dofs[q]) for q in span(d.bc_dof_ptr, b)])
               for b in range(int(d.n_bcs))]
        cloads = [ConcentratedLoad(int(d.cload_node_ids[k]), int(d.cload_dofs[k]),
                                   float(d.cload_values[k])) for k in range(int(d.n_cloads))]
        dloads = [DistributedLoad(int(d.dload_elem_ids[k]), int(d.dload_faces[k]),
                                  float(d.dload_values[k])) for k in range(int(d.n_dloads))]
        gravity = ((float(d.gravity_magnitude), tuple(float(v) for v in d.gravity_dir))
                   if d.has_gravity else None)
        model = Model(mesh=Mesh(nodes, elems), thickness=float(d.thickness),
                      density=float(d.density), materials=mats, elsets=sets,
                      mat_assignments=assign, boundary_conditions=bcs, cloads=cloads)
        if dloads or gravity is not None:
            # distributed loads and gravity live in steps (Model::load_state
            # reads them only from the last step)
            model.steps = [Step(boundary_conditions=bcs, cloads=cloads, dloads=dloads,
                                gravity=gravity)]
        warnings = [lib.svx_inp_warning(h, i).decode()
                    for i in range(lib.svx_inp_warning_count(h))]
        steps = int(lib.svx_inp_step_count(h))
    finally:
        lib.svx_inp_free(h)
    return model, warnings, steps
