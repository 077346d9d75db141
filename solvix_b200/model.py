"""Python mirror of solvix-core's public data model and solve API.

Names, fields and error behaviour follow ``crates/solvix-core/src/lib.rs``:

* ``Node`` / ``Element`` / ``ElemKind`` / ``Mesh``   (lib.rs:39-109)
* ``Material`` / ``ElementSet`` / ``BoundaryCondition`` / ``ConcentratedLoad``
  / ``Step`` / ``Model``                              (lib.rs:111-330)
* ``Solution`` / ``Reaction``                         (lib.rs:475-513)
* ``SolveError`` and its variants                     (lib.rs:515-521)
* ``Method``, ``solve``, ``solve_with_method``        (lib.rs:523-590)

Large meshes are held as numpy arrays (``Mesh.from_arrays``); the
list-of-records constructors exist so that tests read like the reference's.
The computation itself happens behind the C ABI of ``libsolvix_b200.so``.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np


class ElemKind(enum.IntEnum):
    """Element kinds, same order as the reference's ``ElemKind``."""

    Cps3 = 0
    Cps4 = 1
    Cps8 = 2
    Cpe4 = 3
    Cpe8 = 4
    C3d8 = 5
    C3d4 = 6
    B31 = 7

    def node_count(self) -> int:
        return {0: 3, 1: 4, 2: 8, 3: 4, 4: 8, 5: 8, 6: 4, 7: 2}[int(self)]


NODE_COUNT = np.array([3, 4, 8, 4, 8, 8, 4, 2], dtype=np.int64)


@dataclass
class Node:
    id: int
    coords: Sequence[float]


@dataclass
class Element:
    id: int
    kind: ElemKind
    connectivity: Sequence[int]


class Mesh:
    """Nodes and elements, stored as arrays.

    ``node_ids`` uint32[n], ``coords`` float64[n,3], ``elem_ids`` uint32[m],
    ``elem_kinds`` uint8[m], ``conn_ptr`` int64[m+1], ``conn`` uint32 node ids.
    """

    def __init__(self, nodes: Sequence[Node] = (), elements: Sequence[Element] = ()):
        self.node_ids = np.array([n.id for n in nodes], dtype=np.uint32)
        self.coords = np.array([list(n.coords) + [0.0] * (3 - len(n.coords)) for n in nodes],
                               dtype=np.float64).reshape(-1, 3)
        self.elem_ids = np.array([e.id for e in elements], dtype=np.uint32)
        self.elem_kinds = np.array([int(e.kind) for e in elements], dtype=np.uint8)
        lens = np.array([len(e.connectivity) for e in elements], dtype=np.int64)
        self.conn_ptr = np.zeros(len(elements) + 1, dtype=np.int64)
        np.cumsum(lens, out=self.conn_ptr[1:])
        self.conn = np.array([c for e in elements for c in e.connectivity], dtype=np.uint32)

    @classmethod
    def from_arrays(cls, node_ids, coords, elem_ids, elem_kinds, conn_ptr, conn) -> "Mesh":
        m = cls.__new__(cls)
        m.node_ids = np.ascontiguousarray(node_ids, dtype=np.uint32)
        m.coords = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).reshape(-1, 3))
        m.elem_ids = np.ascontiguousarray(elem_ids, dtype=np.uint32)
        m.elem_kinds = np.ascontiguousarray(elem_kinds, dtype=np.uint8)
        m.conn_ptr = np.ascontiguousarray(conn_ptr, dtype=np.int64)
        m.conn = np.ascontiguousarray(conn, dtype=np.uint32)
        return m

    @property
    def n_nodes(self) -> int:
        return int(self.node_ids.shape[0])

    @property
    def n_elements(self) -> int:
        return int(self.elem_ids.shape[0])

    @property
    def nodes(self):
        return [Node(int(i), tuple(c)) for i, c in zip(self.node_ids, self.coords)]

    @property
    def elements(self):
        return [Element(int(self.elem_ids[e]), ElemKind(int(self.elem_kinds[e])),
                        [int(x) for x in self.conn[self.conn_ptr[e]:self.conn_ptr[e + 1]]])
                for e in range(self.n_elements)]

    def node_index(self, node_id: int) -> Optional[int]:
        """Position of the first node with ``node_id`` (lib.rs:106-108)."""
        hit = np.nonzero(self.node_ids == node_id)[0]
        return int(hit[0]) if hit.size else None

    def element_index(self, elem_id: int) -> Optional[int]:
        hit = np.nonzero(self.elem_ids == elem_id)[0]
        return int(hit[0]) if hit.size else None


@dataclass
class Material:
    name: str
    youngs_modulus: float
    poisson_ratio: float


@dataclass
class ElementSet:
    name: str
    element_ids: Sequence[int]


@dataclass
class BoundaryCondition:
    node_ids: Sequence[int]
    dofs: Sequence[int]


@dataclass
class ConcentratedLoad:
    node_id: int
    dof: int
    value: float


@dataclass
class DistributedLoad:
    """Edge pressure on a plane element (lib.rs:150-158): `face` is the
    1-based Abaqus edge (P1..P4 on CPS4, P1..P3 on CPS3), edge n joining
    local nodes n and n+1; positive magnitude acts into the element."""

    element_id: int
    face: int
    magnitude: float


@dataclass
class Step:
    """One analysis step's accumulated state (lib.rs:309-330)."""

    boundary_conditions: list = field(default_factory=list)
    cloads: list = field(default_factory=list)
    dloads: list = field(default_factory=list)
    gravity: Optional[tuple] = None
    nlgeom: bool = False


@dataclass
class Model:
    """A complete, solvable model (lib.rs:250-307); defaults of lib.rs:309-333."""

    mesh: Mesh = field(default_factory=Mesh)
    thickness: float = 1.0
    density: float = 7850.0
    materials: list = field(default_factory=list)
    elsets: list = field(default_factory=list)
    mat_assignments: list = field(default_factory=list)
    boundary_conditions: list = field(default_factory=list)
    cloads: list = field(default_factory=list)
    steps: list = field(default_factory=list)

    def load_state(self):
        """(bcs, cloads, dloads, gravity) after step normalisation (lib.rs:388-403)."""
        if self.steps:
            s = self.steps[-1]
            return s.boundary_conditions, s.cloads, s.dloads, s.gravity
        return self.boundary_conditions, self.cloads, [], None


@dataclass
class Reaction:
    node_id: int
    dof: int
    value: float


@dataclass
class Solution:
    """Solver output; arrays parallel to mesh nodes / elements (lib.rs:485-513)."""

    displacements: np.ndarray
    von_mises: np.ndarray
    nodal_von_mises: np.ndarray
    reactions: list
    iterations: int
    final_residual: float
    solver_method: str
    cond_estimate: float
    u: Optional[np.ndarray] = None
    reaction_values: Optional[np.ndarray] = None
    outer_iterations: int = 0
    ms_assemble: float = 0.0
    ms_solve: float = 0.0
    ms_stress: float = 0.0
    factor_bandwidth: int = 0   # direct path: half-bandwidth of K in the RCM order
    ms_factor: float = 0.0      # direct path: device time of factorization + solves
    fp32_iterations: int = 0    # mixed forms: iterations on the FP32 operator


class SolveError(Exception):
    """Base of the reference's ``SolveError`` variants (lib.rs:515-521)."""


class EmptyMesh(SolveError):
    pass


class NoConstraints(SolveError):
    pass


class InvalidModel(SolveError):
    def __init__(self, message: str, reason: int = 0, elem_index: int = -1):
        super().__init__(message)
        self.message = message
        self.reason = reason
        self.elem_index = elem_index

    def __eq__(self, other):
        return isinstance(other, InvalidModel) and other.message == self.message

    __hash__ = Exception.__hash__


class NotConverged(SolveError):
    def __init__(self, iterations: int, residual: float):
        super().__init__(f"not converged after {iterations} iterations (residual {residual:.3e})")
        self.iterations = iterations
        self.residual = residual


class DeviceError(SolveError):
    """CUDA / allocation failure on the device (no CPU fallback exists)."""


class Method(enum.Enum):
    """Linear solver selection (lib.rs:523-534): ``Pcg`` (Jacobi-PCG),
    ``Ldlt`` (the direct path) or ``Auto`` (PCG, then the direct path when
    the PCG does not converge; the default of ``solve``)."""

    Auto = "auto"
    Pcg = "pcg"
    Ldlt = "ldlt"
