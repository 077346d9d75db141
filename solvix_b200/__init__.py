"""solvix_b200 - the linear-static hot path of Solvix on one NVIDIA B200.

Element stiffness integration (CPS3 / CPS4 / C3D8), deterministic CSR
assembly, Jacobi-PCG (plain FP64 and FP32-inner mixed precision) and stress
recovery run as hand-written sm_100a CUDA kernels in ``libsolvix_b200.so``,
reached through the C ABI declared in ``include/solvix_gpu.h``.  This package
mirrors solvix-core's data model and ``solve`` entry points on top of it.
"""
from .model import (BoundaryCondition, ConcentratedLoad, DeviceError, DistributedLoad,
                    ElemKind, Element, ElementSet, EmptyMesh, InvalidModel, Material, Mesh, Method, Model, Node,
                    NoConstraints, NotConverged, Reaction, SolveError, Solution, Step)
from .marshal import FlatModel
from .core import Context, Operator, default_context, solve, solve_with_method
from . import abi

__all__ = [
    "BoundaryCondition", "ConcentratedLoad", "DeviceError", "DistributedLoad", "ElemKind", "Element", "ElementSet",
    "EmptyMesh", "InvalidModel", "Material", "Mesh", "Method", "Model", "Node", "NoConstraints",
    "NotConverged", "Reaction", "SolveError", "Solution", "Step", "FlatModel", "Context",
    "Operator", "default_context", "solve", "solve_with_method", "abi",
]
