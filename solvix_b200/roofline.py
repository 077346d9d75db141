"""Algorithmic bytes of the PCG kernels, the numerators of their rooflines.

The PCG path is HBM-bound, so every roofline figure divides the bytes a
kernel must move (not the bytes ncu sees it move) by its measured duration.
K is stored in node blocks (a node's ndof rows over its sorted neighbours):
one 4-byte column index per ndof x ndof block, and per node one row-block
offset and one adjacency offset (8 bytes each).
"""
from __future__ import annotations


def spmv_node_bytes(n: int, nnz: int, ndof: int, n_nodes: int, value_bytes: int = 8) -> int:
    """One node-block SpMV with p.Kp (spmv_node_dot): K values, one column
    index per block, adj_ptr and node_base, p gathered once, q written and
    p read for the dot (the vectors are FP64)."""
    return int(value_bytes * nnz + 4 * nnz // (ndof * ndof) + 16 * (n_nodes + 1) + 24 * n)


def pcg_iteration_bytes(n: int, nnz: int, ndof: int, n_nodes: int) -> int:
    """One FP64 PCG iteration: the node-block SpMV with p.Kp, then the u/r
    update (u r/w, p, r r/w, q, inv_diag) and the p update (p r/w, r,
    inv_diag)."""
    return spmv_node_bytes(n, nnz, ndof, n_nodes) + 8 * n * 11
