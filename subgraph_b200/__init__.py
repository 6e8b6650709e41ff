"""subgraph_b200: color-coding tree-template counting on B200 (sm_100a).

A drop-in for the counting path of dsc-nec/subgraph: the same inputs
(text edge lists, CSC/CSR graphs, graph.data, tree templates), the same
sub-template division and color-set indexing, and per-coloring counts from
hand-written sm_100a kernels behind a C ABI (include/sg_api.h).
"""
from .api import (DUMMY_VAL, MODE_FP64, MODE_ORIGINAL, MODE_ORIGINAL_CSR, MODE_REFERENCE, CountMat, CSCGraph, CSRGraph,
                  DeviceGraph, DivideTemplates, EdgeList, Graph, IndexSys, SGError, count, count_jobs,
                  debug_count_unsatisfiable_wait, debug_root,
                  debug_sub_table, estimate, rmat)
from ._lib import LIB_PATH, lib

__all__ = ["EdgeList", "CSCGraph", "CSRGraph", "DeviceGraph", "Graph", "DivideTemplates", "IndexSys", "CountMat",
           "count", "count_jobs", "estimate", "rmat", "debug_sub_table", "debug_root", "debug_count_unsatisfiable_wait", "MODE_REFERENCE", "MODE_FP64",
           "MODE_ORIGINAL", "MODE_ORIGINAL_CSR", "DUMMY_VAL", "SGError", "LIB_PATH", "lib"]
