"""B200-native exact subgraph isomorphism behind MatrixGraph's subiso API.

Everything computes in libmg_subiso.so (hand-written CUDA for sm_100a behind
a C-ABI, include/mg_subiso.h); this package is the host-side mirror of the
reference's task/runtime interface plus ctypes plumbing.
"""
from ._lib import MGError, lib  # noqa: F401  (fails loudly when the .so is absent)
from .graph import (SHAPES, CSRGraph, chung_lu, gen_labels, query_edges,  # noqa: F401
                    query_random, query_walk, rmat)
from .subiso import (DeviceGraph, MatrixGraph, SchedulerType, SubIso, TaskType,  # noqa: F401
                     level0_sizes, make_opts, plan_order, root_costs, shard_batch,
                     shard_roots, shard_roots_weighted, shard_strided)
from .matrix_filter import MatrixFilter  # noqa: F401

__all__ = ["MGError", "CSRGraph", "DeviceGraph", "SubIso", "MatrixGraph", "TaskType",
           "SchedulerType", "chung_lu", "rmat", "query_walk", "query_random", "gen_labels",
           "plan_order", "shard_roots", "shard_roots_weighted", "shard_strided", "shard_batch",
           "root_costs", "level0_sizes", "SHAPES", "query_edges", "make_opts", "MatrixFilter"]
