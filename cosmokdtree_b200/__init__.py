"""cosmokdtree_b200 -- B200-native (sm_100a) k-d tree build / kNN / ball / box search.

A drop-in for cosmokdtree's Python API (``cosmokdtree.kdtree``): ``from
cosmokdtree_b200 import kdtree`` and call ``kdtree.build_kdtree`` etc. exactly as with
the reference.  All compute runs in hand-written CUDA kernels in ``libckd.so``.
"""
from . import kdtree  # noqa: F401
from .kdtree import (  # noqa: F401
    KDTree, ball_search, ball_search_csr, box_search, box_search_csr, build_kdtree,
    deallocate_kdtree, knn_search, knn_search_batch,
)
from .forest import Forest, ForestPlan, build_forest  # noqa: F401

__version__ = "0.1.0"
