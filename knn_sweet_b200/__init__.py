"""knn_sweet_b200: B200-native exact kNN join with triangle-inequality pruning.

The compute path is libknnsweet.so (hand-written CUDA for sm_100a) behind the
C ABI in include/knnsweet.h; this package is its Python front end.
"""
from ._lib import KnnError, load  # noqa: F401
from .join import (JoinStats, knnjoin, knnjoin_partition, knnjoin_sharded,  # noqa: F401
                   pack_indexdist)

__all__ = ["knnjoin", "knnjoin_sharded", "knnjoin_partition", "pack_indexdist", "JoinStats",
           "KnnError", "load"]
