"""tensorjoin_variants_b200 -- B200-native certified exact epsilon-join.

Public API (drop-in for the reference's join path):
    join(R, S, eps)            -> (i, j) sorted, R-S mode
    self_join(X, eps, mode=)   -> (i, j) sorted, 'upper' (i < j) or 'directed'
    join_result(...)           -> Result handle (pairs / keys / neighbour table / stats)
    build_index(X, eps)        -> Index (Morton order, cells, candidate tile pairs)
    join_batched([(R,S,eps)])  -> per-join (i, j)
    autotune.Tuner             -> per-(d, dtype, screen, mode, size, selectivity) choice of the
                                  run-time variants, measured on a row sample
All work runs in libtensorjoin.so (hand-written sm_100a CUDA behind a C ABI).
"""
from .api import (BatchResult, Index, Result, build_index, join, join_batched, join_batched_result,  # noqa: F401
                  join_result, self_join)
from . import autotune  # noqa: F401

__version__ = "0.1.0"
