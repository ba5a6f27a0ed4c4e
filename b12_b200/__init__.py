"""b12_b200 - B200-native (sm_100a) box-image path of an implicit box tree.

The compute runs in libb12g.so (hand-written CUDA behind the C ABI of
include/b12g.h).  This package is the Python host mirror of the reference's
ImplicitBoxTree interface used by the tests and the benchmark.
"""
from ._lib import (ALL, ARITH_FMA, ARITH_STRICT, B12gError, ENTR, EQU, EXPD, EXTR, GRID_FULL, GRID_INNER,
                   GRID_PHILOX, HIT, INS, INVALID_INDEX, LEAF_DEPTH, MAP_COUPLED_DUFFING, MAP_FORCED_DUFFING,
                   MAP_HENON, MAP_LORENZ, NONE, SD)
from .tree import (Batch, CsrMatrix, GridSpec, ImplicitBoxTree, MapSpec, Scheme, coupled_duffing, forced_duffing,
                   full_grid, henon, inner_grid, lorenz, philox_grid)
from .server import JobServer

__all__ = [
    "ImplicitBoxTree", "Batch", "JobServer", "CsrMatrix", "Scheme", "MapSpec", "GridSpec", "henon", "lorenz", "coupled_duffing",
    "forced_duffing", "inner_grid", "full_grid", "philox_grid", "B12gError", "NONE", "HIT", "INS", "EXPD", "SD",
    "EQU", "ENTR", "EXTR", "ALL", "LEAF_DEPTH", "INVALID_INDEX", "MAP_HENON", "MAP_LORENZ", "MAP_COUPLED_DUFFING",
    "MAP_FORCED_DUFFING", "GRID_INNER", "GRID_FULL", "GRID_PHILOX", "ARITH_STRICT", "ARITH_FMA",
]
