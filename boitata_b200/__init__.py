"""boitata_b200 — B200-native ordinary / simple / indicator kriging of block models.

A drop-in for the kriging path of gstvschlz/boitata (`OrdinaryKriging`,
`SimpleKriging`, `IndicatorKriging`, `BlockKriging`, `Variogram`,
`Structure`, `Search`):
neighbour search, covariance assembly, bordered solve and estimate /
variance run as hand-written sm_100a CUDA kernels behind the C ABI of
include/boitata_b200.h.
"""

from .errors import BoitataError, InvalidInput, MissingColumn, Unsupported
from .persist import FileError
from .estimation import BlockKriging, CrossValidation, IndicatorKriging, OrdinaryKriging, SimpleKriging
from .calibrate import calibrate_search, global_bias
from .declustering import Declustering, weight_declustering
from .geometry import BlockModel, Geometry, PointSet
from .search import Search
from .simulation import SGS, Simulation
from .table import Table
from .variogram import Structure, Variogram

__all__ = [
    "BlockKriging",
    "BlockModel",
    "BoitataError",
    "CrossValidation",
    "Declustering",
    "FileError",
    "Geometry",
    "IndicatorKriging",
    "InvalidInput",
    "MissingColumn",
    "OrdinaryKriging",
    "PointSet",
    "SGS",
    "Search",
    "Simulation",
    "SimpleKriging",
    "Structure",
    "Table",
    "Unsupported",
    "Variogram",
    "calibrate_search",
    "global_bias",
    "weight_declustering",
]
__version__ = "0.1.0"
