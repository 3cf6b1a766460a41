"""pkde_b200: the B200-native ``:gradepro`` estimator of ParallelKDE.jl behind its own
API (initialize_estimation / estimate_density / get_density), over a C-ABI CUDA library.
"""
from ._lib import LIB_PATH, ArgumentError, CudaLibraryError, context, load
from .api import (DEFAULT_IMPLEMENTATIONS, DEVICE_IMPLEMENTATIONS, KDE, AbstractEstimator, DensityEstimation,
                  GradeProEstimator, RoTEstimator, add_estimator, bootstrap_indices, ensure_valid_implementation, estimate,
                  estimate_density, estimator_lookup, get_data, get_density, get_grid, get_nsamples, has_grid,
                  initialize_estimation, initialize_kde, set_density, set_nan_density)
from .grids import Grid, find_grid, initialize_grid

__all__ = [
    "ArgumentError", "CudaLibraryError", "DensityEstimation", "Grid", "KDE", "AbstractEstimator",
    "GradeProEstimator", "RoTEstimator", "add_estimator", "bootstrap_indices", "ensure_valid_implementation", "estimate",
    "estimate_density", "estimator_lookup", "find_grid", "get_data", "get_density", "get_grid", "get_nsamples",
    "has_grid", "initialize_estimation", "initialize_grid", "initialize_kde", "set_density", "set_nan_density",
    "load", "context", "LIB_PATH", "DEFAULT_IMPLEMENTATIONS", "DEVICE_IMPLEMENTATIONS",
]
