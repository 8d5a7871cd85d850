"""kwave_b200 -- KWave.jl's k-space time-stepping solvers (fluid, axisymmetric, elastic) on NVIDIA B200 (sm_100a).

The user-facing names mirror KWave.jl (KWave.jl/src/KWave.jl exports): build a grid, medium,
source and sensor, then call ``kspace_first_order``.  The time loop runs in libkwb.so
(hand-written CUDA, C ABI in include/kwb.h); there is no CPU fallback.
"""

from .core import (Additive, AdditiveNoCorrection, Dirichlet, ElasticMedium, ElasticSource, KWaveGrid, KWaveMedium, KWaveSensor,
                   KWaveSource, SimulationOutput, SourceMode, VALID_RECORD_FIELDS, db2neper,
                   get_optimal_pml_size, get_pml, grid_size, grid_spacing, k_max, make_ball, make_circle,
                   make_disc, make_line, total_grid_points,
                   make_time, neper2db, smooth, tone_burst, validate_record_fields)
from ._lib import KWaveB200Error, LIB_PATH, load_library
from .solver import (Context, Prepared, Request, Simulation, prepare, solve_prepared, submit_prepared, build_problem, default_context, estimate_device_bytes,
                     kspace_first_order, kspace_first_order_as, pstd_elastic_2d, pstd_elastic_3d, run_sharded, serving_config, serving_stats, shard_jobs, solve_batch, submit)

make_time_ = make_time  # `make_time!` in the reference

__all__ = [
    "Additive", "AdditiveNoCorrection", "Dirichlet", "KWaveGrid", "KWaveMedium", "KWaveSensor",
    "KWaveSource", "SimulationOutput", "SourceMode", "VALID_RECORD_FIELDS", "db2neper",
    "get_optimal_pml_size", "get_pml", "make_ball", "make_circle", "make_disc", "make_line",
    "make_time", "make_time_", "neper2db", "smooth", "tone_burst", "validate_record_fields",
    "KWaveB200Error", "LIB_PATH", "load_library", "Context", "Simulation", "build_problem",
    "default_context", "kspace_first_order", "kspace_first_order_as", "Request", "estimate_device_bytes", "serving_config",
    "serving_stats", "shard_jobs", "run_sharded", "solve_batch", "submit", "Prepared", "prepare", "solve_prepared",
    "submit_prepared", "ElasticMedium", "ElasticSource", "pstd_elastic_2d", "pstd_elastic_3d",
    "grid_size", "grid_spacing", "k_max", "total_grid_points",
]
