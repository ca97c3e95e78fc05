"""hammerhead_b200 -- B200 (sm_100a) backend for Hammerhead's planar WIDIM path.

Host layer over the C ABI of libhammerhead_b200.so (include/hammerhead_b200.h),
with the reference's public surface for the path:

    PIVParameters, multipass_parameters, effort_schedule   (src/types.jl, src/pipeline.jl)
    run_piv, piv_workspace, PIVWorkspace, PIVResult         (src/pipeline.jl, src/types.jl)
    run_piv_sequence (in-memory pairs), run_piv_batch,
    BatchRunner                                             (src/io.jl; batched device schedule)
    NCCLoss                                                 (adjoint of deformation + correlation)
    run_piv_ensemble                                        (src/ensemble.jl)
    validators: PeakRatioValidator, CorrelationMomentValidator,
                VelocityMagnitudeValidator, UniversalOutlierValidator
    error_statistics                                        (src/statistics.jl)
    synthetic                                               (src/synthetic_data.jl)

Everything numerical runs in the library on the GPU; there is no CPU path.
"""
from ._lib import ArgumentError, DimensionMismatch, HammerheadError, LIBPATH
from .params import (CorrelationMomentValidator, PeakRatioValidator, PIVParameters, UniversalOutlierValidator,
                     VelocityMagnitudeValidator, effort_schedule, multipass_parameters, parse_validator)
from .pipeline import (PhysicalScale, PIVResult, PIVWorkspace, check_backend_params, pass_grid, piv_workspace, run_piv,
                       with_scale)
from . import adjoint
from .adjoint import NCCLoss
from .batch import BatchRunner, run_piv_batch, run_piv_batch_stream, run_piv_sequence
from .ensemble import collective_reducer, run_piv_ensemble, shard_pairs
from .statistics import error_statistics, rms_error
from . import synthetic
from . import autotune as tuning
from .autotune import autotune

__all__ = [
    "ArgumentError", "DimensionMismatch", "HammerheadError", "LIBPATH", "PIVParameters", "multipass_parameters",
    "effort_schedule", "parse_validator", "PeakRatioValidator", "CorrelationMomentValidator",
    "VelocityMagnitudeValidator", "UniversalOutlierValidator", "PIVResult", "PIVWorkspace", "PhysicalScale",
    "piv_workspace", "run_piv", "pass_grid", "check_backend_params", "with_scale", "error_statistics", "rms_error",
    "synthetic", "BatchRunner", "run_piv_batch", "run_piv_batch_stream", "run_piv_sequence", "NCCLoss", "adjoint",
    "run_piv_ensemble",
    "autotune",
    "shard_pairs",
    "collective_reducer",
]
