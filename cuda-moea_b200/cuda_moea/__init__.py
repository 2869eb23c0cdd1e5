"""B200 implementation of the CUDA-MOEA generation hot path.

Public API of CUDA-MOEA (python/cuda_moea/__init__.py): NSGA3, RVEA, Algorithm,
AlgorithmBuilder, Population, Result, the strategy specifications and the
built-in problems.  The computation runs in libmoea_b200.so (C ABI in
include/moea_b200.h); ``cuda_moea.stages`` exposes the individual stages.
"""
import torch  # noqa: F401  -- CUDA tensors of the results

from .algorithm import Algorithm, AlgorithmBuilder, NSGA3, Population, RVEA, Result
from .batch import Batch
from . import metrics
from . import problem as _problem
from .problem import *  # noqa: F401,F403
from ._specs import (
    AdaptiveRVEADirections, CudaConfig, DasDennisDirections,
    NSGA3EnvironmentSelector, NoMutation, PolynomialMutation,
    PythonCrossover, PythonEnvironmentSelector, PythonMating, PythonMutation,
    PythonReferenceDirections, RandomMating, RVEAEnvironmentSelector, SBX,
    TournamentMating, UserDefinedDirections, two_layer_directions,
)

__version__ = "0.2.0+b200"

__all__ = [
    "Algorithm", "AlgorithmBuilder", "NSGA3", "RVEA", "Population", "Result", "Batch",
    "CudaConfig", "SBX", "PolynomialMutation", "NoMutation",
    "RandomMating", "TournamentMating", "DasDennisDirections",
    "AdaptiveRVEADirections", "UserDefinedDirections",
    "NSGA3EnvironmentSelector", "RVEAEnvironmentSelector",
    "PythonProblem", "PythonMating", "PythonCrossover", "PythonMutation",
    "PythonReferenceDirections", "PythonEnvironmentSelector", "NativeProblem",
    "two_layer_directions",
] + _problem.__all__


def __getattr__(name):
    # imported on first use, so `python -m cuda_moea.native` runs the module once
    if name == "NativeProblem":
        from .native import NativeProblem
        return NativeProblem
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
