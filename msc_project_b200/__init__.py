"""B200-native Wilson-flow engine for pure SU(3) lattice gauge fields.

A drop-in for the LGF reference's FlowSavedGaugeConfigurations path: CUDA
kernels for sm_100a behind the C ABI in include/lgf_b200.h (liblgf_b200.so),
the reference's C++ workflow entry points in include/lgf_dropin.h, and this
Python mirror for tests and benchmarks.
"""
from ._capi import LIB_PATH, load  # noqa: F401
from .lgf import (FP32MIXED, FP64, Context, FlowParameters, FlowResult, FlowSavedGaugeConfigurations,  # noqa: F401
                  GenerateHeatBathGaugeConfigurations, HBParameters,
                  Job, Lattice, LGFError, MeasureFlowedGaugeConfigurations, MeasureQdensityDistribution, ResumeFlowedConfiguration, Server,
                  SimulationParameters, configure, volume)
