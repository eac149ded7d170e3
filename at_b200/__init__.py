"""at_b200: B200-native tracking engine for AT (Accelerator Toolbox) lattices.

A drop-in for pyat's ``atpass``/``gpupass``/``elempass`` tracking calls:
lattices are compiled to a flat element table and tracked by a persistent
sm_100a CUDA kernel in FP64 behind the C ABI of ``include/atb200.h``.
"""
from . import elements
from .lattice import CompiledLattice, compile_lattice
from .tracking import atpass, elempass, gpuinfo, gpupass, reset_cache, reset_rng

__all__ = ["atpass", "gpupass", "elempass", "gpuinfo", "reset_cache", "reset_rng",
           "compile_lattice", "CompiledLattice", "elements"]
__version__ = "0.1.0"
