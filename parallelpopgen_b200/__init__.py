"""ParallelPopGen on B200: GO_Fish forward Wright-Fisher engine and Spectrum SFS path (sm_100a).

The product is the CUDA library libgofish_b200.so with the C ABI in include/gofish_b200.h and the
drop-in C++ headers in include/3P/.  This package builds it (`python -m parallelpopgen_b200.build`)
and exposes it to Python through ctypes (`Engine`).
"""
from ._capi import GoFishError, load, LIB_PATH, MAX_POPULATIONS, GEN_DTYPE, MSE_DTYPE  # noqa: F401
from .engine import (ConstantModel, Engine, constant_generations, new_mutation_count, replicate,  # noqa: F401
                     replicate_mse_pops, replicate_plain_generations, replicate_population)

__version__ = "0.1.0"
