"""ope_b200 — B200-native (sm_100a) Heston/Bates characteristic-function pricer.

A drop-in for the CPU pricing path of the reference Rust crate
(options_pricing_engine): the same entry points over a C ABI
(include/ope.h), computed by hand-written FP64 CUDA kernels.
"""
from .api import *  # noqa: F401,F403
from .api import __all__  # noqa: F401
