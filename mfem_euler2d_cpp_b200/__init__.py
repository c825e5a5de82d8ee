"""B200-native engine for the per-Newton-update hot path of the frozen-HLL
DG / condensed-HDG 2-D Euler solver (YueWu2002/mfem_euler2d_cpp).

The compute path is the in-tree CUDA library ``lib/libeuler2d_cuda.so``
(include/euler2d_cuda.h); ``capi`` binds it with ctypes. There is no CPU
fallback.
"""
from . import capi  # noqa: F401
from .capi import Context, EngineError, Stepper, default_opts, load, simple_wave_desc  # noqa: F401

__all__ = ["capi", "Context", "EngineError", "Stepper", "default_opts", "load", "simple_wave_desc"]
