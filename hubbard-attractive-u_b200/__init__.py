"""B200 (sm_100a) DQMC sweep of the attractive-U Hubbard model.

A drop-in for the sweep of JefferyWangSH/hubbard-attractive-U behind the C ABI of
include/hubbard_b200.h. This package holds the CUDA sources (csrc/), the build recipe of
the in-tree shared library, its ctypes binding and the host-side mirror of the
reference's configuration and measurement schedule.
"""
from .capi import (Engine, HqError, lib, EXPORTS, SWEEP_UP, SWEEP_DOWN, SWEEP_DYNAMIC, SWEEP_MEASURE,
                   SWEEP_SNAPSHOT, SWEEP_LOG_RATIOS, G_CURRENT, G_TT, G_T0, G_0T, EXPK_DENSE,
                   EXPK_SEPARABLE, EXPK_AUTO, SWEEP_LAUNCHES, SWEEP_PERSISTENT)

__all__ = ["Engine", "HqError", "lib", "EXPORTS", "SWEEP_UP", "SWEEP_DOWN", "SWEEP_DYNAMIC", "SWEEP_MEASURE",
           "SWEEP_SNAPSHOT", "SWEEP_LOG_RATIOS", "G_CURRENT", "G_TT", "G_T0", "G_0T", "EXPK_DENSE",
           "EXPK_SEPARABLE", "EXPK_AUTO", "SWEEP_LAUNCHES", "SWEEP_PERSISTENT"]
