"""os_d_b200: B200-native quantum-jump trajectory engine (drop-in for os_d's QJX QJ path).

The compute path is the native library libqjx_b200.so (sm_100a kernels behind a C ABI,
include/qjx_b200.h).  Importing this package never falls back to CPU code.
"""
from ._native import (QjxError, build_dimer, build_dimer_deep, build_dimer_gpu, mem_info, build_dimer_rk, build_floq2spins, build_floqnspins, build_floqspph, build_integrable, build_jcs, build_mbl, build_ps, dimer_generators, expm, fb_build_dimer, lib,  # noqa: F401
                      mbl_imbalance, measure_fp64_peak, random_observables)
from .engine import Engine, FBasis, autotune, fbasis_pure_state  # noqa: F401
