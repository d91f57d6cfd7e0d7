"""B200-native (sm_100a) LES time step for the LES_Halo reference.

The hot path lives in liblesb200.so (CUDA kernels behind the C ABI of
include/les_abi.h); this package is the thin host-side mirror of the
reference's driver: Fortran-layout arrays, the synthetic benchmark inputs,
and ``GpuLes`` (initialise_LES_kernel / run_LES_kernel).
"""
from . import abi, fields
from .model import (Ensemble, GpuAdjoint, GpuLes, LesCase, default_params, set_drag, synth_cfg,
                    synthetic_case, tke_forward, tke_gradient, tke_reverse)

__all__ = ["abi", "fields", "Ensemble", "GpuAdjoint", "GpuLes", "LesCase", "default_params", "set_drag", "synth_cfg",
           "synthetic_case", "tke_forward", "tke_gradient", "tke_reverse"]
