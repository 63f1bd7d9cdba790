"""zldsp_fft_b200 — a B200 (sm_100a) FFT engine that is a drop-in for
zldsp::fft::CFFT<F> and RFFT<F> (ZL-Audio/zldsp_fft).

Layers:
  include/zlfft.h                 C ABI (the drop-in boundary)
  include/zldsp_fft_cuda/*.hpp    C++ drop-in classes over the C ABI
  zldsp_fft_b200/csrc/*.cu        CUDA kernels + C ABI implementation
  zldsp_fft_b200/fft.py           Python mirror of the reference's classes
"""
from . import _capi
from ._capi import (AOS, BACKWARD, C2C, F32, F64, FORWARD, FORWARD_SQR_MAG, MODE_PLAIN,
                    MODE_FAST, MODE_HOST, MODE_TC_FP16, MODE_TUNED, R2C, SCHED_GRAPH, SCHED_PER_ORDER,
                    SCHED_PERSISTENT, SOA, ZlfftError)
from .fft import (CFFT, RFFT, MixedBatch, Plan, autotune, host_switch_order, tuning, tuning_clear, tuning_load,
                  tuning_save)

__all__ = [
    "CFFT", "RFFT", "Plan", "MixedBatch", "ZlfftError", "AOS", "SOA", "C2C", "R2C", "F32", "F64", "FORWARD", "BACKWARD",
    "FORWARD_SQR_MAG", "MODE_PLAIN", "MODE_TC_FP16", "MODE_TUNED", "MODE_FAST",
    "MODE_HOST", "SCHED_PER_ORDER", "SCHED_PERSISTENT", "SCHED_GRAPH", "autotune", "host_switch_order", "tuning",
    "tuning_save", "tuning_load", "tuning_clear",
]
