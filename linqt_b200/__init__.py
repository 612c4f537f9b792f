"""linqt_b200 -- LinQT's Chebyshev-moment hot path on the NVIDIA B200.

The compute path is liblinqt_gpu.so (hand-written CUDA for sm_100a behind the
C ABI of include/linqt_gpu.h); this package is its Python host binding plus the
LinQT file formats and seeded synthetic inputs.  Importing it does not load the
library; the first call does, and fails loudly if the library is not built.
"""
from ._lib import LinqtError, load  # noqa: F401
from .core import (FORMAT_AUTO, FORMAT_CSR, FORMAT_SELL, FORMAT_LOCAL, OP_C128, OP_C64, KUBO_BASTIN, KUBO_GREENWOOD, PREC_FP32, PREC_FP64, PREC_MIXED, PREC_MIXED_FAST, PREC_MIXED_TF32,  # noqa: F401
                   STORAGE_GENERAL, STORAGE_HERMITIAN_UPPER, W2S_OPERATORS, Operator, Session, TBModel, bastin_from_moments,
                   dos_from_moments, spectral_function_from_moments, jackson1d, jackson2d, kubo_bastin, kubo_bastin_dev, kubo_bastin_host_ptr,
                   kubo_fft, kubo_fft_dev, make_opts, moments1d,
                   moments1d_dev, moments1d_noalloc, moments1d_nonorth, moments1d_nonorth_dev, moments2d, moments2d_dev, moments_td, moments_td_dev, time_correlation_from_moments,
                   random_phase_states_dev, locality_order,
                   kubo_from_moments, moments1d_realisations, moments1d_realisations_dev, GRID_UNIFORM, GRID_CHEBYSHEV, GRID_CHEBYSHEV_ASCENDING)

__all__ = [
    "OP_C128", "OP_C64", "LinqtError", "load", "Operator", "Session", "moments1d", "moments1d_dev", "moments1d_noalloc", "moments1d_nonorth", "moments1d_nonorth_dev", "moments2d", "moments2d_dev",
    "kubo_fft", "kubo_fft_dev", "kubo_bastin", "kubo_bastin_dev", "kubo_bastin_host_ptr", "dos_from_moments", "spectral_function_from_moments", "bastin_from_moments", "jackson1d", "jackson2d",
    "make_opts", "PREC_FP64", "PREC_MIXED", "PREC_FP32", "PREC_MIXED_TF32", "PREC_MIXED_FAST", "KUBO_GREENWOOD", "KUBO_BASTIN",
    "STORAGE_HERMITIAN_UPPER", "STORAGE_GENERAL", "random_phase_states_dev", "kubo_from_moments", "moments1d_realisations", "moments1d_realisations_dev",
    "moments_td", "moments_td_dev", "time_correlation_from_moments", "TBModel", "W2S_OPERATORS",
    "FORMAT_CSR", "FORMAT_SELL", "FORMAT_AUTO", "FORMAT_LOCAL", "locality_order",
]
