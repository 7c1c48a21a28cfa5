"""B200-native tile-low-rank Cholesky engine with HiCMA-PaRSEC's operator surface.

The compute path is the CUDA library ``lib/libhicma_tlr.so`` (C ABI declared in
``include/hicma_tlr.h``); ``tlr`` binds it through ctypes.
"""
from .tlr import (Context, Problem, TLRMatrix, TLRError, STARSH_gen, HiCMA_dpotrf_L,  # noqa: F401
                  parsec_band_size_auto_tuning, HICMA_get_stat2, load_library, points, points_mesh,
                  LOWER, UPPER, KIND_RANDTLR, KIND_ED_SIN_2D, KIND_SQEXP_2D, KIND_SQEXP_3D, KIND_EXP_3D,
                  KIND_ED_SIN_3D, KIND_MD_VIRUS, KIND_MD_CUBE, PREC_FP64, PREC_MIXED)
