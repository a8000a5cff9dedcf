"""rvvlasparse_b200 — SpMV for NVIDIA B200 (sm_100a) with RVVLASparse's API.

The compute path is the CUDA library ``lib/librvvla_b200.so`` (C ABI in
``include/rvvla.h``); this package is its Python binding and the mirror of the
reference's ``sparse_mv`` / ``convert`` / ``spMtx*`` interface.  Importing the
package does not touch the GPU; the first call that needs the library loads it
and fails loudly if it has not been built.
"""
from ._capi import RvvlaError, load  # noqa: F401
from .formats import (  # noqa: F401
    SPARSE_MATRIX_MV_ALL_STAGES,
    SPARSE_MATRIX_MV_GET_RESULTS,
    SPARSE_MATRIX_MV_MULT,
    SPARSE_MATRIX_MV_PREPARATION,
    SPARSE_OPERATION_NON_TRANSPOSE,
    SPARSE_OPERATION_TRANSPOSE,
    convert,
    convertParams,
    sparse_matrix_descr,
    sparse_matrix_status,
    sparse_mv,
    sparse_mv_mixed,
    spMtxCRS,
    spMtxCSR5,
    spMtxCVR,
    spMtxHCSR,
    spMtxLAV,
    spMtxSELL_C_Sigma,
    spMtxVHCC,
    spMtxVNEC,
)

__version__ = "0.1.0"
