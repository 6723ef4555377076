"""ftd_b200 -- B200 (sm_100a) X-engine correlator, a drop-in for the HERK
entry points of cpviolator/ftd.

The compute path is ``libftdx.so`` (hand-written tcgen05/TMA CUDA behind the
C ABI in ``include/ftdx.h``).  Importing this package does not need a GPU;
calling into the library does, and fails loudly without one.
"""
from ._lib import FtdxError, LIB_PATH, load  # noqa: F401
from .herk import (Correlator, Pipeline, herk_batched_cutlass_fp16,  # noqa: F401
                   herk_batched_cutlass_qc, herk_batched_cutlass_qc_fp16, init_cutlass_api,
                   tri_size)

__version__ = "0.1.0"
