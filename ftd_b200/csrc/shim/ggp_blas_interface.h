// ggp_blas_interface.h -- the BLAS types of GGP's public header that the
// XEngine's BLAS route passes to quda::stridedBatchGEMMCutlass
// (lib/cutlass_interface.cu:316-381, called from
// lib/interface/blas_interface.cpp:157).  The struct tag, the enum tags, the
// enumerator values and the member order and types are those of
// include/ggp.h:27-62 and include/enum_ggp.h:40-113, so that the C++ mangled
// name of stridedBatchGEMMCutlass and the by-value layout of QudaBLASParam
// match the reference's: a GGP build keeps including its own ggp.h and links
// this library's symbol unchanged.  This header is for callers without
// ggp.h (the tests); do not include both.
#pragma once
#include <cstddef>

#include "cutlass_gemm_api.h"  // FTDX_SHIM_API

#ifndef QUDA_INVALID_ENUM
#define QUDA_INVALID_ENUM (-0x7fffffff - 1)
#endif

extern "C" {
typedef enum QudaFieldLocation_s {
  QUDA_CPU_FIELD_LOCATION = 1,
  QUDA_CUDA_FIELD_LOCATION = 2,
  QUDA_INVALID_FIELD_LOCATION = QUDA_INVALID_ENUM
} QudaFieldLocation;

typedef enum QudaBLASType_s {
  QUDA_BLAS_GEMM = 0,
  QUDA_BLAS_LU_INV = 1,
  QUDA_BLAS_INVALID = QUDA_INVALID_ENUM
} QudaBLASType;

typedef enum QudaBLASOperation_s {
  QUDA_BLAS_OP_N = 0,
  QUDA_BLAS_OP_T = 1,
  QUDA_BLAS_OP_C = 2,
  QUDA_BLAS_OP_INVALID = QUDA_INVALID_ENUM
} QudaBLASOperation;

typedef enum QudaBLASDataType_s {
  QUDA_BLAS_DATATYPE_S = 0,
  QUDA_BLAS_DATATYPE_D = 1,
  QUDA_BLAS_DATATYPE_C = 2,
  QUDA_BLAS_DATATYPE_Z = 3,
  QUDA_BLAS_DATATYPE_H = 4,
  QUDA_BLAS_DATATYPE_HC = 5,
  QUDA_BLAS_DATATYPE_QC = 6,
  QUDA_BLAS_DATATYPE_INVALID = QUDA_INVALID_ENUM
} QudaBLASDataType;

typedef enum QudaBLASDataOrder_s {
  QUDA_BLAS_DATAORDER_ROW = 0,
  QUDA_BLAS_DATAORDER_COL = 1,
  QUDA_BLAS_DATAORDER_INVALID = QUDA_INVALID_ENUM
} QudaBLASDataOrder;

typedef enum QudaBLASEngine_s {
  QUDA_BLAS_ENGINE_CUBLAS = 0,
  QUDA_BLAS_ENGINE_CUTLASS = 1,
  QUDA_BLAS_ENGINE_TCC = 2,
  QUDA_BLAS_ENGINE_INVALID = QUDA_INVALID_ENUM
} QudaBLASEngine;

typedef struct QudaBLASParam_s {
  size_t struct_size;
  QudaBLASType blas_type;
  QudaFieldLocation location;
  QudaBLASOperation trans_a;
  QudaBLASOperation trans_b;
  int m, n, k;
  int lda, ldb, ldc;
  int a_offset, b_offset, c_offset;
  int a_stride, b_stride, c_stride;
  double _Complex alpha;
  double _Complex beta;
  int inv_mat_size;
  int batch_count;
  QudaBLASEngine engine;
  QudaBLASDataType data_type;
  QudaBLASDataOrder data_order;
  int stream_idx;
} QudaBLASParam;
}

namespace quda {
// HERK pattern (A == B, trans_a = QUDA_BLAS_OP_C, trans_b = QUDA_BLAS_OP_N,
// m == n, QUDA_BLAS_DATATYPE_C): packed lower triangles of C = A A^H for
// [batch_count][n][k] complex64 A, with the reference's FP16 narrowing
// arithmetic; returns the flop count 8*m*n*k*batch, or -1 for any other
// pattern or on failure (the reference stops in errorQuda there).  Blocks
// until the result is in C, as the reference's cudaDeviceSynchronize does.
FTDX_SHIM_API long long stridedBatchGEMMCutlass(void* A_data, void* B_data, void* C_data,
                                                QudaBLASParam param, QudaFieldLocation location);
}  // namespace quda
