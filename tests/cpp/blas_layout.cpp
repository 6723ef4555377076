// blas_layout.cpp -- prints sizeof and the offset of every member of
// QudaBLASParam, declared either by GGP's own header (-DUSE_GGP_HEADER, the
// reference's include/ggp.h) or by this library's ggp_blas_interface.h, and
// calls quda::stridedBatchGEMMCutlass with a non-HERK pattern (which must
// return -1 without touching the GPU), so that linking it against libftdx.so
// checks the exported symbol.
#include <cstddef>
#include <cstdio>
#ifdef USE_GGP_HEADER
#include <ggp.h>
namespace quda {
long long stridedBatchGEMMCutlass(void* A_data, void* B_data, void* C_data, QudaBLASParam param,
                                  QudaFieldLocation location);
}
#else
#include "ggp_blas_interface.h"
#endif

#define OFF(m) std::printf(#m " %zu\n", offsetof(QudaBLASParam, m))

int main(int argc, char**) {
  std::printf("size %zu\n", sizeof(QudaBLASParam));
  OFF(struct_size); OFF(blas_type); OFF(location); OFF(trans_a); OFF(trans_b);
  OFF(m); OFF(n); OFF(k); OFF(lda); OFF(ldb); OFF(ldc);
  OFF(a_offset); OFF(b_offset); OFF(c_offset); OFF(a_stride); OFF(b_stride); OFF(c_stride);
  OFF(alpha); OFF(beta); OFF(inv_mat_size); OFF(batch_count); OFF(engine); OFF(data_type);
  OFF(data_order); OFF(stream_idx);
  std::printf("enums %d %d %d %d\n", int(QUDA_BLAS_OP_C), int(QUDA_BLAS_DATATYPE_C),
              int(QUDA_CUDA_FIELD_LOCATION), int(QUDA_BLAS_ENGINE_CUTLASS));
  if (argc > 1) {  // call through the library: a real GEMM pattern is refused with -1
    QudaBLASParam p{};
    p.trans_a = QUDA_BLAS_OP_N;
    p.trans_b = QUDA_BLAS_OP_N;
    p.m = p.n = p.k = 4;
    p.batch_count = 1;
    p.data_type = QUDA_BLAS_DATATYPE_C;
    int x = 0;
    std::printf("call %lld\n",
                quda::stridedBatchGEMMCutlass(&x, &x, &x, p, QUDA_CUDA_FIELD_LOCATION));
  }
  return 0;
}
