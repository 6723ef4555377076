/* herk_oracle.c -- CPU oracle for the correlator (test infrastructure only).
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * use this file, and only as the checker: the product never calls it.
 *
 * It restates the reference's host correlator:
 *   - QC decode: high nibble = Re, low nibble = Im, each sign-magnitude
 *     (bit 3 sign, bits 2:0 magnitude), as encode_int4 / decode_qc_byte in
 *     cutlass_interface/test_herk_int4.cu:41-45 and
 *     tests/visibility_pipeline_test.cpp:42-53.
 *   - cpu_herk (cutlass_interface/test_herk_int4.cu:51-70): for every j <= i,
 *     C[i(i+1)/2 + j] = sum_k A[i,k] * conj(A[j,k]); Im of the diagonal is 0.
 * Integer inputs are accumulated in int64, which is exact and equal to the
 * reference's FP64 result for every size used here.  Float inputs are
 * accumulated in FP64 like the reference.
 *
 * Build: oracle/Makefile -> oracle/liboracle.so.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static inline int qc_re(uint8_t b) {
  const int m = (b >> 4) & 7;
  return (b & 0x80) ? -m : m;
}
static inline int qc_im(uint8_t b) {
  const int m = b & 7;
  return (b & 0x08) ? -m : m;
}

/* Encode integer pairs in [-7, 7] to QC bytes (test_herk_int4.cu:41-45). */
void oracle_encode_qc(const int32_t* re, const int32_t* im, int64_t n, uint8_t* out) {
  for (int64_t t = 0; t < n; ++t) {
    const int r = re[t], i = im[t];
    const uint8_t rn = (uint8_t)(r < 0 ? (0x8 | ((-r) & 7)) : (r & 7));
    const uint8_t in = (uint8_t)(i < 0 ? (0x8 | ((-i) & 7)) : (i & 7));
    out[t] = (uint8_t)((rn << 4) | in);
  }
}

void oracle_decode_qc(const uint8_t* qc, int64_t n, int32_t* re, int32_t* im) {
  for (int64_t t = 0; t < n; ++t) {
    re[t] = qc_re(qc[t]);
    im[t] = qc_im(qc[t]);
  }
}

/* Rows [i_begin, i_end) of the packed lower triangle of channel b.
 * out receives, for each row i in the range, the (i+1) complex entries
 * j = 0..i as int64 (re, im) pairs, rows back to back. */
void oracle_herk_qc_rows(const uint8_t* qc, int N, int K, int b, int i_begin, int i_end,
                         int64_t* out) {
  const uint8_t* A = qc + (int64_t)b * N * K;
  int32_t* re = (int32_t*)malloc(sizeof(int32_t) * (size_t)N * K);
  int32_t* im = (int32_t*)malloc(sizeof(int32_t) * (size_t)N * K);
  oracle_decode_qc(A, (int64_t)N * K, re, im);
  const int64_t base = (int64_t)i_begin * (i_begin + 1) / 2;
#pragma omp parallel for schedule(dynamic)
  for (int i = i_begin; i < i_end; ++i) {
    const int32_t* ri = re + (int64_t)i * K;
    const int32_t* ii = im + (int64_t)i * K;
    int64_t* o = out + 2 * ((int64_t)i * (i + 1) / 2 - base);
    for (int j = 0; j <= i; ++j) {
      const int32_t* rj = re + (int64_t)j * K;
      const int32_t* ij = im + (int64_t)j * K;
      int64_t sr = 0, si = 0;
      for (int k = 0; k < K; ++k) {
        sr += (int64_t)ri[k] * rj[k] + (int64_t)ii[k] * ij[k];
        si += (int64_t)ii[k] * rj[k] - (int64_t)ri[k] * ij[k];
      }
      o[2 * j] = sr;
      o[2 * j + 1] = (i == j) ? 0 : si;
    }
  }
  free(re);
  free(im);
}

/* Whole batch: out = [batch][N(N+1)/2][2] int64. */
void oracle_herk_qc(const uint8_t* qc, int N, int K, int batch, int64_t* out) {
  const int64_t P = (int64_t)N * (N + 1) / 2;
  for (int b = 0; b < batch; ++b) oracle_herk_qc_rows(qc, N, K, b, 0, N, out + 2 * P * b);
}

/* Float input: a = [batch][N][K][2] double (re, im); out = [batch][P][2] double. */
void oracle_herk_c128(const double* a, int N, int K, int batch, double* out) {
  const int64_t P = (int64_t)N * (N + 1) / 2;
  for (int b = 0; b < batch; ++b) {
    const double* A = a + 2 * (int64_t)b * N * K;
    double* C = out + 2 * P * b;
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < N; ++i) {
      const double* ai = A + 2 * (int64_t)i * K;
      double* o = C + 2 * ((int64_t)i * (i + 1) / 2);
      for (int j = 0; j <= i; ++j) {
        const double* aj = A + 2 * (int64_t)j * K;
        double sr = 0.0, si = 0.0;
        for (int k = 0; k < K; ++k) {
          sr += ai[2 * k] * aj[2 * k] + ai[2 * k + 1] * aj[2 * k + 1];
          si += ai[2 * k + 1] * aj[2 * k] - ai[2 * k] * aj[2 * k + 1];
        }
        o[2 * j] = sr;
        o[2 * j + 1] = (i == j) ? 0.0 : si;
      }
    }
  }
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
