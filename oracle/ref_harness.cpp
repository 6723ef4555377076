// ref_harness.cpp -- C entry points around the reference's own host-side
// correlator code, for pinning the oracle and for the timed CPU baseline.
//
// The functions below are NOT restated here: oracle/build_ref.sh extracts
// them verbatim from the reference tree at build time into the git-ignored
// oracle/_ref/ref_extract.inc, which this file includes:
//   encode_int4           cutlass_interface/test_herk_int4.cu:41-45
//   cpu_herk              cutlass_interface/test_herk_int4.cu:51-70
//   decode_qc_byte        tests/visibility_pipeline_test.cpp:42-53
//   cpu_herk_batch_first  tests/visibility_pipeline_test.cpp:136-168
//   cpu_herk_ftd          tests/visibility_pipeline_test.cpp:55-96
// Test infrastructure only; the product never links it.
#include <complex>
#include <cstdint>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "ref_extract.inc"

extern "C" {

// Input generation of test_herk_int4.cu:313-321: std::mt19937(seed),
// uniform_int_distribution(-7, 7), Re drawn before Im for every element.
void ref_gen_int4(uint32_t seed, int64_t n, uint8_t* qc) {
  std::mt19937 rng(seed);
  std::uniform_int_distribution<int> dist(-7, 7);
  for (int64_t i = 0; i < n; ++i) {
    const int re = dist(rng);
    const int im = dist(rng);
    qc[i] = encode_int4(re, im);
  }
}

void ref_encode(const int32_t* re, const int32_t* im, int64_t n, uint8_t* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = encode_int4(re[i], im[i]);
}

// The reference's cpu_herk on QC input decoded with decode_qc_byte.
// out = [batch][N(N+1)/2][2] double.
void ref_cpu_herk(const uint8_t* qc, int N, int K, int batch, double* out) {
  const int64_t per_A = int64_t(N) * K;
  const int64_t P = int64_t(N) * (N + 1) / 2;
  std::vector<std::complex<double>> A(per_A);
  std::vector<std::complex<double>> C(P);
  for (int b = 0; b < batch; ++b) {
    for (int64_t t = 0; t < per_A; ++t) {
      float re, im;
      decode_qc_byte(qc[b * per_A + t], re, im);
      A[t] = std::complex<double>(re, im);
    }
    cpu_herk(A, C, N, K);
    for (int64_t p = 0; p < P; ++p) {
      out[2 * (b * P + p)] = C[p].real();
      out[2 * (b * P + p) + 1] = C[p].imag();
    }
  }
}

// The reference's batch-first single-thread correlator; out = [batch][P][2] float.
void ref_cpu_herk_batch_first(const uint8_t* qc, int N, int K, int batch, float* out) {
  const int64_t P = int64_t(N) * (N + 1) / 2;
  for (int b = 0; b < batch; ++b) cpu_herk_batch_first(qc, b, N, K, out + 2 * P * b);
}

// The reference's FTD-layout correlator for one batch; out = [P][2] float.
void ref_cpu_herk_ftd(const uint8_t* qc, int batch_idx, int n_ant, int n_chan, int n_pol,
                      int n_time_inner, int n_time, float* out) {
  cpu_herk_ftd(qc, batch_idx, n_ant, n_chan, n_pol, n_time_inner, n_time, out);
}

int ref_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
}
