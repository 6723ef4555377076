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
// and, into oracle/_ref/ref_extract_kernels.inc, the XEngine and imaging
// helpers (device code of the reference, compiled here for the host with
// empty stand-ins for the CUDA qualifiers):
//   DataPromote           include/kernels/promote_data.cuh:70-88
//   HermToTri             include/kernels/tri_from_herm.cuh:28-73
//   C_LIGHT, tri_decode, uv_cell   include/kernels/imaging_kernels.cuh:24-46
//   promote_to_float      tests/xengine_test.cpp:162-167
// Test infrastructure only; the product never links it.
#include <cmath>
#include <complex>
#include <cstdint>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "ref_extract.inc"

namespace refk {
using std::sqrt;
template <typename T> using complex = std::complex<T>;
// argument blocks with the members the functors read
template <typename T> struct PromoteArgHost {
  using Prec = T;
  T* output;
  const uint8_t* input;
};
template <typename T> struct HermToTriArgHost {
  using real = T;
  complex<T>* output;
  const complex<T>* input;
  unsigned long long N;
  unsigned long long N_batch;
};
#define __device__
#define __host__
#define __forceinline__ inline
#define KERNEL_FILE "ref_extract_kernels.inc"
#define MASK1 0x0F
#define MASK2 0xF0
#include "ref_extract_kernels.inc"
#undef __device__
#undef __host__
#undef __forceinline__
#undef KERNEL_FILE
#undef MASK1
#undef MASK2
}  // namespace refk

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

// DataPromote (the XEngine's promoteData functor) over n QC bytes:
// out[2i] = Re, out[2i+1] = Im as doubles.
void ref_data_promote(const uint8_t* in, int64_t n, double* out) {
  refk::PromoteArgHost<double> a{out, in};
  refk::DataPromote<refk::PromoteArgHost<double>> f(a);
  for (int64_t i = 0; i < n; ++i) f(int(i));
}

// The XEngine test's host decode, promote_to_float<double>.
void ref_promote_to_float(const uint8_t* in, int64_t n, double* out) {
  std::vector<unsigned char> tmp(in, in + n);
  refk::promote_to_float<double>(out, tmp.data(), uint64_t(n));
}

// HermToTri over `batches` full n x n complex128 matrices (row-major, back
// to back) -> packed upper triangles (n(n+1)/2 complex128 each).
void ref_herm_to_tri(const double* in, int n, int batches, double* out) {
  refk::HermToTriArgHost<double> a;
  a.input = reinterpret_cast<const std::complex<double>*>(in);
  a.output = reinterpret_cast<std::complex<double>*>(out);
  a.N_batch = static_cast<unsigned long long>(n) * n;
  a.N = a.N_batch * batches;
  refk::HermToTri<refk::HermToTriArgHost<double>> f(a);
  for (unsigned long long i = 0; i < a.N; ++i) f(int(i));
}

// tri_decode (packed lower index -> row, col) for k = 0 .. n-1.
void ref_tri_decode(int64_t n, int32_t* row, int32_t* col) {
  for (int64_t k = 0; k < n; ++k) {
    int r, c;
    refk::tri_decode(int(k), r, c);
    row[k] = r;
    col[k] = c;
  }
}

// uv_cell for n baselines (u, v in metres) at one frequency.
void ref_uv_cell(const float* u, const float* v, int64_t n, double freq, float cell,
                 float half_ng, float* ul, float* vl, int32_t* iu, int32_t* iv) {
  for (int64_t k = 0; k < n; ++k) {
    int a, b;
    refk::uv_cell(u[k], v[k], freq, cell, half_ng, ul[k], vl[k], a, b);
    iu[k] = a;
    iv[k] = b;
  }
}

int ref_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
}
