// shim_check.cpp -- a caller written against the reference's C++ HERK API
// (cutlass_gemm_api::CutlassComplexGemm and the ggp:: engine-boundary
// functions), compiled unchanged against this library's drop-in header and
// linked to libftdx.so.  Exit status 0 when every result matches a CPU
// correlator bit-exactly.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "cutlass_gemm_api.h"
#include "ftdx.h"
#include "ggp_blas_interface.h"

namespace ggp {
void initCutlassApi(int kernel_tune_verbosity, const char* kernel_tune_cache_path,
                    const char* strategy_tune_cache_path, bool herk_tune,
                    int strategy_tune_verbosity = 1);
int herkBatchedCutlassQC(const void* qc_data, void* tri_output, int N, int K, int batch,
                         cudaStream_t stream = 0);
int herkBatchedCutlassQC_FP16(const void* qc_data, void* tri_output, int N, int K, int batch,
                              cudaStream_t stream = 0);
}  // namespace ggp

using namespace cutlass_gemm_api;

static int nib(uint8_t n) { return (n & 8) ? -int(n & 7) : int(n & 7); }

int main() {
  const int N = 200, K = 77, B = 3;
  const size_t P = size_t(N) * (N + 1) / 2;
  std::vector<uint8_t> qc(size_t(B) * N * K);
  uint32_t x = 12345u;
  for (auto& v : qc) {
    x = x * 1664525u + 1013904223u;
    v = uint8_t(x >> 24);
  }
  std::vector<float> ref(B * P * 2);
  for (int b = 0; b < B; ++b)
    for (int i = 0; i < N; ++i)
      for (int j = 0; j <= i; ++j) {
        long long sr = 0, si = 0;
        for (int k = 0; k < K; ++k) {
          const uint8_t a = qc[(size_t(b) * N + i) * K + k], c = qc[(size_t(b) * N + j) * K + k];
          const int ar = nib(a >> 4), ai = nib(a & 15), cr = nib(c >> 4), ci = nib(c & 15);
          sr += ar * cr + ai * ci;
          si += ai * cr - ar * ci;
        }
        const size_t e = b * P + size_t(i) * (i + 1) / 2 + j;
        ref[2 * e] = float(sr);
        ref[2 * e + 1] = (i == j) ? 0.f : float(si);
      }
  void *d_qc = nullptr, *d_c = nullptr;
  cudaMalloc(&d_qc, qc.size());
  cudaMalloc(&d_c, B * P * 8);
  cudaMemcpy(d_qc, qc.data(), qc.size(), cudaMemcpyHostToDevice);
  std::vector<float> got(B * P * 2);
  int fails = 0;

  ggp::initCutlassApi(0, nullptr, nullptr, false, 0);
  if (ggp::herkBatchedCutlassQC(d_qc, d_c, N, K, B) != 0) ++fails;
  cudaMemcpy(got.data(), d_c, B * P * 8, cudaMemcpyDeviceToHost);
  if (got != ref) {
    printf("ggp::herkBatchedCutlassQC mismatch\n");
    ++fails;
  }

  CutlassComplexGemm api;
  cudaMemset(d_c, 0, B * P * 8);
  int rc = api.herk(d_qc, d_c, N, K, B, InputPrecision::INT4, ComputePrecision::FP8,
                    OutputPrecision::FP32, OutputFormat::PackedTriangle, 1.0f, 0.0f, nullptr,
                    false);
  cudaMemcpy(got.data(), d_c, B * P * 8, cudaMemcpyDeviceToHost);
  if (rc != 0 || got != ref) {
    printf("CutlassComplexGemm::herk rc=%d mismatch=%d\n", rc, int(got != ref));
    ++fails;
  }
  // FP6 compute on INT4 input: E3M2 operands, exact, so the same triangles
  cudaMemset(d_c, 0, B * P * 8);
  rc = api.herk(d_qc, d_c, N, K, B, InputPrecision::INT4, ComputePrecision::FP6,
                OutputPrecision::FP32, OutputFormat::PackedTriangle, 1.0f, 0.0f, nullptr, false);
  cudaMemcpy(got.data(), d_c, B * P * 8, cudaMemcpyDeviceToHost);
  if (rc != 0 || got != ref) {
    printf("CutlassComplexGemm::herk FP6 rc=%d mismatch=%d\n", rc, int(got != ref));
    ++fails;
  }
  // FP4 compute is not provided by this entry point: a non-zero status, no throw
  if (api.herk(d_qc, d_c, N, K, B, InputPrecision::INT4, ComputePrecision::FP4,
               OutputPrecision::FP32) == 0) {
    printf("FP4 request was accepted\n");
    ++fails;
  }
  // graph replay as set_direct_herk_graph asks: the second identical call
  // replays the captured graph, same triangles
  {
    CutlassComplexGemm g;
    g.set_direct_herk_graph(true);
    for (int rep = 0; rep < 2; ++rep) {
      cudaMemset(d_c, 0, B * P * 8);
      rc = g.herk(d_qc, d_c, N, K, B, InputPrecision::INT4, ComputePrecision::FP8,
                  OutputPrecision::FP32, OutputFormat::PackedTriangle, 1.0f, 0.0f, nullptr, false);
      cudaMemcpy(got.data(), d_c, B * P * 8, cudaMemcpyDeviceToHost);
      if (rc != 0 || got != ref) {
        printf("graph replay %d rc=%d mismatch=%d\n", rep, rc, int(got != ref));
        ++fails;
      }
    }
    const int graphs = ftdx_graph_count(static_cast<ftdx_handle>(g.native_handle()));
    if (graphs < 1) {
      printf("set_direct_herk_graph(true) captured no graph (%d)\n", graphs);
      ++fails;
    }
    g.set_direct_herk_graph(false);
    if (ftdx_graph_count(static_cast<ftdx_handle>(g.native_handle())) != 0) {
      printf("set_direct_herk_graph(false) kept graphs\n");
      ++fails;
    }
  }
  // both forced kernels (single CTA, CTA pair) give the same triangles
  for (HerkMode mode : {HerkMode::ForceDirect, HerkMode::ForceBaseline, HerkMode::Auto}) {
    CutlassComplexGemm m;
    m.set_herk_mode(mode);
    cudaMemset(d_c, 0, B * P * 8);
    rc = m.herk(d_qc, d_c, N, K, B, InputPrecision::INT4, ComputePrecision::FP8,
                OutputPrecision::FP32);
    cudaMemcpy(got.data(), d_c, B * P * 8, cudaMemcpyDeviceToHost);
    if (rc != 0 || got != ref) {
      printf("herk mode %d rc=%d mismatch=%d\n", int(mode), rc, int(got != ref));
      ++fails;
    }
  }
  // quda::stridedBatchGEMMCutlass, HERK pattern: small integers (exact in FP16
  // and E4M3, integer sums below 2048 exact in FP16) give the same triangles
  {
    const int n = 40, k = 24, nb = 2;
    std::vector<float> a(size_t(nb) * n * k * 2);
    for (auto& v : a) {
      x = x * 1664525u + 1013904223u;
      v = float(int(x >> 29) - 4);  // -4..3
    }
    const size_t p = size_t(n) * (n + 1) / 2;
    std::vector<float> want(nb * p * 2), have(nb * p * 2);
    for (int b = 0; b < nb; ++b)
      for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
          double sr = 0, si = 0;
          for (int t = 0; t < k; ++t) {
            const float* u = &a[((size_t(b) * n + i) * k + t) * 2];
            const float* w = &a[((size_t(b) * n + j) * k + t) * 2];
            sr += double(u[0]) * w[0] + double(u[1]) * w[1];
            si += double(u[1]) * w[0] - double(u[0]) * w[1];
          }
          const size_t e = b * p + size_t(i) * (i + 1) / 2 + j;
          want[2 * e] = float(sr);
          want[2 * e + 1] = i == j ? 0.f : float(si);
        }
    void *d_a = nullptr, *d_t = nullptr;
    cudaMalloc(&d_a, a.size() * 4);
    cudaMalloc(&d_t, have.size() * 4);
    cudaMemcpy(d_a, a.data(), a.size() * 4, cudaMemcpyHostToDevice);
    QudaBLASParam bp{};
    bp.struct_size = sizeof(bp);
    bp.trans_a = QUDA_BLAS_OP_C;
    bp.trans_b = QUDA_BLAS_OP_N;
    bp.m = bp.n = n;
    bp.k = k;
    bp.batch_count = nb;
    bp.data_type = QUDA_BLAS_DATATYPE_C;
    const long long flops = quda::stridedBatchGEMMCutlass(d_a, d_a, d_t, bp, QUDA_CUDA_FIELD_LOCATION);
    cudaMemcpy(have.data(), d_t, have.size() * 4, cudaMemcpyDeviceToHost);
    if (flops != 8LL * n * n * k * nb || have != want) {
      printf("quda::stridedBatchGEMMCutlass flops=%lld mismatch=%d\n", flops, int(have != want));
      ++fails;
    }
    cudaFree(d_a);
    cudaFree(d_t);
  }
  api.init_herk(N, K, B);
  api.end_herk();
  CutlassComplexGemm::print_build_info();
  cudaFree(d_qc);
  cudaFree(d_c);
  printf("%s\n", fails ? "FAIL" : "OK");
  return fails ? 1 : 0;
}
