// pipeline.cu -- host-to-host correlation pipeline (ftdx_pipeline_*): H2D of
// raw QC payloads, correlation and D2H of the packed triangles on four
// streams (H2D, correlation, two D2H halves: two copy engines) with two
// device buffer sets.  Replaces the CUTLASS branch of
// ggp::VisibilityPipeline::correlate / correlate_pipelined
// (lib/visibility_pipeline.cu:253-308, 483-549), which copies through one
// pinned staging buffer and waits for each payload's D2H before the next.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "context.h"

struct ftdx_pipeline {
  ftdx_handle h = nullptr;
  int N = 0, K = 0, batch = 0;
  ftdx_output output = FTDX_OUT_FP32;
  bool raw = false;
  ftdx_ftd_desc ftd{};
  int threads = 1;
  size_t in_bytes = 0, out_bytes = 0;
  void* d_in[2] = {nullptr, nullptr};
  void* d_out[2] = {nullptr, nullptr};
  void* h_in[2] = {nullptr, nullptr};   // pinned staging, allocated on first pageable payload
  void* h_out[2] = {nullptr, nullptr};
  cudaStream_t s_h2d = nullptr, s_comp = nullptr, s_d2h = nullptr;
  cudaStream_t s_d2h2 = nullptr;  // second D2H stream: each output leaves in two halves
  cudaEvent_t ev_h2d[2] = {}, ev_comp[2] = {}, ev_d2h[2] = {}, ev_d2h2[2] = {};
};

namespace ftdx {
namespace {

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// memcpy split over n threads (pageable <-> pinned staging)
void par_copy(void* dst, const void* src, size_t bytes, int n) {
  if (n <= 1 || bytes < (size_t(8) << 20)) {
    std::memcpy(dst, src, bytes);
    return;
  }
  std::vector<std::thread> ts;
  const size_t per = (bytes + n - 1) / n;
  for (int t = 0; t < n; ++t) {
    const size_t b0 = size_t(t) * per;
    if (b0 >= bytes) break;
    const size_t len = std::min(per, bytes - b0);
    ts.emplace_back([=] {
      std::memcpy(static_cast<char*>(dst) + b0, static_cast<const char*>(src) + b0, len);
    });
  }
  for (auto& t : ts) t.join();
}

void release(ftdx_pipeline* p) {
  if (!p) return;
  if (p->h) cudaSetDevice(p->h->device);
  for (cudaStream_t s : {p->s_h2d, p->s_comp, p->s_d2h, p->s_d2h2})
    if (s) cudaStreamSynchronize(s);
  for (int i = 0; i < 2; ++i) {
    if (p->d_in[i]) cudaFree(p->d_in[i]);
    if (p->d_out[i]) cudaFree(p->d_out[i]);
    if (p->h_in[i]) cudaFreeHost(p->h_in[i]);
    if (p->h_out[i]) cudaFreeHost(p->h_out[i]);
    for (cudaEvent_t e : {p->ev_h2d[i], p->ev_comp[i], p->ev_d2h[i], p->ev_d2h2[i]})
      if (e) cudaEventDestroy(e);
  }
  for (cudaStream_t s : {p->s_h2d, p->s_comp, p->s_d2h, p->s_d2h2})
    if (s) cudaStreamDestroy(s);
  delete p;
}

ftdx_status correlate_one(ftdx_pipeline* p, int slot) {
  if (p->raw)
    return ftdx_herk_ftd(p->h, p->d_in[slot], p->d_out[slot], &p->ftd, p->output, 1.f, 0.f,
                         p->s_comp);
  return ftdx_herk(p->h, p->d_in[slot], p->d_out[slot], p->N, p->K, p->batch, FTDX_IN_INT4,
                   FTDX_COMPUTE_FP8, p->output, FTDX_FORMAT_PACKED_TRIANGLE, 1.f, 0.f, p->s_comp,
                   1);
}

}  // namespace
}  // namespace ftdx

using namespace ftdx;

extern "C" {

ftdx_status ftdx_pipeline_create(ftdx_handle h, const ftdx_pipeline_config* cfg,
                                 ftdx_pipeline_t* out) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!cfg || !out) return fail(h, FTDX_ERR_INVALID_ARG, "pipeline_create: null argument");
  *out = nullptr;
  auto* p = new ftdx_pipeline;
  p->h = h;
  p->output = cfg->output;
  p->threads = cfg->host_threads > 0
                   ? cfg->host_threads
                   : int(std::min(8u, std::max(1u, std::thread::hardware_concurrency())));
  int64_t N, K, batch, in_elems;
  if (cfg->ftd) {
    const ftdx_ftd_desc& d = *cfg->ftd;
    if (d.n_ant < 1 || d.n_chan < 1 || d.n_pol < 1 || d.n_time_inner < 1 || d.n_time < 1 ||
        d.n_time % d.n_time_inner != 0 || (d.pol_sum != 0 && d.pol_sum != 1)) {
      delete p;
      return fail(h, FTDX_ERR_INVALID_ARG, "pipeline_create: bad raw-layout geometry");
    }
    p->raw = true;
    p->ftd = d;
    N = d.n_ant;
    K = d.n_time / d.n_time_inner;
    batch = int64_t(d.n_chan) * d.n_time_inner * (d.pol_sum ? 1 : d.n_pol);
    in_elems = int64_t(d.n_time) * d.n_ant * d.n_chan * d.n_pol;
  } else {
    N = cfg->N, K = cfg->K, batch = cfg->batch;
    in_elems = N * K * batch;
  }
  if (N < 1 || K < 1 || batch < 1 || (cfg->output != FTDX_OUT_FP32 && cfg->output != FTDX_OUT_FP16)) {
    delete p;
    return fail(h, FTDX_ERR_INVALID_ARG, "pipeline_create: bad sizes or output precision");
  }
  p->N = int(N), p->K = int(K), p->batch = int(batch);
  p->in_bytes = size_t(in_elems);
  p->out_bytes = size_t(batch) * size_t(N) * size_t(N + 1) / 2 * (cfg->output == FTDX_OUT_FP32 ? 8 : 4);
  cudaError_t e = cudaSetDevice(h->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->s_h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->s_comp, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->s_d2h, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->s_d2h2, cudaStreamNonBlocking);
  for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
    e = cudaEventCreateWithFlags(&p->ev_h2d[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_comp[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_d2h[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_d2h2[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_in[i], p->in_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_out[i], p->out_bytes);
  }
  if (e != cudaSuccess) {
    ftdx_status st = cuda_fail(h, e, "pipeline_create");
    release(p);
    return st;
  }
  // size the correlator's workspace and tile plan now, not inside the loop
  ftdx_status st = ftdx_init_herk(h, p->N, p->K * (p->raw && p->ftd.pol_sum ? p->ftd.n_pol : 1),
                                  p->batch, p->s_comp);
  if (st != FTDX_OK) {
    release(p);
    return st;
  }
  *out = p;
  return FTDX_OK;
}

ftdx_status ftdx_pipeline_sizes(ftdx_pipeline_t p, size_t* in_bytes, size_t* out_bytes) {
  if (!p) return FTDX_ERR_INVALID_ARG;
  if (in_bytes) *in_bytes = p->in_bytes;
  if (out_bytes) *out_bytes = p->out_bytes;
  return FTDX_OK;
}

ftdx_status ftdx_pipeline_correlate(ftdx_pipeline_t p, void* const* vis_outputs,
                                    const void* const* raw_inputs, int n) {
  if (!p) return FTDX_ERR_INVALID_ARG;
  ftdx_handle h = p->h;
  if (n < 0 || (n > 0 && (!vis_outputs || !raw_inputs)))
    return fail(h, FTDX_ERR_INVALID_ARG, "pipeline_correlate: bad payload list");
  for (int i = 0; i < n; ++i)
    if (!vis_outputs[i] || !raw_inputs[i])
      return fail(h, FTDX_ERR_INVALID_ARG, "pipeline_correlate: null buffer for payload %d", i);
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  std::vector<char> staged_out(size_t(n), 0);
  ftdx_status st = FTDX_OK;
  // host copy of a staged output once its D2H is done
  auto drain = [&](int q) -> ftdx_status {
    if (q < 0 || !staged_out[size_t(q)]) return FTDX_OK;
    cudaError_t ee = cudaEventSynchronize(p->ev_d2h[q & 1]);
    if (ee != cudaSuccess) return cuda_fail(h, ee, "pipeline D2H");
    par_copy(vis_outputs[q], p->h_out[q & 1], p->out_bytes, p->threads);
    staged_out[size_t(q)] = 0;
    return FTDX_OK;
  };
  for (int i = 0; i < n && st == FTDX_OK; ++i) {
    const int s = i & 1;
    // ---- H2D: d_in[s] is free once payload i-2's correlation has read it
    if (i >= 2) e = cudaStreamWaitEvent(p->s_h2d, p->ev_comp[s], 0);
    if (e == cudaSuccess) {
      if (is_pinned(raw_inputs[i])) {
        e = cudaMemcpyAsync(p->d_in[s], raw_inputs[i], p->in_bytes, cudaMemcpyHostToDevice,
                            p->s_h2d);
      } else {
        if (!p->h_in[s]) e = cudaMallocHost(&p->h_in[s], p->in_bytes);
        // the staging buffer is free once payload i-2's H2D has finished
        if (e == cudaSuccess) e = cudaEventSynchronize(p->ev_h2d[s]);
        if (e == cudaSuccess) {
          par_copy(p->h_in[s], raw_inputs[i], p->in_bytes, p->threads);
          e = cudaMemcpyAsync(p->d_in[s], p->h_in[s], p->in_bytes, cudaMemcpyHostToDevice,
                              p->s_h2d);
        }
      }
    }
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_h2d[s], p->s_h2d);
    // ---- correlation: d_out[s] is free once payload i-2's D2H has read it
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s_comp, p->ev_h2d[s], 0);
    if (e == cudaSuccess && i >= 2) e = cudaStreamWaitEvent(p->s_comp, p->ev_d2h[s], 0);
    if (e != cudaSuccess) {
      st = cuda_fail(h, e, "pipeline H2D");
      break;
    }
    st = correlate_one(p, s);
    if (st != FTDX_OK) break;
    e = cudaEventRecord(p->ev_comp[s], p->s_comp);
    // ---- D2H, in two halves on two streams (two copy engines)
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s_d2h, p->ev_comp[s], 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s_d2h2, p->ev_comp[s], 0);
    void* dst = vis_outputs[i];
    if (e == cudaSuccess && !is_pinned(vis_outputs[i])) {
      // the staging buffer holds payload i-2 until its host copy is done
      st = drain(i - 2);
      if (st != FTDX_OK) break;
      if (!p->h_out[s]) e = cudaMallocHost(&p->h_out[s], p->out_bytes);
      dst = p->h_out[s];
      staged_out[size_t(i)] = 1;
    }
    const size_t half = (p->out_bytes / 2 + 255) & ~size_t(255);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(dst, p->d_out[s], std::min(half, p->out_bytes), cudaMemcpyDeviceToHost,
                          p->s_d2h);
    if (e == cudaSuccess && half < p->out_bytes)
      e = cudaMemcpyAsync(static_cast<char*>(dst) + half, static_cast<char*>(p->d_out[s]) + half,
                          p->out_bytes - half, cudaMemcpyDeviceToHost, p->s_d2h2);
    // ev_d2h[s]: both halves done
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_d2h2[s], p->s_d2h2);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->s_d2h, p->ev_d2h2[s], 0);
    if (e == cudaSuccess) e = cudaEventRecord(p->ev_d2h[s], p->s_d2h);
    if (e != cudaSuccess) {
      st = cuda_fail(h, e, "pipeline D2H");
      break;
    }
    // copy out the previous payload while this one is in flight
    st = drain(i - 1);
  }
  // finish: every queued copy, then the staged outputs still pending
  for (cudaStream_t s : {p->s_h2d, p->s_comp, p->s_d2h, p->s_d2h2}) {
    const cudaError_t ee = cudaStreamSynchronize(s);
    if (ee != cudaSuccess && st == FTDX_OK) st = cuda_fail(h, ee, "pipeline sync");
  }
  for (int q = std::max(0, n - 2); q < n && st == FTDX_OK; ++q) st = drain(q);
  if (st == FTDX_OK) {
    uint32_t flags = 0;
    st = ftdx_device_status(h, p->s_comp, &flags);
  }
  return st;
}

ftdx_status ftdx_pipeline_destroy(ftdx_pipeline_t p) {
  if (!p) return FTDX_ERR_INVALID_ARG;
  release(p);
  return FTDX_OK;
}

}  // extern "C"
