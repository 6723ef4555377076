// herk_api.cu -- correlator entry points of the C ABI: ftdx_herk, workspace
// pre-sizing, the strategy autotuner with its disk cache, and CUDA-graph
// replay.  Mirrors CutlassComplexGemm::herk (cutlass_interface/cutlass_gemm_api.cu:1707-1878),
// tune_herk / strategy_cache::run_autotune (cutlass_gemm_api.cu:1389-1409,
// strategy_cache.hpp:504-721) and the direct-HERK graph cache
// (cutlass_gemm_api.cu:200-315, 1738-1807) of the reference.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>

#include "context.h"

namespace ftdx {
namespace {

struct HerkCall {
  const void* A;
  void* C;
  int N, K, batch;
  ftdx_input input;
  ftdx_output output;
  float alpha, beta;
  ftdx_compute compute = FTDX_COMPUTE_FP8;
  void* comp = nullptr;  // Kahan compensation buffer (ftdx_herk_kahan)
  const ftdx_ftd_desc* ftd = nullptr;  // raw packet-ordered input (ftdx_herk_ftd)
  bool xeng = false;   // XEngine payload: [batch][K][N] (4,4)b two's complement (ftdx_xengine)
  int out_format = 0;  // HerkArgs::out_format
};

bool is_split(const HerkCall& c) { return c.compute == FTDX_COMPUTE_FP8_SPLIT; }
bool is_fp4(const HerkCall& c) {
  return c.compute == FTDX_COMPUTE_FP4 || c.compute == FTDX_COMPUTE_FP4_SPLIT;
}

ftdx_status validate(ftdx_handle h, const HerkCall& c, ftdx_compute compute, ftdx_format format) {
  if (!c.A || !c.C) return fail(h, FTDX_ERR_INVALID_ARG, "herk: null A or C");
  if (c.N < 1 || c.K < 1 || c.batch < 1)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: N, K and batch must be >= 1 (got %d, %d, %d)",
                c.N, c.K, c.batch);
  if (c.input != FTDX_IN_INT4 && c.input != FTDX_IN_FP16 && c.input != FTDX_IN_FP32)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: bad input precision %d", int(c.input));
  if (c.output != FTDX_OUT_FP32 && c.output != FTDX_OUT_FP16)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: bad output precision %d", int(c.output));
  if (format != FTDX_FORMAT_PACKED_TRIANGLE)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: only the packed triangle format exists");
  if (compute == FTDX_COMPUTE_FP8_SPLIT && c.input != FTDX_IN_FP32)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: split FP8 needs FP32 input");
  if ((compute == FTDX_COMPUTE_FP4 || compute == FTDX_COMPUTE_FP4_SPLIT) &&
      (c.input != FTDX_IN_FP32 || c.output != FTDX_OUT_FP32 || c.comp != nullptr))
    return fail(h, FTDX_ERR_UNSUPPORTED, "herk: NVFP4 needs FP32 input and FP32 output");
  if (compute == FTDX_COMPUTE_FP6 && (c.input != FTDX_IN_INT4 || c.comp != nullptr))
    return fail(h, FTDX_ERR_UNSUPPORTED, "herk: FP6 compute needs INT4 input (block-scaled FP6 "
                "of FP16/FP32 input is not implemented)");
  if (compute != FTDX_COMPUTE_FP8 && compute != FTDX_COMPUTE_FP8_SPLIT &&
      compute != FTDX_COMPUTE_FP4 && compute != FTDX_COMPUTE_FP4_SPLIT &&
      compute != FTDX_COMPUTE_FP6)
    return fail(h, FTDX_ERR_UNSUPPORTED, "herk: compute precision %d not implemented for "
                "this entry point", int(compute));
  if (c.input == FTDX_IN_FP32 && (reinterpret_cast<uintptr_t>(c.A) & 7) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: FP32 complex A must be 8-byte aligned");
  if ((reinterpret_cast<uintptr_t>(c.C) & (c.output == FTDX_OUT_FP32 ? 7 : 3)) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: C is not aligned to one complex element");
  if (c.input == FTDX_IN_FP16 && (reinterpret_cast<uintptr_t>(c.A) & 3) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: FP16 A must be 4-byte aligned");
  // Row coordinates of the TMA boxes are 32-bit.
  if (int64_t(c.N) * c.batch + 256 > (int64_t(1) << 31))
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: N*batch too large for one call");
  if (c.N > 65535 * kTile) return fail(h, FTDX_ERR_INVALID_ARG, "herk: N too large");
  if (int64_t(c.K) > (int64_t(1) << 30)) return fail(h, FTDX_ERR_INVALID_ARG, "herk: K too large");
  return FTDX_OK;
}

// Tile plan of the NVFP4 kernels, tiles holding at least one j <= i: single
// CTA: ti over 64 row inputs, tj over 128 column inputs; pair: ti over 112,
// tj over 256 (nvfp4_pair_tiles).  Cached with a negative kblocks key so it
// never collides with the FP8 plans.
ftdx_status get_fp4_plan(ftdx_handle h, int N, int kblocks, int batch, cudaStream_t s,
                         const Plan** out, bool pair) {
  const auto key = std::make_tuple(N, -1 - kblocks - (pair ? (1 << 24) : 0), batch);
  auto it = h->plans.find(key);
  if (it != h->plans.end()) {
    *out = it->second.get();
    return FTDX_OK;
  }
  if (stream_capturing(s))
    return fail(h, FTDX_ERR_CAPACITY, "NVFP4 tile plan built while capturing; call once first");
  const int ni = (N + 63) / 64, nj = (N + 127) / 128;
  std::vector<ChanDesc> chans(batch);
  std::vector<TileDesc> tiles;
  for (int c = 0; c < batch; ++c) {
    chans[c] = ChanDesc{N, kblocks, int64_t(c) * N, int64_t(c) * (int64_t(N) * (N + 1) / 2), 0};
    if (pair) {
      nvfp4_pair_tiles(N, c, tiles);
      continue;
    }
    for (int ti = 0; ti < ni; ++ti)
      for (int tj = 0; tj < nj && tj * 128 <= ti * 64 + 63; ++tj)
        tiles.push_back(TileDesc{c, uint16_t(ti), uint16_t(tj)});
  }
  auto p = std::make_unique<Plan>();
  p->num_tiles = int(tiles.size());
  p->num_chans = batch;
  cudaError_t e = cudaMalloc(&p->d_tiles, tiles.size() * sizeof(TileDesc));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_chans, chans.size() * sizeof(ChanDesc));
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_tiles, tiles.data(), tiles.size() * sizeof(TileDesc),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_chans, chans.data(), chans.size() * sizeof(ChanDesc),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(h, e, "NVFP4 plan upload");
  *out = p.get();
  h->plans.emplace(key, std::move(p));
  return FTDX_OK;
}

// store mode 2 (the CTA-pair strategy) selects the NVFP4 pair kernel too.
ftdx_status launch_fp4(ftdx_handle h, const HerkCall& c, const Strategy& strat, cudaStream_t s) {
  const int64_t rows = int64_t(c.N) * c.batch;
  const int split = c.compute == FTDX_COMPUTE_FP4_SPLIT ? 1 : 0;
  const int pair = ((strat.store_mode & 3) >= 2 && nvfp4_pair_limit() >= 1) ? 1 : 0;
  ftdx_status st = ensure_workspace(h, nvfp4_workspace_bytes(c.N, c.batch, c.K, split, pair), s);
  const Plan* plan = nullptr;
  if (st == FTDX_OK)
    st = get_fp4_plan(h, c.N, nvfp4_kblocks(c.K), c.batch, s, &plan, pair != 0);
  if (st != FTDX_OK) return st;
  cudaError_t e;
  {
    ScopedTimer tm(h, s, 1);  // quantiser passes
    e = launch_nvfp4(c.A, rows, c.K, c.N, c.batch, h->z, plan->d_tiles, plan->d_chans,
                     plan->num_tiles, c.C, c.alpha, c.beta, h->d_status, h->sm_count,
                     tensor_map_encoder(), s, split, pair, 1);
  }
  if (e == cudaSuccess) {
    ScopedTimer tm(h, s, 0);  // correlator
    e = launch_nvfp4(c.A, rows, c.K, c.N, c.batch, h->z, plan->d_tiles, plan->d_chans,
                     plan->num_tiles, c.C, c.alpha, c.beta, h->d_status, h->sm_count,
                     tensor_map_encoder(), s, split, pair, 2);
  }
  return e == cudaSuccess ? FTDX_OK : cuda_fail(h, e, "NVFP4 launch");
}

// Calls whose operands may take the packed FP6 form: QC input through the
// plain promotion (E3M2 holds every QC value, so results stay exact).
bool fp6_ok(const HerkCall& c) {
  return c.input == FTDX_IN_INT4 && !c.ftd && !c.xeng && !is_split(c) && !is_fp4(c);
}

// The fused-promotion kernel: uniform QC input (TMA rows of K bytes, so K a
// multiple of 16 and A 16-byte aligned), FP8 compute, packed lower triangle.
bool fused_ok(const HerkCall& c) {
  return fp6_ok(c) && c.compute == FTDX_COMPUTE_FP8 && c.out_format == 0 && c.K % 16 == 0 &&
         (reinterpret_cast<uintptr_t>(c.A) & 15) == 0;
}

bool use_pair(ftdx_handle h, const Strategy& strat) {
  return (strat.store_mode & 3) >= 2 && pair_grid_limit(h) >= 2;
}

// Split-K count a call actually uses: none for Kahan, the XEngine formats and
// NVFP4; at most one split per k-block.
int effective_splits(const HerkCall& c, const Strategy& strat) {
  if (strat.splits <= 1 || c.comp || c.out_format != 0 || is_fp4(c)) return 1;
  const int kblocks = int(round_up(c.K, kStageK) / kStageK);
  return std::min(strat.splits, kblocks);
}

// Workspace and tile plan for a call; allocates, so never while capturing.
ftdx_status prepare(ftdx_handle h, const HerkCall& c, cudaStream_t s, const Plan** plan,
                    bool pair = false, int splits = 1, bool fused = false) {
  const int64_t Kp = round_up(c.K, kStageK);
  const int64_t zpitch = is_split(c) ? 2 * Kp : Kp;
  const int64_t rows = int64_t(c.N) * c.batch;
  // the pair kernel reads a third plane, -Re; the fused kernel no planes
  ftdx_status st =
      fused ? FTDX_OK : ensure_workspace(h, size_t((pair ? 3 : 2) * rows * zpitch), s);
  if (st != FTDX_OK) return st;
  if (c.input == FTDX_IN_FP32) {
    st = ensure_aux(h, size_t(140) * size_t(c.batch) + 256, s);
    if (st != FTDX_OK) return st;
  }
  if (splits > 1) {
    st = ensure_split_ws(h, size_t(splits) * size_t(c.batch) *
                                size_t(int64_t(c.N) * (c.N + 1) / 2) * sizeof(float2), s);
    if (st != FTDX_OK) return st;
  }
  return get_plan(h, c.N, int(Kp / kStageK), c.batch, s, plan, pair, splits, c.out_format == 1);
}

// Promotion kernel + correlator kernel on stream s.
ftdx_status launch_all(ftdx_handle h, const HerkCall& c, const Strategy& strat, cudaStream_t s) {
  if (is_fp4(c)) return launch_fp4(h, c, strat, s);
  const bool pair = use_pair(h, strat);
  const bool fused = strat.store_mode == kStoreFused && fused_ok(c);
  const int splits = effective_splits(c, strat);
  const Plan* plan = nullptr;
  ftdx_status st = prepare(h, c, s, &plan, pair, splits, fused);
  if (st != FTDX_OK) return st;
  const int64_t Kp = round_up(c.K, kStageK);
  const int64_t zpitch = is_split(c) ? 2 * Kp : Kp;
  const int64_t rows = int64_t(c.N) * c.batch;
  const bool fp6 = ((strat.store_mode & kStoreFp6) || c.compute == FTDX_COMPUTE_FP6) && fp6_ok(c);
  const bool s8 = !fp6 && pair && (strat.store_mode & kStoreS8) && fp6_ok(c);
  // float inputs: arrival words (32 per channel), amax, qscale, out_scale
  uint32_t* arrive = reinterpret_cast<uint32_t*>(h->aux);
  uint32_t* amax = arrive + int64_t(c.batch) * 32;
  float* qscale = reinterpret_cast<float*>(amax + c.batch);
  float* out_scale = qscale + c.batch;
  cudaError_t e = cudaSuccess;
  if (!fused) {
    ScopedTimer tm(h, s, 1);
    if (c.xeng) {
      FtdGeom g{};
      g.n_ant = c.N, g.n_chan = 1, g.n_pol = 1, g.n_ti = c.batch;
      g.K = c.K, g.n_time = c.K, g.pol_sum = 0, g.Kp = int(Kp), g.rows = rows;
      g.neg_plane = pair ? 1 : 0;
      g.t_stride = c.N, g.z_stride = int64_t(c.K) * c.N, g.twos = 1;
      e = launch_ftd_to_planes(static_cast<const uint8_t*>(c.A), h->z, g, 0, h->sm_count, s);
    } else if (c.ftd) {
      const ftdx_ftd_desc& d = *c.ftd;
      FtdGeom g{};
      g.n_ant = d.n_ant, g.n_chan = d.n_chan, g.n_pol = d.n_pol, g.n_ti = d.n_time_inner;
      g.K = d.n_time / d.n_time_inner;
      g.n_time = d.n_time;
      g.pol_sum = d.pol_sum;
      g.Kp = int(Kp);
      g.rows = rows;
      g.neg_plane = pair ? 1 : 0;
      e = launch_ftd_to_planes(static_cast<const uint8_t*>(c.A), h->z, g, int(d.layout),
                               h->sm_count, s);
    } else if (c.input == FTDX_IN_INT4) {
      const uint8_t* qc = static_cast<const uint8_t*>(c.A);
      e = fp6  ? launch_qc_to_planes6(qc, h->z, rows, c.K, int(Kp), s, pair)
          : s8 ? launch_qc_to_planes_s8(qc, h->z, rows, c.K, int(Kp), s, pair)
               : launch_qc_to_planes(qc, h->z, rows, c.K, int(Kp), s, pair);
    } else {
      if (c.input == FTDX_IN_FP16) {
        e = launch_fp16_to_planes(c.A, h->z, rows, c.K, int(Kp), s);
        if (e == cudaSuccess && pair) e = launch_negate_plane(h->z, rows * zpitch, h->sm_count, s);
      } else {
        e = launch_float_to_planes(c.A, h->z, rows, c.K, int(Kp), int(zpitch), c.N, c.batch,
                                   is_split(c) ? 1 : 0, pair ? 1 : 0, qscale, out_scale, amax,
                                   arrive, h->d_status, h->sm_count, s);
      }
    }
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "operand promotion launch");
  CUtensorMap tmZ;  // the operand planes, or (fused) the raw QC bytes
  st = fused ? encode_qc_map(h, c.A, rows, c.K, &tmZ)
             : encode_planes_map(h, h->z, rows, zpitch, &tmZ, kTile, pair ? 3 : 2, fp6);
  if (st != FTDX_OK) return st;
  HerkArgs args = herk_args_default();
  args.tiles = plan->d_tiles;
  args.chans = plan->d_chans;
  args.num_tiles = plan->num_tiles;
  args.out_fp16 = (c.output == FTDX_OUT_FP16) ? 1 : 0;
  args.bulk_store = (strat.store_mode & 1) ? 1 : 0;  // modes 1 and 3
  args.fp6 = fp6 ? 1 : 0;
  args.s8 = s8 ? 1 : 0;
  args.out_format = c.out_format;
  args.out = c.C;
  args.alpha = c.alpha;
  args.beta = c.beta;
  args.status = h->d_status;
  if (c.input == FTDX_IN_FP32) args.chan_scale = out_scale;
  if (is_split(c)) {  // (hi, hi) + (hi, lo) + (lo, hi)
    const int kb = int(Kp / kStageK);
    args.nseg = 3;
    args.seg_a[0] = 0, args.seg_a[1] = 0, args.seg_a[2] = kb;
    args.seg_b[0] = 0, args.seg_b[1] = kb, args.seg_b[2] = 0;
  }
  if (c.comp) {
    args.kahan = 1;
    args.out2 = c.comp;
  }
  if (splits > 1) {  // partial triangles, reduced below
    args.out = h->split_ws;
    args.out_fp16 = 0;
    args.alpha = 1.f;
    args.beta = 0.f;
    args.chan_scale = nullptr;
  }
  if (pair) {
    // persistent pairs, at most as many as can be resident together
    const int limit = pair_grid_limit(h);
    int grid = strat.grid > 0 ? std::min(strat.grid, limit) : limit;
    if (strat.grid < 0) grid = 2 * plan->num_tiles;
    grid = std::min(grid, 2 * plan->num_tiles) & ~1;
    ScopedTimer tm(h, s, 0);
    e = launch_herk_fp8_pair(tmZ, args, grid, s);
  } else {
    int grid = strat.grid > 0 ? strat.grid : h->sm_count;
    if (grid > h->sm_count) grid = h->sm_count;  // persistent: at most one CTA per SM
    if (strat.grid < 0) grid = plan->num_tiles;   // one tile per CTA
    if (grid > plan->num_tiles) grid = plan->num_tiles;
    ScopedTimer tm(h, s, 0);
    e = fused ? launch_herk_fp8_fused(tmZ, args, grid, s) : launch_herk_fp8(tmZ, args, grid, s);
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "correlator kernel launch");
  if (splits > 1) {
    e = launch_split_reduce(reinterpret_cast<const float2*>(h->split_ws), c.C,
                            c.output == FTDX_OUT_FP16 ? 1 : 0, int64_t(c.N) * (c.N + 1) / 2,
                            c.batch, splits, c.alpha, c.beta,
                            c.input == FTDX_IN_FP32 ? out_scale : nullptr, h->sm_count, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "split-K reduction launch");
  }
  return FTDX_OK;
}

TuneKey tune_key(ftdx_handle h, const HerkCall& c) {
  return TuneKey{h->device_name, c.N, int(round_up(c.K, kStageK)), c.batch,
                 int(c.input) | (int(c.compute) << 4) | (c.comp ? 256 : 0), int(c.output)};
}

// Times every candidate strategy on the caller's buffers (beta must be 0, so
// repeated runs leave C as one run would) and records the fastest.
ftdx_status run_tune(ftdx_handle h, const HerkCall& c, cudaStream_t s, TuneEntry* out) {
  if (c.beta != 0.f)
    return fail(h, FTDX_ERR_INVALID_ARG, "tuning needs beta == 0 (C is overwritten)");
  const Plan* plan = nullptr;
  ftdx_status st = prepare(h, c, s, &plan);
  if (st != FTDX_OK) return st;
  TuneEntry best;
  // NVFP4: the single-CTA and the pair kernel (store modes and grids do not apply)
  std::vector<Strategy> cands =
      is_fp4(c) ? std::vector<Strategy>{Strategy{0, h->sm_count}}
                : default_candidates(h, c.output == FTDX_OUT_FP32, true);
  if (is_fp4(c) && nvfp4_pair_limit() >= 1) cands.push_back(Strategy{2, 0});
  // QC input: promotion fused into the single-CTA correlator
  if (fused_ok(c)) cands.push_back(Strategy{kStoreFused, h->sm_count});
  // QC input: the pair kernel on signed 8-bit operands (kind::i8, exact)
  if (fp6_ok(c) && c.compute == FTDX_COMPUTE_FP8 && !c.comp && pair_grid_limit(h) >= 2) {
    cands.push_back(Strategy{2 | kStoreS8, pair_grid_limit(h)});
    if (c.output == FTDX_OUT_FP32) {  // the pair with bulk-copy stores (complex64 rows)
      cands.push_back(Strategy{3, pair_grid_limit(h)});
      cands.push_back(Strategy{3 | kStoreS8, pair_grid_limit(h)});
    }
  }
  const int kblocks = int(round_up(c.K, kStageK) / kStageK);
  if (!is_fp4(c) && !c.comp && plan->num_tiles < h->sm_count)
    for (int sp : {2, 4, 8, 16, 32})
      if (sp <= kblocks && plan->num_tiles * (sp / 2) < 2 * h->sm_count)
        cands.push_back(Strategy{0, h->sm_count, sp});
  st = tune_sweep(
      h, [&](const Strategy& cand, cudaStream_t ss) { return launch_all(h, c, cand, ss); },
      cands, s, &best);
  if (st != FTDX_OK) return st;
  record_tuned(h, tune_key(h, c), best);
  if (out) *out = best;
  return FTDX_OK;
}

ftdx_status run_graph(ftdx_handle h, const HerkCall& c, const Strategy& strat, cudaStream_t s) {
  const GraphKey key{c.A, c.C, c.N, c.K, c.batch,
                     int(c.input) | (int(c.compute) << 4) | (c.comp ? 256 : 0), int(c.output),
                     c.alpha, c.beta, strat.store_mode, strat.grid, strat.splits};
  return graph_launch(
      h, key,
      [&](cudaStream_t ss) {
        const Plan* plan = nullptr;
        return ss == h->capture_stream ? launch_all(h, c, strat, ss)
                                       : prepare(h, c, ss, &plan, use_pair(h, strat),
                                                 effective_splits(c, strat));
      },
      s);
}

}  // namespace

std::vector<Strategy> default_candidates(ftdx_handle h, bool fp32_out, bool pair_ok) {
  std::vector<Strategy> v;
  const int grids[2] = {h->sm_count, h->sm_count - h->sm_count / 8};
  for (int g : grids) {
    v.push_back(Strategy{0, g});
    if (fp32_out) v.push_back(Strategy{1, g});
  }
  if (pair_ok && pair_grid_limit(h) >= 2) v.push_back(Strategy{2, pair_grid_limit(h)});
  return v;
}

// Candidates are interleaved: a pre-heat (kTunePreheat launches of the first
// candidate, so that the sweep runs at the clock a sustained run settles to
// under the power limit), two warm-up rounds, then kTuneRounds timed rounds in
// which every candidate runs once (each launch between its own pair of
// events), and each candidate's median decides.  A part at its power limit
// slows as it heats; interleaving gives every candidate the same drift, where
// timing them one after the other would favour the first ones.
ftdx_status tune_sweep(ftdx_handle h, const LaunchFn& launch, const std::vector<Strategy>& cands,
                       cudaStream_t s, TuneEntry* best_out) {
  constexpr int kTuneRounds = 5;
  constexpr int kTunePreheat = 50;
  const size_t nc = cands.size();
  std::vector<cudaEvent_t> ev(2 * nc, nullptr);
  ftdx_status st = FTDX_OK;
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) st = fail(h, FTDX_ERR_CUDA, "tuner events");
  const bool prof = h->profiling;
  h->profiling = false;
  std::vector<std::vector<float>> times(nc);
  for (int w = 0; w < kTunePreheat && nc > 1 && st == FTDX_OK; ++w) st = launch(cands[0], s);
  for (int w = 0; w < 2 && st == FTDX_OK; ++w)
    for (size_t i = 0; i < nc && st == FTDX_OK; ++i) st = launch(cands[i], s);
  for (int r = 0; r < kTuneRounds && st == FTDX_OK; ++r) {
    for (size_t i = 0; i < nc && st == FTDX_OK; ++i) {
      cudaEventRecord(ev[2 * i], s);
      st = launch(cands[i], s);
      cudaEventRecord(ev[2 * i + 1], s);
    }
    for (size_t i = 0; i < nc && st == FTDX_OK; ++i) {
      float ms = 0.f;
      cudaError_t ce = cudaEventSynchronize(ev[2 * i + 1]);
      if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
      if (ce != cudaSuccess) st = cuda_fail(h, ce, "tuner timing");
      times[i].push_back(ms);
    }
  }
  TuneEntry best;
  best.ms = -1.f;
  for (size_t i = 0; i < nc && st == FTDX_OK; ++i) {
    std::vector<float> t = times[i];
    std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
    const float ms = t[t.size() / 2];
    if (h->verbosity > 1)
      fprintf(stderr, "ftdx tune: store=%d grid=%d splits=%d %.4f ms (median of %d)\n",
              cands[i].store_mode, cands[i].grid, cands[i].splits, ms, kTuneRounds);
    if (best.ms < 0.f || ms < best.ms) best = TuneEntry{cands[i], ms};
  }
  h->profiling = prof;
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  if (st == FTDX_OK && best_out) *best_out = best;
  return st;
}

void record_tuned(ftdx_handle h, const TuneKey& k, const TuneEntry& e) {
  h->tuned[k] = e;
  if (h->verbosity > 0)
    fprintf(stderr, "ftdx tuned n=%d kp=%d batch=%d -> store=%d grid=%d splits=%d (%.4f ms)\n",
            k.n, k.kp, k.batch, e.st.store_mode, e.st.grid, e.st.splits, e.ms);
  if (h->tune_cache.empty()) return;
  FILE* f = fopen(h->tune_cache.c_str(), "a");
  if (!f) {
    fail(h, FTDX_ERR_CACHE, "cannot append to tune cache %s: %s", h->tune_cache.c_str(),
         strerror(errno));
    return;
  }
  fprintf(f, "ftdx-tune 2 %s %d %d %d %d %d %d %d %d %.6f\n", k.device.c_str(), k.n, k.kp,
          k.batch, k.input, k.output, e.st.store_mode, e.st.grid, e.st.splits, e.ms);
  fclose(f);
}

// Replays a launch sequence as one CUDA graph per key (least-recently-used
// cache of kGraphCacheSize entries).  `launch` is first called on the
// caller's stream outside capture to allocate what it needs, then on the
// capture stream.
ftdx_status graph_launch(ftdx_handle h, const GraphKey& key,
                         const std::function<ftdx_status(cudaStream_t)>& launch, cudaStream_t s) {
  for (auto it = h->graphs.begin(); it != h->graphs.end(); ++it) {
    if (it->key == key) {
      h->graphs.splice(h->graphs.begin(), h->graphs, it);
      cudaError_t e = cudaGraphLaunch(h->graphs.front().exec, s);
      return e == cudaSuccess ? FTDX_OK : cuda_fail(h, e, "cudaGraphLaunch");
    }
  }
  ftdx_status st = launch(s == h->capture_stream ? nullptr : s);  // allocation pass
  if (st != FTDX_OK) return st;
  GraphEntry ge;
  ge.key = key;
  cudaError_t e = cudaStreamBeginCapture(h->capture_stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamBeginCapture");
  st = launch(h->capture_stream);
  e = cudaStreamEndCapture(h->capture_stream, &ge.graph);
  if (st != FTDX_OK) {
    if (ge.graph) cudaGraphDestroy(ge.graph);
    return st;
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&ge.exec, ge.graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(ge.graph);
    return cuda_fail(h, e, "cudaGraphInstantiate");
  }
  h->graphs.push_front(ge);
  while (h->graphs.size() > kGraphCacheSize) {
    cudaGraphExecDestroy(h->graphs.back().exec);
    cudaGraphDestroy(h->graphs.back().graph);
    h->graphs.pop_back();
  }
  e = cudaGraphLaunch(h->graphs.front().exec, s);
  return e == cudaSuccess ? FTDX_OK : cuda_fail(h, e, "cudaGraphLaunch");
}

void release_graphs(ftdx_handle h) {
  for (auto& g : h->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  h->graphs.clear();
}

// Store modes 0..3, each optionally + kStoreFp6, or 2 / 3 + kStoreS8, or
// kStoreFused alone.
static bool valid_store_mode(int m) {
  if (m == kStoreFused) return true;
  if (m < 0 || (m & ~(3 | kStoreFp6 | kStoreS8)) != 0) return false;
  return !(m & kStoreS8) || m == (2 | kStoreS8) || m == (3 | kStoreS8);
}

// Text cache, one entry per line:
//   ftdx-tune 2 <device> <N> <Kp> <batch> <input> <output> <store_mode> <grid> <splits> <ms>
// (version 1 lines, without <splits>, are read as splits = 1).
// Unreadable or malformed lines are skipped and counted.
void load_tune_cache(ftdx_handle h) {
  h->cache_bad_lines = 0;
  if (h->tune_cache.empty()) return;
  std::ifstream f(h->tune_cache);
  if (!f) return;  // a cache that does not exist yet is not an error
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream is(line);
    std::string magic, dev;
    int ver = 0;
    TuneKey k;
    TuneEntry e;
    bool ok = static_cast<bool>(is >> magic >> ver >> dev >> k.n >> k.kp >> k.batch >> k.input >>
                                k.output >> e.st.store_mode >> e.st.grid);
    e.st.splits = 1;
    if (ok && ver == 2) ok = static_cast<bool>(is >> e.st.splits);
    if (ok) ok = static_cast<bool>(is >> e.ms);
    if (!ok || magic != "ftdx-tune" || (ver != 1 && ver != 2) || (k.n < 1 && k.n != -1) ||
        k.kp < 1 || k.batch < 1 || !valid_store_mode(e.st.store_mode) || e.st.grid < 0 ||
        e.st.splits < 1 || e.st.splits > 32 || !(e.ms >= 0.f)) {
      ++h->cache_bad_lines;
      continue;
    }
    k.device = dev;
    h->tuned[k] = e;
  }
}

}  // namespace ftdx

using namespace ftdx;

extern "C" {

ftdx_status ftdx_herk(ftdx_handle h, const void* A, void* C, int N, int K, int batch,
                      ftdx_input input, ftdx_compute compute, ftdx_output output,
                      ftdx_format format, float alpha, float beta, void* stream, int tune) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  HerkCall c{A, C, N, K, batch, input, output, alpha, beta};
  c.compute = compute;
  ftdx_status st = validate(h, c, compute, format);
  if (st != FTDX_OK) return st;
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool capturing = stream_capturing(s);
  Strategy strat = h->default_strategy;
  if (tune) {
    auto it = h->tuned.find(tune_key(h, c));
    if (it != h->tuned.end()) {
      strat = it->second.st;
    } else if (beta == 0.f && !capturing) {
      TuneEntry te;
      st = run_tune(h, c, s, &te);
      if (st != FTDX_OK) return st;
      strat = te.st;
    }
  }
  if (h->graph_mode && !capturing) return run_graph(h, c, strat, s);
  return launch_all(h, c, strat, s);
}

ftdx_status ftdx_init_herk(ftdx_handle h, int N, int K, int batch, void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (N < 1 || K < 1 || batch < 1) return fail(h, FTDX_ERR_INVALID_ARG, "init_herk: bad sizes");
  cudaSetDevice(h->device);
  const HerkCall c{reinterpret_cast<const void*>(16), reinterpret_cast<void*>(16), N, K, batch,
                   FTDX_IN_INT4, FTDX_OUT_FP32, 1.f, 0.f};
  const Plan* p = nullptr;
  return prepare(h, c, static_cast<cudaStream_t>(stream), &p, use_pair(h, h->default_strategy));
}

ftdx_status ftdx_end_herk(ftdx_handle h) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  cudaDeviceSynchronize();
  release_graphs(h);
  if (h->z) cudaFree(h->z);
  h->z = nullptr;
  h->z_cap = 0;
  h->plans.clear();
  h->vplans.clear();
  return FTDX_OK;
}

ftdx_status ftdx_set_tune_cache(ftdx_handle h, const char* path) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  h->tune_cache = path ? path : "";
  load_tune_cache(h);
  if (h->cache_bad_lines)
    return fail(h, FTDX_ERR_CACHE, "tune cache %s: %d malformed line(s) skipped",
                h->tune_cache.c_str(), h->cache_bad_lines);
  return FTDX_OK;
}

ftdx_status ftdx_tune(ftdx_handle h, const void* A, void* C, int N, int K, int batch,
                      ftdx_input input, ftdx_output output, void* stream, int* store_mode,
                      int* grid, float* ms) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  const HerkCall c{A, C, N, K, batch, input, output, 1.f, 0.f};
  ftdx_status st = validate(h, c, FTDX_COMPUTE_FP8, FTDX_FORMAT_PACKED_TRIANGLE);
  if (st != FTDX_OK) return st;
  cudaSetDevice(h->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (stream_capturing(s)) return fail(h, FTDX_ERR_CAPACITY, "cannot tune while capturing");
  TuneEntry te;
  st = run_tune(h, c, s, &te);
  if (st != FTDX_OK) return st;
  if (store_mode) *store_mode = te.st.store_mode;
  if (grid) *grid = te.st.grid;
  if (ms) *ms = te.ms;
  return FTDX_OK;
}

ftdx_status ftdx_lookup_tuned(ftdx_handle h, int N, int K, int batch, ftdx_input input,
                              ftdx_output output, int* store_mode, int* grid, float* ms) {
  return ftdx_lookup_tuned_compute(h, N, K, batch, input, FTDX_COMPUTE_FP8, output, store_mode,
                                   grid, ms);
}

ftdx_status ftdx_lookup_tuned_compute(ftdx_handle h, int N, int K, int batch, ftdx_input input,
                                      ftdx_compute compute, ftdx_output output, int* store_mode,
                                      int* grid, float* ms) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  HerkCall c{nullptr, nullptr, N, K, batch, input, output, 1.f, 0.f};
  c.compute = compute;
  auto it = h->tuned.find(tune_key(h, c));
  if (it == h->tuned.end()) return fail(h, FTDX_ERR_CACHE, "no tuned entry for this shape");
  if (store_mode) *store_mode = it->second.st.store_mode;
  if (grid) *grid = it->second.st.grid;
  if (ms) *ms = it->second.ms;
  return FTDX_OK;
}

ftdx_status ftdx_set_graph_mode(ftdx_handle h, int enable) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  h->graph_mode = enable != 0;
  if (!h->graph_mode) {
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    release_graphs(h);
  }
  return FTDX_OK;
}

int ftdx_graph_count(ftdx_handle h) { return h ? int(h->graphs.size()) : -1; }

ftdx_status ftdx_herk_adjoint(ftdx_handle h, const void* G, const void* V, void* dV, int N, int K,
                              int batch, ftdx_input input, void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!G || !V || !dV || N < 8 || K < 1 || batch < 1 || batch > 65535 || (N % 8) != 0 ||
      N > (1 << 17) || K > (1 << 20) || int64_t(batch) * K > (int64_t(1) << 30))
    return fail(h, FTDX_ERR_INVALID_ARG, "adjoint: bad sizes (N a multiple of 8, >= 8)");
  if (input != FTDX_IN_INT4)
    return fail(h, FTDX_ERR_UNSUPPORTED, "adjoint: only QC int4 voltages are implemented");
  if (((reinterpret_cast<uintptr_t>(G) | reinterpret_cast<uintptr_t>(dV)) & 7) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "adjoint: misaligned G or dV");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ftdx_status st = ensure_workspace(h, adjoint_workspace_bytes(N, K, batch), s);
  if (st != FTDX_OK) return st;
  {
    ScopedTimer tm(h, s, 0);
    e = launch_adjoint(G, static_cast<const uint8_t*>(V), dV, N, K, batch, h->z, h->sm_count,
                       h->d_status, tensor_map_encoder(), s);
  }
  return e == cudaSuccess ? FTDX_OK : cuda_fail(h, e, "adjoint launch");
}

ftdx_status ftdx_gain_gradient(ftdx_handle h, const void* R_obs, const void* R_mod,
                               const float* W, const void* g, int N, int n_chans, double* grad,
                               double* loss, void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!R_obs || !R_mod || !W || !g || !grad || !loss || N < 1 || n_chans < 1 ||
      n_chans > 65535 || N > (1 << 20))
    return fail(h, FTDX_ERR_INVALID_ARG, "gain_gradient: bad arguments");
  if (((reinterpret_cast<uintptr_t>(R_obs) | reinterpret_cast<uintptr_t>(R_mod) |
        reinterpret_cast<uintptr_t>(g) | reinterpret_cast<uintptr_t>(grad) |
        reinterpret_cast<uintptr_t>(loss)) & 7) != 0 ||
      (reinterpret_cast<uintptr_t>(W) & 3) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "gain_gradient: misaligned pointer");
  cudaError_t e = cudaSetDevice(h->device);
  if (e == cudaSuccess)
    e = launch_gain_grad(static_cast<const float2*>(R_obs), static_cast<const float2*>(R_mod), W,
                         static_cast<const float2*>(g), N, n_chans, grad, loss,
                         static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? FTDX_OK : cuda_fail(h, e, "gain gradient launch");
}

ftdx_status ftdx_herk_ftd(ftdx_handle h, const void* raw, void* C, const ftdx_ftd_desc* d,
                          ftdx_output output, float alpha, float beta, void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!d) return fail(h, FTDX_ERR_INVALID_ARG, "herk_ftd: null descriptor");
  if (d->n_ant < 1 || d->n_chan < 1 || d->n_pol < 1 || d->n_time_inner < 1 || d->n_time < 1 ||
      d->n_time % d->n_time_inner != 0)
    return fail(h, FTDX_ERR_INVALID_ARG,
                "herk_ftd: bad geometry (n_ant %d, n_chan %d, n_pol %d, n_time %d, n_time_inner %d)",
                d->n_ant, d->n_chan, d->n_pol, d->n_time, d->n_time_inner);
  if (d->layout != FTDX_LAYOUT_TIME_ANT_CHAN_POL && d->layout != FTDX_LAYOUT_CHAN_POL_ANT_TIME)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk_ftd: bad layout %d", int(d->layout));
  if (d->pol_sum != 0 && d->pol_sum != 1)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk_ftd: pol_sum must be 0 or 1");
  const int K = d->n_time / d->n_time_inner;
  const int64_t keff = d->pol_sum ? int64_t(d->n_pol) * K : int64_t(K);
  const int64_t batch = int64_t(d->n_chan) * d->n_time_inner * (d->pol_sum ? 1 : d->n_pol);
  if (keff > (int64_t(1) << 30) || batch > (int64_t(1) << 30) ||
      int64_t(d->n_time) * d->n_ant * d->n_chan * d->n_pol > (int64_t(1) << 40))
    return fail(h, FTDX_ERR_INVALID_ARG, "herk_ftd: problem too large");
  HerkCall c{raw, C, d->n_ant, int(keff), int(batch), FTDX_IN_INT4, output, alpha, beta};
  c.ftd = d;
  ftdx_status st = validate(h, c, FTDX_COMPUTE_FP8, FTDX_FORMAT_PACKED_TRIANGLE);
  if (st != FTDX_OK) return st;
  if (d->layout == FTDX_LAYOUT_TIME_ANT_CHAN_POL &&
      (round_up(keff, kStageK) > 64 * 65535 || d->n_time_inner > 65535))
    return fail(h, FTDX_ERR_INVALID_ARG, "herk_ftd: K or n_time_inner too large for this layout");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  // strategy of the equivalent batch-first call (tuned entry if one exists)
  Strategy strat = h->default_strategy;
  HerkCall plain = c;
  plain.ftd = nullptr;
  auto it = h->tuned.find(tune_key(h, plain));
  if (it != h->tuned.end()) strat = it->second.st;
  return launch_all(h, c, strat, static_cast<cudaStream_t>(stream));
}

ftdx_status ftdx_xengine(ftdx_handle h, const void* payload, void* out, int n_ant, int K,
                         int batch, int mat_format, ftdx_output output, void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (mat_format != 0 && mat_format != 1)
    return fail(h, FTDX_ERR_INVALID_ARG, "xengine: mat_format must be 0 (full) or 1 (packed upper)");
  if (batch > 65535)
    return fail(h, FTDX_ERR_INVALID_ARG, "xengine: at most 65535 matrices per call");
  HerkCall c{payload, out, n_ant, K, batch, FTDX_IN_INT4, output, 1.f, 0.f};
  c.xeng = true;
  c.out_format = mat_format == 1 ? 1 : 2;
  ftdx_status st = validate(h, c, FTDX_COMPUTE_FP8, FTDX_FORMAT_PACKED_TRIANGLE);
  if (st != FTDX_OK) return st;
  if (round_up(K, kStageK) > 64 * 65535)
    return fail(h, FTDX_ERR_INVALID_ARG, "xengine: K too large");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  // the XEngine formats are written with direct stores, by the single-CTA
  // kernel or (store modes 2 and 3) the CTA pair
  Strategy strat = h->default_strategy;
  strat.store_mode = (strat.store_mode & 3) >= 2 ? 2 : 0;
  return launch_all(h, c, strat, static_cast<cudaStream_t>(stream));
}

ftdx_status ftdx_herk_kahan(ftdx_handle h, const void* A, void* sum, void* comp, int N, int K,
                            int batch, ftdx_input input, ftdx_compute compute, void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!comp || comp == sum)
    return fail(h, FTDX_ERR_INVALID_ARG, "kahan: need a separate compensation buffer");
  if ((reinterpret_cast<uintptr_t>(comp) & 7) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "kahan: compensation buffer misaligned");
  HerkCall c{A, sum, N, K, batch, input, FTDX_OUT_FP32, 1.f, 0.f};
  c.compute = compute;
  c.comp = comp;
  ftdx_status st = validate(h, c, compute, FTDX_FORMAT_PACKED_TRIANGLE);
  if (st != FTDX_OK) return st;
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  // Read-modify-write of sum and compensation: no tuning sweep (it would
  // accumulate the same dump several times); direct stores only (the
  // single-CTA kernel, two-pass or with the promotion fused in).
  Strategy strat = h->default_strategy;
  if (strat.store_mode != kStoreFused) strat.store_mode = 0;
  return launch_all(h, c, strat, static_cast<cudaStream_t>(stream));
}

ftdx_status ftdx_set_split_k(ftdx_handle h, int splits) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (splits < 1 || splits > 32)
    return fail(h, FTDX_ERR_INVALID_ARG, "set_split_k: splits must be 1..32 (got %d)", splits);
  h->default_strategy.splits = splits;
  return FTDX_OK;
}

int ftdx_tuned_split_k(ftdx_handle h, int N, int K, int batch, ftdx_input input,
                       ftdx_output output) {
  if (!h) return -1;
  const HerkCall c{nullptr, nullptr, N, K, batch, input, output, 1.f, 0.f};
  auto it = h->tuned.find(tune_key(h, c));
  return it == h->tuned.end() ? -1 : it->second.st.splits;
}

ftdx_status ftdx_set_strategy(ftdx_handle h, int store_mode, int grid) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!valid_store_mode(store_mode) || grid < -1)
    return fail(h, FTDX_ERR_INVALID_ARG, "set_strategy: store_mode %d / grid %d", store_mode,
                grid);
  if ((store_mode & 3) >= 2) {
    cudaSetDevice(h->device);
    if (pair_grid_limit(h) < 2)
      return fail(h, FTDX_ERR_UNSUPPORTED, "set_strategy: no CTA pair fits on this device");
  }
  h->default_strategy = Strategy{store_mode, grid, h->default_strategy.splits};
  return FTDX_OK;
}

}  // extern "C"
