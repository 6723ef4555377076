// batched_api.cu -- one launch for many channels with their own number of
// inputs (antenna flagging), their own integration length K, their own input
// rows (pitch, active-row list) and their own output buffers.
//
// The reference batches only uniform problems (N, K, batch): its callers loop
// over channel groups (lib/visibility_pipeline.cu:268-277).  Here the
// promotion pass gathers each channel's active rows into the FP8 planes and
// the persistent correlator walks one tile list over all channels, longest
// integration first so that the short channels fill the last wave.  Store
// modes 2 and 3 run the CTA-pair kernel on the same channel table, with its
// own tile list (256 column x 128 row inputs) and the -Re plane.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "context.h"

namespace ftdx {
namespace {

// Device-resident description of one batched call.
struct VPlan {
  GatherDesc* d_gather = nullptr;
  TileDesc* d_tiles = nullptr;
  TileDesc* d_tiles_pair = nullptr;
  ChanDesc* d_chans = nullptr;
  int num_tiles = 0;
  int num_tiles_pair = 0;
  int num_chans = 0;
  int max_n = 0;
  int64_t rows = 0;
  int kp = 0;
  ~VPlan() {
    if (d_gather) cudaFree(d_gather);
    if (d_tiles) cudaFree(d_tiles);
    if (d_tiles_pair) cudaFree(d_tiles_pair);
    if (d_chans) cudaFree(d_chans);
  }
};

uint64_t mix(uint64_t h, uint64_t v) {
  h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  return h * 0x100000001b3ull;
}

uint64_t fingerprint(const ftdx_channel_desc* d, int n, int output) {
  uint64_t h = mix(0xcbf29ce484222325ull, uint64_t(n) * 131 + uint64_t(output));
  for (int c = 0; c < n; ++c) {
    h = mix(h, reinterpret_cast<uintptr_t>(d[c].A));
    h = mix(h, reinterpret_cast<uintptr_t>(d[c].C));
    h = mix(h, reinterpret_cast<uintptr_t>(d[c].active));
    h = mix(h, uint64_t(d[c].n_inputs) << 32 | uint32_t(d[c].K));
    h = mix(h, uint64_t(d[c].lda));
  }
  return h;
}

// Builds (or finds) the plan: gather table, channel table and the tile list,
// channels ordered by descending K, each channel's tiles in triangle order;
// the same for the pair kernel's tiles (tj over 256 column inputs).
ftdx_status get_vplan(ftdx_handle h, const ftdx_channel_desc* d, int n, int output, uint64_t fp,
                      cudaStream_t s, const VPlan** out) {
  auto it = h->vplans.find(fp);
  if (it != h->vplans.end()) {
    *out = static_cast<const VPlan*>(it->second.get());
    return FTDX_OK;
  }
  if (stream_capturing(s))
    return fail(h, FTDX_ERR_CAPACITY, "batched plan built while capturing; call once first");
  auto p = std::make_shared<VPlan>();
  std::vector<GatherDesc> g(n);
  std::vector<ChanDesc> ch(n);
  int kp = 0;
  int64_t rows = 0;
  for (int c = 0; c < n; ++c) {
    const int kpc = int(round_up(d[c].K, kStageK));
    kp = std::max(kp, kpc);
    g[c].a = static_cast<const uint8_t*>(d[c].A);
    g[c].active = d[c].active;
    g[c].lda = d[c].lda > 0 ? d[c].lda : d[c].K;
    g[c].row0 = rows;
    g[c].n = d[c].n_inputs;
    g[c].k = d[c].K;
    ch[c].n = d[c].n_inputs;
    ch[c].kblocks = kpc / kStageK;
    ch[c].row0 = rows;
    ch[c].out0 = 0;
    ch[c].out_ptr = int64_t(reinterpret_cast<uintptr_t>(d[c].C));
    rows += d[c].n_inputs;
    p->max_n = std::max(p->max_n, d[c].n_inputs);
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return ch[a].kblocks > ch[b].kblocks; });
  std::vector<TileDesc> tiles, tiles_pair;
  for (int c : order) {
    const int nb = (ch[c].n + kTile - 1) / kTile;
    for (int ti = 0; ti < nb; ++ti) {
      for (int tj = 0; tj <= ti; ++tj) tiles.push_back(TileDesc{c, uint16_t(ti), uint16_t(tj)});
      for (int tj = 0; tj <= ti / 2; ++tj)
        tiles_pair.push_back(TileDesc{c, uint16_t(ti), uint16_t(tj)});
    }
  }
  if (tiles.size() > size_t(1) << 30) return fail(h, FTDX_ERR_INVALID_ARG, "too many tiles");
  p->num_tiles = int(tiles.size());
  p->num_tiles_pair = int(tiles_pair.size());
  p->num_chans = n;
  p->rows = rows;
  p->kp = kp;
  cudaError_t e = cudaMalloc(&p->d_gather, g.size() * sizeof(GatherDesc));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_chans, ch.size() * sizeof(ChanDesc));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_tiles, tiles.size() * sizeof(TileDesc));
  if (e == cudaSuccess)
    e = cudaMalloc(&p->d_tiles_pair, tiles_pair.size() * sizeof(TileDesc));
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_gather, g.data(), g.size() * sizeof(GatherDesc), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_chans, ch.data(), ch.size() * sizeof(ChanDesc), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_tiles, tiles.data(), tiles.size() * sizeof(TileDesc),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_tiles_pair, tiles_pair.data(), tiles_pair.size() * sizeof(TileDesc),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(h, e, "batched plan upload");
  if (h->vplans.size() >= 8) h->vplans.erase(h->vplans.begin());
  h->vplans[fp] = p;
  *out = p.get();
  return FTDX_OK;
}

struct VCall {
  const ftdx_channel_desc* d;
  int n;
  ftdx_output output;
  float alpha, beta;
  uint64_t fp;
};

// The CTA-pair kernel (store modes 2 and 3) when a pair fits on the device.
bool pair_strategy(ftdx_handle h, const Strategy& strat) {
  return (strat.store_mode & 3) >= 2 && pair_grid_limit(h) >= 2;
}

// Plan and workspace (two planes, three for the pair kernel's -Re operand).
ftdx_status prepare_v(ftdx_handle h, const VCall& c, cudaStream_t s, const VPlan** plan,
                      bool pair) {
  ftdx_status st = get_vplan(h, c.d, c.n, int(c.output), c.fp, s, plan);
  if (st != FTDX_OK) return st;
  return ensure_workspace(
      h, size_t(pair ? 3 : 2) * size_t((*plan)->rows) * size_t((*plan)->kp), s);
}

ftdx_status launch_v(ftdx_handle h, const VCall& c, const Strategy& strat, cudaStream_t s) {
  const bool pair = pair_strategy(h, strat);
  const VPlan* p = nullptr;
  ftdx_status st = prepare_v(h, c, s, &p, pair);
  if (st != FTDX_OK) return st;
  cudaError_t e;
  {
    ScopedTimer tm(h, s, 1);
    e = launch_gather_qc_to_planes(p->d_gather, p->num_chans, p->max_n, h->z, p->rows, p->kp, s,
                                   pair ? 1 : 0);
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "gathered promotion launch");
  CUtensorMap tmZ;
  st = encode_planes_map(h, h->z, p->rows, p->kp, &tmZ, kTile, pair ? 3 : 2);
  if (st != FTDX_OK) return st;
  HerkArgs args = herk_args_default();
  args.tiles = pair ? p->d_tiles_pair : p->d_tiles;
  args.chans = p->d_chans;
  args.num_tiles = pair ? p->num_tiles_pair : p->num_tiles;
  args.out_fp16 = (c.output == FTDX_OUT_FP16) ? 1 : 0;
  args.bulk_store = (strat.store_mode & 1) ? 1 : 0;  // modes 1 and 3
  args.out_format = 0;
  args.out = nullptr;
  args.alpha = c.alpha;
  args.beta = c.beta;
  args.status = h->d_status;
  if (pair) {
    // persistent pairs, at most as many as can be resident together
    const int limit = pair_grid_limit(h);
    int grid = strat.grid > 0 ? std::min(strat.grid, limit) : limit;
    if (strat.grid < 0) grid = 2 * p->num_tiles_pair;
    grid = std::min(grid, 2 * p->num_tiles_pair) & ~1;
    ScopedTimer tm(h, s, 0);
    e = launch_herk_fp8_pair(tmZ, args, grid, s);
  } else {
    int grid = strat.grid > 0 ? std::min(strat.grid, h->sm_count) : h->sm_count;
    if (strat.grid < 0) grid = p->num_tiles;
    grid = std::min(grid, p->num_tiles);
    ScopedTimer tm(h, s, 0);
    e = launch_herk_fp8(tmZ, args, grid, s);
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "correlator kernel launch");
  return FTDX_OK;
}

}  // namespace
}  // namespace ftdx

using namespace ftdx;

extern "C" ftdx_status ftdx_herk_batched_v(ftdx_handle h, const ftdx_channel_desc* chans,
                                           int n_chans, ftdx_output output, float alpha,
                                           float beta, void* stream, int tune) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!chans || n_chans < 1 || n_chans > (1 << 24))
    return fail(h, FTDX_ERR_INVALID_ARG, "batched: need 1..2^24 channel descriptors");
  if (output != FTDX_OUT_FP32 && output != FTDX_OUT_FP16)
    return fail(h, FTDX_ERR_INVALID_ARG, "batched: bad output precision %d", int(output));
  int64_t rows = 0;
  for (int c = 0; c < n_chans; ++c) {
    const ftdx_channel_desc& d = chans[c];
    if (!d.A || !d.C || d.n_inputs < 1 || d.K < 1 || d.n_inputs > 65535 * kTile ||
        int64_t(d.K) > (int64_t(1) << 30) || (d.lda != 0 && d.lda < d.K))
      return fail(h, FTDX_ERR_INVALID_ARG, "batched: channel %d has a bad descriptor", c);
    if ((reinterpret_cast<uintptr_t>(d.C) & (output == FTDX_OUT_FP32 ? 7 : 3)) != 0)
      return fail(h, FTDX_ERR_INVALID_ARG, "batched: channel %d output misaligned", c);
    rows += d.n_inputs;
  }
  if (rows + 256 > (int64_t(1) << 31))
    return fail(h, FTDX_ERR_INVALID_ARG, "batched: too many rows for one call");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool capturing = stream_capturing(s);
  const VCall call{chans, n_chans, output, alpha, beta, fingerprint(chans, n_chans, int(output))};

  // Tune key: batched problems are keyed by their fingerprint (n = -1).
  int kp = 0;
  for (int c = 0; c < n_chans; ++c) kp = std::max(kp, int(round_up(chans[c].K, kStageK)));
  const TuneKey key{h->device_name, -1, kp, n_chans, int(FTDX_IN_INT4),
                    int(output) | int((call.fp & 0xffffff) << 4)};
  Strategy strat = h->default_strategy;
  if (tune) {
    auto it = h->tuned.find(key);
    if (it != h->tuned.end()) {
      strat = it->second.st;
    } else if (beta == 0.f && !capturing) {
      TuneEntry best;
      std::vector<Strategy> cands = default_candidates(h, output == FTDX_OUT_FP32, true);
      if (output == FTDX_OUT_FP32 && pair_grid_limit(h) >= 2)
        cands.push_back(Strategy{3, pair_grid_limit(h)});  // pair with bulk-copy stores
      ftdx_status st = tune_sweep(
          h, [&](const Strategy& cand, cudaStream_t ss) { return launch_v(h, call, cand, ss); },
          cands, s, &best);
      if (st != FTDX_OK) return st;
      record_tuned(h, key, best);
      strat = best.st;
    }
  }
  if (h->graph_mode && !capturing) {
    const GraphKey gk{reinterpret_cast<const void*>(call.fp), nullptr, -1, kp, n_chans,
                      int(FTDX_IN_INT4), int(output), alpha, beta, strat.store_mode, strat.grid,
                      1};
    return graph_launch(
        h, gk,
        [&](cudaStream_t ss) {
          const VPlan* p = nullptr;
          return ss == h->capture_stream ? launch_v(h, call, strat, ss)
                                         : prepare_v(h, call, ss, &p, pair_strategy(h, strat));
        },
        s);
  }
  return launch_v(h, call, strat, s);
}
