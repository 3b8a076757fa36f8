// Batched single-level SGM: many stereo pairs of different sizes and disparity ranges in one
// CUDA graph launch. No counterpart in the reference (it matches one pair per call).
//
// Layout: one device arena holds every pair's images, census words, cost/path volumes and
// disparity maps (dense, as in sgm_kernels.cuh); a device table of BatchPair descriptors points
// into it. Pairs are grouped into buckets by (D, width class); each bucket has its own cost,
// row-scan and column-scan launches, whose bodies and shapes an autotuner picks per bucket.
//
// Stages (one graph, captured once per batch):
//   census      all pairs, one launch, one warp per (pair, view, row)
//   cost        per bucket when its row scans read a cost volume: one block per 128 pixels
//   row scans   per bucket, a persistent kernel whose warps take items from an atomic queue,
//               longest rows first: either one warp per (pair, view, row, direction) with the
//               cost computed in the warp, or 32/G scanlines of G lanes each (u16x2 SIMD)
//   col scans   per bucket, persistent, (pair, view, columns) items, tallest pairs first; sums
//               the four paths and selects the disparity (one warp per column, or G lanes)
//   LR/median   all pairs, one launch, one block per 32x8 tile
// The buckets' kernels run on parallel graph branches. Every item runs the same device code as
// the single-pair kernels (hpaths2_warp, hpaths3_lane, vpaths1/2_warp, vpaths3_lane,
// cost3_block, census_value, lr_median_tile), so a batched pair is bit-identical to
// sgm_match_device on that pair.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/sgm_b200.h"
#include "sgm_alloc.h"
#include "sgm_batch_kernels.cuh"
#include "sgm_levels.h"

void sgm_set_process_error(const char* msg);
// Per-launch profiler of the engine (sgm_profile_enable): while it is on, a run enqueues its
// kernels directly on the caller's stream, one after another, each timed alone.
bool sgm_prof_on();
void sgm_prof_start(cudaStream_t s);
void sgm_prof_end(const char* name);

namespace {

using namespace sgm::batch;

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Runs fn, which enqueues one kernel on s; with prof, between the profiler's two events.
template <typename F>
int timed(bool prof, cudaStream_t s, const char* name, F&& fn) {
  if (prof) sgm_prof_start(s);
  const int r = fn();
  if (prof) sgm_prof_end(name);
  return r;
}

int width_class(int W) { return W <= 640 ? 0 : (W <= 1280 ? 1 : 2); }

}  // namespace

struct sgm_batch_tuning_t_internal {
  int rows_lanes = 0;  // 0: one warp per scanline (cost in the warp); 1/2/4/8: lanes per scanline
  int rows_warps = 4;  // warps per CTA of the row kernel
  int cols_lanes = 0;  // 0: one warp per column; 1/2/4/8: lanes per column
  int cols_warps = 8;
  int cols_pf = 0;     // one warp per column: 0 plain loads, 4/8 prefetch-ring depth
};

struct sgm_batch {
  int dev = 0;
  bool ready = false;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> side;
  std::vector<cudaStream_t> side2;  // the bottom-to-top column pass of each bucket
  std::vector<cudaEvent_t> ev;
  std::vector<sgm_batch_pair_t> pairs;
  sgm_option_t opt{};
  sgm_ext_options_t ext{};
  int word = 8;
  unsigned char* arena = nullptr;
  size_t arena_bytes = 0;
  std::vector<BatchPair> hdesc;
  BatchPair* ddesc = nullptr;
  int* dtab = nullptr;  // all int tables
  int* queues = nullptr;
  int nqueues = 0;
  int census_prefix = 0, tile_prefix = 0;  // offsets into dtab (tile: LR/median tiles, 32 x kLrmRows)
  int census_items = 0, tile_items = 0;
  struct Bucket {
    int K = 2, wclass = 0;
    std::vector<int> members;
    // offsets into dtab: pair order (longest rows first / tallest first) and item prefixes per
    // item size (index 0: one scanline per warp; 1..4: 32/G scanlines per warp for G = 1, 2, 4, 8)
    int rows_ids = 0, cols_ids = 0, cost_prefix = 0;
    int rows_prefix[5] = {}, cols_prefix[5] = {};
    int rows_items[5] = {}, cols_items[5] = {}, cost_items = 0;
    sgm_batch_tuning_t_internal tune;
    int rows_blocks = 0, cols_blocks = 0;
  };
  std::vector<Bucket> buckets;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nsm = 148;
  int64_t graph_kernels = 0;
  int64_t runs = 0;
  std::string err;

  void free_all() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    if (arena) sgm_dev_free(arena);
    if (ddesc) sgm_dev_free(ddesc);
    if (dtab) sgm_dev_free(dtab);
    if (queues) sgm_dev_free(queues);
    arena = nullptr;
    ddesc = nullptr;
    dtab = nullptr;
    queues = nullptr;
    for (auto s : side) cudaStreamDestroy(s);
    side.clear();
    for (auto s : side2) cudaStreamDestroy(s);
    side2.clear();
    for (auto e : ev) cudaEventDestroy(e);
    ev.clear();
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    buckets.clear();
    hdesc.clear();
    pairs.clear();
    ready = false;
  }
};

namespace {

int berr(sgm_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  else sgm_set_process_error(buf);
  return code;
}

#define BTRY(b, expr)                                                                        \
  do {                                                                                       \
    cudaError_t _st = (expr);                                                                \
    if (_st != cudaSuccess)                                                                  \
      return berr(b, _st == cudaErrorMemoryAllocation ? SGM_ERR_NOMEM : SGM_ERR_CUDA, "%s failed: %s", #expr, \
                  cudaGetErrorString(_st));                                                  \
  } while (0)

// Process-wide cache of tuned shapes: (K, census word, width class) -> tuning.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, sgm_batch_tuning_t_internal> g_tuned;

int lanes_index(int G) { return G == 1 ? 1 : G == 2 ? 2 : G == 4 ? 3 : G == 8 ? 4 : 0; }

// Lanes per scanline the u16x2 bodies support for K (D = 128 keeps 2 or 4: register budget).
bool lanes_ok(int K, int G) {
  if (K == 4) return G == 2 || G == 4;
  return G == 1 || G == 2 || G == 4 || G == 8;
}

// Prefetch depths of the u16x2 bodies (rows: cost slices; columns: four volumes' slices).
template <int K, int G>
constexpr int pf_rows() {
  return 32 * K / G >= 64 ? 2 : (32 * K / G >= 32 ? 4 : 8);
}
template <int K, int G>
constexpr int pf_cols() {
  return 32 * K / G >= 32 ? 1 : (32 * K / G >= 16 ? 2 : 4);
}

// Sizes a persistent grid: min(resident CTAs on the device, CTAs needed for the items).
template <typename F>
int size_grid(sgm_batch* b, F* fn, int threads, size_t smem, int items, int warps, int* blocks) {
  BTRY(b, sgm::allow_max_dynamic_smem(fn));
  int occ = 0;
  BTRY(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem));
  *blocks = std::max(1, std::min(b->nsm * std::max(occ, 1), (items + warps - 1) / warps));
  return SGM_OK;
}

// prepare == true: raises the kernel's shared-memory limit and sizes the persistent grid (outside
// any stream capture); prepare == false: launches with the prepared shape.
template <int K, typename Word>
int rows_t(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* queue, bool prepare) {
  const int wp = k.tune.rows_warps;
  const int G = k.tune.rows_lanes;
  const int li = lanes_index(G);
  const int n = (int)k.members.size();
  const int* ids = b->dtab + k.rows_ids;
  const int* pre = b->dtab + k.rows_prefix[li];
  if (G == 0) {
    const size_t smem = (size_t)wp * sgm::hpaths2_warp_smem<K, Word>();
    auto fn = kb_rows<K, Word>;
    if (prepare) return size_grid(b, fn, 32 * wp, smem, k.rows_items[0], wp, &k.rows_blocks);
    fn<<<k.rows_blocks, dim3(32, wp), smem, s>>>(b->ddesc, ids, pre, n, queue);
  } else {
    auto go = [&](auto fn) -> int {
      if (prepare) return size_grid(b, fn, 32 * wp, 0, k.rows_items[li], wp, &k.rows_blocks);
      fn<<<k.rows_blocks, dim3(32, wp), 0, s>>>(b->ddesc, ids, pre, n, queue);
      return SGM_OK;
    };
    int st;
    if constexpr (K == 4) {
      st = G == 4 ? go(kb_rows3<K, 4, pf_rows<K, 4>()>) : go(kb_rows3<K, 2, pf_rows<K, 2>()>);
    } else {
      st = G == 1 ? go(kb_rows3<K, 1, pf_rows<K, 1>()>) : G == 2 ? go(kb_rows3<K, 2, pf_rows<K, 2>()>)
         : G == 4 ? go(kb_rows3<K, 4, pf_rows<K, 4>()>) : go(kb_rows3<K, 8, pf_rows<K, 8>()>);
    }
    if (st || prepare) return st;
  }
  BTRY(b, cudaGetLastError());
  return SGM_OK;
}

template <int K, int PF>
int cols_warp_t(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* queue, bool prepare) {
  const int wp = k.tune.cols_warps;
  auto fn = kb_cols<K, PF>;
  if (prepare) return size_grid(b, fn, 32 * wp, 0, k.cols_items[0], wp, &k.cols_blocks);
  fn<<<k.cols_blocks, dim3(32, wp), 0, s>>>(b->ddesc, b->dtab + k.cols_ids, b->dtab + k.cols_prefix[0],
                                            (int)k.members.size(), queue);
  BTRY(b, cudaGetLastError());
  return SGM_OK;
}

template <int K, int PASS = 0>
int cols_t(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* queue, bool prepare) {
  const int G = k.tune.cols_lanes;
  if (G == 0) {
    switch (k.tune.cols_pf) {
      case 0: return cols_warp_t<K, 0>(b, k, s, queue, prepare);
      case 4: return cols_warp_t<K, 4>(b, k, s, queue, prepare);
      default: return cols_warp_t<K, 8>(b, k, s, queue, prepare);
    }
  }
  const int wp = k.tune.cols_warps;
  const int li = lanes_index(G);
  const size_t smem = (size_t)wp * (32 / G) * sgm::vpaths3_col_smem<K>();
  const int n = (int)k.members.size();
  const int* ids = b->dtab + k.cols_ids;
  const int* pre = b->dtab + k.cols_prefix[li];
  auto go = [&](auto fn) -> int {
    if (prepare) return size_grid(b, fn, 32 * wp, smem, k.cols_items[li], wp, &k.cols_blocks);
    fn<<<k.cols_blocks, dim3(32, wp), smem, s>>>(b->ddesc, ids, pre, n, queue);
    return SGM_OK;
  };
  int st;
  if constexpr (K == 4) {
    st = G == 4 ? go(kb_cols3<K, 4, pf_cols<K, 4>(), PASS>) : go(kb_cols3<K, 2, pf_cols<K, 2>(), PASS>);
  } else {
    st = G == 1   ? go(kb_cols3<K, 1, pf_cols<K, 1>(), PASS>)
         : G == 2 ? go(kb_cols3<K, 2, pf_cols<K, 2>(), PASS>)
         : G == 4 ? go(kb_cols3<K, 4, pf_cols<K, 4>(), PASS>)
                  : go(kb_cols3<K, 8, pf_cols<K, 8>(), PASS>);
  }
  if (st || prepare) return st;
  BTRY(b, cudaGetLastError());
  return SGM_OK;
}

int rows(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* queue, bool prepare) {
  const bool w64 = b->word == 8;
  switch (k.K) {
    case 1: return w64 ? rows_t<1, uint64_t>(b, k, s, queue, prepare) : rows_t<1, uint32_t>(b, k, s, queue, prepare);
    case 2: return w64 ? rows_t<2, uint64_t>(b, k, s, queue, prepare) : rows_t<2, uint32_t>(b, k, s, queue, prepare);
    default: return w64 ? rows_t<4, uint64_t>(b, k, s, queue, prepare) : rows_t<4, uint32_t>(b, k, s, queue, prepare);
  }
}

// PASS: 0 both column passes, 1 bottom-to-top only, 2 top-to-bottom + WTA only (thread-per-
// scanline column bodies; the persistent grid is sized for PASS 0, the queue counts any grid)
template <int PASS = 0>
int cols(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* queue, bool prepare) {
  switch (k.K) {
    case 1: return cols_t<1, PASS>(b, k, s, queue, prepare);
    case 2: return cols_t<2, PASS>(b, k, s, queue, prepare);
    default: return cols_t<4, PASS>(b, k, s, queue, prepare);
  }
}

// The cost volume of the bucket's pairs (needed when its row scans run the u16x2 bodies).
template <int K, typename Word>
int cost_t(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s) {
  kb_cost3<K, Word><<<k.cost_items, 128, 0, s>>>(b->ddesc, b->dtab + k.rows_ids, b->dtab + k.cost_prefix,
                                                 (int)k.members.size());
  BTRY(b, cudaGetLastError());
  return SGM_OK;
}

int launch_cost(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s) {
  if (k.tune.rows_lanes == 0) return SGM_OK;  // the warp-per-scanline body computes its own costs
  const bool w64 = b->word == 8;
  switch (k.K) {
    case 1: return w64 ? cost_t<1, uint64_t>(b, k, s) : cost_t<1, uint32_t>(b, k, s);
    case 2: return w64 ? cost_t<2, uint64_t>(b, k, s) : cost_t<2, uint32_t>(b, k, s);
    default: return w64 ? cost_t<4, uint64_t>(b, k, s) : cost_t<4, uint32_t>(b, k, s);
  }
}

int launch_rows(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* queue) {
  const int st = launch_cost(b, k, s);
  return st ? st : rows(b, k, s, queue, false);
}
int launch_cols(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* queue) {
  return cols(b, k, s, queue, false);
}
// Row and column scans of one bucket on t. When both run the thread-per-scanline bodies (the
// cost volume exists before the rows), the bottom-to-top column pass runs on t2 beside the row
// scans and the top-to-bottom pass follows the join. Queues q, q + 1, q + 2.
int bucket_scans(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t t, cudaStream_t t2, cudaEvent_t ea,
                 cudaEvent_t eb, int* q, int64_t* kernels) {
  if (k.tune.cols_lanes == 0 || k.tune.rows_lanes == 0) {
    int r = launch_rows(b, k, t, q);
    if (!r) r = launch_cols(b, k, t, q + 1);
    *kernels += k.tune.rows_lanes ? 3 : 2;
    return r;
  }
  int r = launch_cost(b, k, t);
  cudaEventRecord(ea, t);
  cudaStreamWaitEvent(t2, ea, 0);
  if (!r) r = cols<1>(b, k, t2, q + 1, false);
  if (!r) r = rows(b, k, t, q, false);
  cudaEventRecord(eb, t2);
  cudaStreamWaitEvent(t, eb, 0);
  if (!r) r = cols<2>(b, k, t, q + 2, false);
  if (!r && cudaGetLastError() != cudaSuccess) r = berr(b, SGM_ERR_CUDA, "column pass launch failed");
  *kernels += 4;
  return r;
}

int prepare_bucket(sgm_batch* b, sgm_batch::Bucket& k) {
  const int st = rows(b, k, nullptr, nullptr, true);
  return st ? st : cols(b, k, nullptr, nullptr, true);
}

int launch_census(sgm_batch* b, cudaStream_t s) {
  const int blocks = b->census_items;  // one block per (pair, view, row block)
  const int n = (int)b->pairs.size();
  if (b->word == 8)
    kb_census4<uint64_t, 4, 3><<<blocks, 128, 0, s>>>(b->ddesc, b->dtab + b->census_prefix, n);
  else
    kb_census4<uint32_t, 2, 2><<<blocks, 128, 0, s>>>(b->ddesc, b->dtab + b->census_prefix, n);
  BTRY(b, cudaGetLastError());
  return SGM_OK;
}

int launch_post(sgm_batch* b, cudaStream_t s) {
  const int n = (int)b->pairs.size();
  const float thr = b->opt.lr_threshold;
  const int* pre = b->dtab + b->tile_prefix;
  const int g = b->tile_items;
  const dim3 blk(32, 8);
  const bool lr = b->opt.do_lr_check, med = b->opt.do_median_filter;
  if (lr && med) kb_lr_median<true, true><<<g, blk, 0, s>>>(b->ddesc, pre, n, thr);
  else if (lr) kb_lr_median<true, false><<<g, blk, 0, s>>>(b->ddesc, pre, n, thr);
  else if (med) kb_lr_median<false, true><<<g, blk, 0, s>>>(b->ddesc, pre, n, thr);
  else kb_lr_median<false, false><<<g, blk, 0, s>>>(b->ddesc, pre, n, thr);
  BTRY(b, cudaGetLastError());
  return SGM_OK;
}

// Times fn() (which enqueues on s) after one warm-up run; milliseconds of the second run.
template <typename F>
int time_ms(sgm_batch* b, cudaStream_t s, F fn, float* ms) {
  cudaEvent_t e0, e1;
  BTRY(b, cudaEventCreate(&e0));
  BTRY(b, cudaEventCreate(&e1));
  int st = fn();
  if (!st) {
    cudaEventRecord(e0, s);
    st = fn();
    cudaEventRecord(e1, s);
  }
  if (!st) {
    const cudaError_t ce = cudaEventSynchronize(e1);
    if (ce != cudaSuccess) st = berr(b, SGM_ERR_CUDA, "autotune timing failed: %s", cudaGetErrorString(ce));
    else cudaEventElapsedTime(ms, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

// Picks each bucket's launch shapes by timing the candidates on this batch's shapes (noise
// images); results are cached per (D, census, width class) for the process.
int autotune(sgm_batch* b, bool force) {
  int st = launch_census(b, b->stream);
  if (st) return st;
  // the u16x2 bodies hold path costs in 16 bits and use min(x + P1, L): exact for P1 <= P2 <= 16383;
  // their WTA implements the lowest-d and the reference tie rules
  const bool u16 = b->opt.p1 <= (int)sgm::kMaxPenalty16 && b->opt.p2_init <= (int)sgm::kMaxPenalty16 &&
                   b->opt.p1 <= b->opt.p2_init &&
                   (b->ext.tie_rule == sgm::kTieLowest || b->ext.tie_rule == sgm::kTieRefB200);
  for (size_t i = 0; i < b->buckets.size(); ++i) {
    auto& k = b->buckets[i];
    const auto key = std::make_tuple(k.K, b->word, k.wclass, (b->opt.do_lr_check ? 2 : 1) + (u16 ? 4 : 0));
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tuned.find(key);
      if (!force && it != g_tuned.end()) {
        k.tune = it->second;
        continue;
      }
    }
    int* q = b->queues + 3 * i;
    auto reset = [&]() { return cudaMemsetAsync(q, 0, 2 * sizeof(int), b->stream) == cudaSuccess ? SGM_OK : SGM_ERR_CUDA; };
    // row scans: warp per scanline (4 or 8 warps per CTA), or G lanes per scanline (+ cost kernel)
    std::vector<std::pair<int, int>> rc = {{0, 4}, {0, 8}};
    if (u16)
      for (int G : {1, 2, 4, 8})
        if (lanes_ok(k.K, G)) rc.push_back({G, 4});
    float best = 1e30f;
    auto brow = rc[0];
    for (const auto& c : rc) {
      k.tune.rows_lanes = c.first;
      k.tune.rows_warps = c.second;
      st = prepare_bucket(b, k);
      if (st) return st;
      float ms = 0;
      st = time_ms(b, b->stream, [&]() { int r = reset(); return r ? r : launch_rows(b, k, b->stream, q); }, &ms);
      if (st) return st;
      if (ms < best) { best = ms; brow = c; }
    }
    k.tune.rows_lanes = brow.first;
    k.tune.rows_warps = brow.second;
    // column scans: warp per column (plain loads or an 8-row prefetch ring), or G lanes per column
    std::vector<std::tuple<int, int, int>> cc = {{0, 8, 0}, {0, 8, 8}};
    if (u16)
      for (int G : {1, 2, 4, 8})
        if (lanes_ok(k.K, G)) cc.push_back({G, 4, 0});
    best = 1e30f;
    auto bcol = cc[0];
    for (const auto& c : cc) {
      k.tune.cols_lanes = std::get<0>(c);
      k.tune.cols_warps = std::get<1>(c);
      k.tune.cols_pf = std::get<2>(c);
      st = prepare_bucket(b, k);
      if (st) return st;
      float ms = 0;
      st = time_ms(b, b->stream, [&]() { int r = reset(); return r ? r : launch_cols(b, k, b->stream, q + 1); }, &ms);
      if (st) return st;
      if (ms < best) { best = ms; bcol = c; }
    }
    k.tune.cols_lanes = std::get<0>(bcol);
    k.tune.cols_warps = std::get<1>(bcol);
    k.tune.cols_pf = std::get<2>(bcol);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = k.tune;
  }
  for (auto& k : b->buckets) {
    st = prepare_bucket(b, k);
    if (st) return st;
  }
  return SGM_OK;
}

// bucket_scans with every launch on s in a valid order, each timed alone (the profiled run).
int bucket_scans_timed(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* q) {
  int r = SGM_OK;
  if (k.tune.rows_lanes) r = timed(true, s, "cost", [&] { return launch_cost(b, k, s); });
  if (k.tune.cols_lanes == 0 || k.tune.rows_lanes == 0) {
    if (!r) r = timed(true, s, "hpaths_plain", [&] { return rows(b, k, s, q, false); });
    if (!r) r = timed(true, s, "vpaths_wta_plain", [&] { return launch_cols(b, k, s, q + 1); });
    return r;
  }
  if (!r) r = timed(true, s, "vpaths_bt_plain", [&] { return cols<1>(b, k, s, q + 1, false); });
  if (!r) r = timed(true, s, "hpaths_plain", [&] { return rows(b, k, s, q, false); });
  if (!r) r = timed(true, s, "vpaths_wta_plain", [&] { return cols<2>(b, k, s, q + 2, false); });
  return r;
}

// The graph's work enqueued directly on s, one launch after another, each timed alone.
int run_timed(sgm_batch* b, cudaStream_t s) {
  if (cudaMemsetAsync(b->queues, 0, b->nqueues * sizeof(int), s) != cudaSuccess)
    return berr(b, SGM_ERR_CUDA, "queue reset failed");
  int st = timed(true, s, "census", [&] { return launch_census(b, s); });
  for (size_t i = 0; !st && i < b->buckets.size(); ++i) st = bucket_scans_timed(b, b->buckets[i], s, b->queues + 3 * i);
  if (!st) st = timed(true, s, "lr_median", [&] { return launch_post(b, s); });
  return st;
}

// Captures census -> per-bucket [rows -> cols] branches -> LR/median into one graph.
int capture(sgm_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  cudaStream_t s = b->stream;
  BTRY(b, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int st = SGM_OK;
  int64_t kernels = 0;
  if (cudaMemsetAsync(b->queues, 0, b->nqueues * sizeof(int), s) != cudaSuccess)
    st = berr(b, SGM_ERR_CUDA, "queue reset failed");
  if (!st) { st = launch_census(b, s); kernels++; }
  if (!st) cudaEventRecord(b->ev[0], s);
  for (size_t i = 0; !st && i < b->buckets.size(); ++i) {
    cudaStream_t t = b->side[i];
    cudaStreamWaitEvent(t, b->ev[0], 0);
    const size_t e2 = 1 + b->buckets.size() + 2 * i;
    st = bucket_scans(b, b->buckets[i], t, b->side2[i], b->ev[e2], b->ev[e2 + 1], b->queues + 3 * i, &kernels);
    cudaEventRecord(b->ev[1 + i], t);
    cudaStreamWaitEvent(s, b->ev[1 + i], 0);
  }
  if (!st) { st = launch_post(b, s); kernels++; }
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (st) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (ce != cudaSuccess) return berr(b, SGM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
  b->graph = g;
  BTRY(b, cudaGraphInstantiate(&b->exec, g, 0));
  b->graph_kernels = kernels;
  return SGM_OK;
}

}  // namespace

extern "C" {

int sgm_batch_create(sgm_batch_t* out) {
  if (!out) return SGM_ERR_ARG;
  *out = new sgm_batch();
  return SGM_OK;
}

int sgm_batch_destroy(sgm_batch_t b) {
  if (!b) return SGM_ERR_ARG;
  b->free_all();
  delete b;
  return SGM_OK;
}

const char* sgm_batch_last_error(sgm_batch_t b) { return b ? b->err.c_str() : ""; }

static int batch_init_impl(sgm_batch_t b, const sgm_batch_pair_t* pairs, int32_t count, const sgm_option_t* option,
                           const sgm_ext_options_t* ext) {
  if (!b) return SGM_ERR_ARG;
  if (!pairs || !option || count <= 0) return berr(b, SGM_ERR_ARG, "empty batch or null argument");
  if (count > 4096) return berr(b, SGM_ERR_ARG, "at most 4096 pairs per batch (got %d)", count);
  for (int i = 0; i < count; ++i) {
    const auto& p = pairs[i];
    if (p.width <= 0 || p.height <= 0) return berr(b, SGM_ERR_ARG, "pair %d: image size error (%dx%d)", i, p.width, p.height);
    if (p.disp_range != 32 && p.disp_range != 64 && p.disp_range != 128)
      return berr(b, SGM_ERR_UNSUPPORTED, "pair %d: disparity range %d unsupported in a batch (32, 64, 128)", i,
                  p.disp_range);
    if ((size_t)p.width * p.height > (size_t)INT32_MAX / 2) return berr(b, SGM_ERR_ARG, "pair %d: image too large", i);
  }
  if (option->cs_type != 0 && option->cs_type != 1) return berr(b, SGM_ERR_ARG, "census type %d invalid", option->cs_type);
  if (option->p1 < 0 || option->p2_init < 0) return berr(b, SGM_ERR_ARG, "negative penalties");
  if (option->do_remove_peaks || option->morphology_type != 0 || option->post_filter_type != 0)
    return berr(b, SGM_ERR_UNSUPPORTED, "small-region removal, morphology and post filters are per-pair stages; "
                                        "use sgm_init / sgm_match_device");
  if (!option->using_constant_p2) return berr(b, SGM_ERR_UNSUPPORTED, "batches need using_constant_p2");
  sgm_ext_options_t ex{};
  ex.tie_rule = ex.init_tie_rule = 4;
  ex.p2_div0 = -1;
  if (ext) ex = *ext;
  if (ex.tie_rule < 0 || ex.tie_rule > 4) return berr(b, SGM_ERR_ARG, "tie rule %d out of range", ex.tie_rule);
  b->free_all();
  b->pairs.assign(pairs, pairs + count);
  b->opt = *option;
  b->ext = ex;
  b->word = option->cs_type == 1 ? 8 : 4;
  BTRY(b, cudaGetDevice(&b->dev));
  BTRY(b, cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->dev));
  BTRY(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));

  // arena layout
  const int nv = option->do_lr_check ? 2 : 1;
  std::vector<size_t> off(count);
  size_t total = 0;
  struct Sz { size_t img, cs, vol, wta, out; };
  std::vector<Sz> sz(count);
  for (int i = 0; i < count; ++i) {
    const size_t N = (size_t)pairs[i].width * pairs[i].height;
    const size_t V = N * pairs[i].disp_range;
    sz[i] = {align256(N), align256(N * b->word), align256(nv * V), align256(2 * N * sizeof(float)),
             align256(N * sizeof(float))};
    off[i] = total;
    total += 2 * sz[i].img + 2 * sz[i].cs + 4 * sz[i].vol + sz[i].wta + sz[i].out;
  }
  b->arena_bytes = total;
  BTRY(b, sgm_dev_malloc(&b->arena, total));
  b->hdesc.resize(count);
  for (int i = 0; i < count; ++i) {
    unsigned char* p = b->arena + off[i];
    BatchPair& d = b->hdesc[i];
    const auto& q = pairs[i];
    d.img_l = p; p += sz[i].img;
    d.img_r = p; p += sz[i].img;
    d.cs_l = p; p += sz[i].cs;
    d.cs_r = p; p += sz[i].cs;
    d.cost = p; p += sz[i].vol;
    d.lr = p; p += sz[i].vol;
    d.rl = p; p += sz[i].vol;
    d.bt = p; p += sz[i].vol;
    d.wta = reinterpret_cast<float*>(p); p += sz[i].wta;
    d.out = reinterpret_cast<float*>(p);
    d.P.W = q.width; d.P.H = q.height; d.P.min_d = q.min_disparity; d.P.x0 = std::max(0, q.min_disparity);
    d.P.p1 = (uint32_t)option->p1; d.P.p2 = (uint32_t)option->p2_init;
    d.P.vstride = (size_t)q.width * q.height * q.disp_range;
    d.Q.uniqueness = option->unique_threshold;
    d.Q.tie_rule = ex.tie_rule;
    d.Q.rows = (q.height / 2) * 2;
    d.Q.dmax_excl = q.disp_range;
    d.Q.dstride = (size_t)q.width * q.height;
    d.Q.image_border(q.width, q.height);
    d.nv = nv;
  }
  BTRY(b, sgm_dev_malloc(&b->ddesc, sizeof(BatchPair) * count));
  BTRY(b, cudaMemcpy(b->ddesc, b->hdesc.data(), sizeof(BatchPair) * count, cudaMemcpyHostToDevice));

  // buckets by (D, width class); item tables
  std::map<std::pair<int, int>, std::vector<int>> groups;
  for (int i = 0; i < count; ++i) groups[{pairs[i].disp_range / 32, width_class(pairs[i].width)}].push_back(i);
  std::vector<int> tab;
  auto prefix_of = [&](const std::vector<int>& ids, auto per_item) {
    const int at = (int)tab.size();
    int acc = 0;
    for (int id : ids) { tab.push_back(acc); acc += per_item(id); }
    tab.push_back(acc);
    return std::make_pair(at, acc);
  };
  std::vector<int> all(count);
  for (int i = 0; i < count; ++i) all[i] = i;
  auto cp = prefix_of(all, [&](int i) { return 2 * ((pairs[i].height + sgm::kCensusRows - 1) / sgm::kCensusRows); });
  b->census_prefix = cp.first; b->census_items = cp.second;
  auto tp = prefix_of(all, [&](int i) {  // LR/median tiles
    return ((pairs[i].width + 31) / 32) * ((pairs[i].height + kLrmRows - 1) / kLrmRows);
  });
  b->tile_prefix = tp.first; b->tile_items = tp.second;
  for (auto& g : groups) {
    sgm_batch::Bucket k;
    k.K = g.first.first;
    k.wclass = g.first.second;
    k.members = g.second;
    std::vector<int> by_w = g.second, by_h = g.second;  // longest work first
    std::stable_sort(by_w.begin(), by_w.end(), [&](int a, int c) { return pairs[a].width > pairs[c].width; });
    std::stable_sort(by_h.begin(), by_h.end(), [&](int a, int c) { return pairs[a].height > pairs[c].height; });
    k.rows_ids = (int)tab.size();
    tab.insert(tab.end(), by_w.begin(), by_w.end());
    for (int li = 0; li < 5; ++li) {  // items of 1 scanline (li 0) or 32/G scanlines (G = 1, 2, 4, 8)
      const int per = li == 0 ? 1 : 32 >> (li - 1);
      auto rp = prefix_of(by_w, [&](int i) { return (nv * 2 * pairs[i].height + per - 1) / per; });
      k.rows_prefix[li] = rp.first;
      k.rows_items[li] = rp.second;
    }
    auto op = prefix_of(by_w, [&](int i) { return nv * pairs[i].height * ((pairs[i].width + 127) / 128); });
    k.cost_prefix = op.first;
    k.cost_items = op.second;
    k.cols_ids = (int)tab.size();
    tab.insert(tab.end(), by_h.begin(), by_h.end());
    for (int li = 0; li < 5; ++li) {  // items of 1 column (li 0) or 32/G columns of one view
      const int per = li == 0 ? 1 : 32 >> (li - 1);
      auto vp = prefix_of(by_h, [&](int i) { return nv * ((pairs[i].width + per - 1) / per); });
      k.cols_prefix[li] = vp.first;
      k.cols_items[li] = vp.second;
    }
    b->buckets.push_back(k);
  }
  BTRY(b, sgm_dev_malloc(&b->dtab, tab.size() * sizeof(int)));
  BTRY(b, cudaMemcpy(b->dtab, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice));
  b->nqueues = 3 * (int)b->buckets.size();
  BTRY(b, sgm_dev_malloc(&b->queues, b->nqueues * sizeof(int)));
  for (size_t i = 0; i < b->buckets.size(); ++i) {
    cudaStream_t t;
    BTRY(b, cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
    b->side.push_back(t);
    BTRY(b, cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
    b->side2.push_back(t);
  }
  for (size_t i = 0; i < 3 * b->buckets.size() + 1; ++i) {
    cudaEvent_t e;
    BTRY(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev.push_back(e);
  }
  // tune on noise images, then capture the graph
  for (int i = 0; i < count; ++i) {
    const size_t N = (size_t)pairs[i].width * pairs[i].height;
    kb_fill_noise<<<64, 256, 0, b->stream>>>(const_cast<uint8_t*>(b->hdesc[i].img_l), N, 17u + 2u * i);
    kb_fill_noise<<<64, 256, 0, b->stream>>>(const_cast<uint8_t*>(b->hdesc[i].img_r), N, 18u + 2u * i);
  }
  BTRY(b, cudaGetLastError());
  int st = autotune(b, false);
  if (st) return st;
  st = capture(b);
  if (st) return st;
  BTRY(b, cudaStreamSynchronize(b->stream));
  b->ready = true;
  return SGM_OK;
}

int sgm_batch_init(sgm_batch_t b, const sgm_batch_pair_t* pairs, int32_t count, const sgm_option_t* option,
                   const sgm_ext_options_t* ext) {
  const int st = batch_init_impl(b, pairs, count, option, ext);
  if (st && b) b->free_all();  // a batch whose init failed keeps no device memory
  return st;
}

int sgm_batch_autotune(sgm_batch_t b) {
  if (!b || !b->ready) return b ? berr(b, SGM_ERR_STATE, "batch not initialised") : SGM_ERR_ARG;
  int st = autotune(b, true);
  if (!st) st = capture(b);
  if (!st && cudaStreamSynchronize(b->stream) != cudaSuccess) st = berr(b, SGM_ERR_CUDA, "autotune failed");
  return st;
}

int sgm_batch_pair_buffers(sgm_batch_t b, int32_t index, uint8_t** d_left, uint8_t** d_right, float** d_disp) {
  if (!b || !b->ready) return b ? berr(b, SGM_ERR_STATE, "batch not initialised") : SGM_ERR_ARG;
  if (index < 0 || index >= (int)b->pairs.size()) return berr(b, SGM_ERR_ARG, "pair index %d out of range", index);
  const BatchPair& d = b->hdesc[index];
  if (d_left) *d_left = const_cast<uint8_t*>(d.img_l);
  if (d_right) *d_right = const_cast<uint8_t*>(d.img_r);
  if (d_disp) *d_disp = d.out;
  return SGM_OK;
}

int sgm_batch_run(sgm_batch_t b, void* stream) {
  if (!b || !b->ready) return b ? berr(b, SGM_ERR_STATE, "batch not initialised") : SGM_ERR_ARG;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
  if (sgm_prof_on()) {  // per-launch timing: the same work without the graph, one launch at a time
    const int st = run_timed(b, s);
    if (!st) b->runs++;
    return st;
  }
  const cudaError_t ce = cudaGraphLaunch(b->exec, s);
  if (ce != cudaSuccess) return berr(b, SGM_ERR_CUDA, "graph launch failed: %s", cudaGetErrorString(ce));
  b->runs++;
  return SGM_OK;
}

int sgm_batch_match(sgm_batch_t b, const uint8_t* const* left, const uint8_t* const* right, float* const* disp) {
  if (!b || !b->ready) return b ? berr(b, SGM_ERR_STATE, "batch not initialised") : SGM_ERR_ARG;
  if (!left || !right || !disp) return berr(b, SGM_ERR_ARG, "null pointer argument");
  const int n = (int)b->pairs.size();
  for (int i = 0; i < n; ++i)
    if (!left[i] || !right[i] || !disp[i]) return berr(b, SGM_ERR_ARG, "pair %d: null buffer", i);
  cudaStream_t s = b->stream;
  for (int i = 0; i < n; ++i) {
    const size_t N = (size_t)b->pairs[i].width * b->pairs[i].height;
    BTRY(b, cudaMemcpyAsync(const_cast<uint8_t*>(b->hdesc[i].img_l), left[i], N, cudaMemcpyHostToDevice, s));
    BTRY(b, cudaMemcpyAsync(const_cast<uint8_t*>(b->hdesc[i].img_r), right[i], N, cudaMemcpyHostToDevice, s));
  }
  int st = sgm_batch_run(b, s);
  if (st) return st;
  for (int i = 0; i < n; ++i) {
    const size_t N = (size_t)b->pairs[i].width * b->pairs[i].height;
    BTRY(b, cudaMemcpyAsync(disp[i], b->hdesc[i].out, N * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  BTRY(b, cudaStreamSynchronize(s));
  return SGM_OK;
}

int sgm_batch_info(sgm_batch_t b, sgm_batch_info_t* info) {
  if (!b || !info) return SGM_ERR_ARG;
  if (!b->ready) return berr(b, SGM_ERR_STATE, "batch not initialised");
  info->pairs = (int32_t)b->pairs.size();
  info->buckets = (int32_t)b->buckets.size();
  info->arena_bytes = b->arena_bytes;
  info->kernels_per_run = b->graph_kernels;
  return SGM_OK;
}

int sgm_batch_bucket(sgm_batch_t b, int32_t index, sgm_batch_bucket_t* out) {
  if (!b || !out) return SGM_ERR_ARG;
  if (!b->ready || index < 0 || index >= (int)b->buckets.size())
    return berr(b, SGM_ERR_ARG, "bucket index %d out of range", index);
  const auto& k = b->buckets[index];
  out->disp_range = 32 * k.K;
  out->width_class = k.wclass;
  out->pairs = (int32_t)k.members.size();
  out->rows_lanes = k.tune.rows_lanes;
  out->cols_lanes = k.tune.cols_lanes;
  out->rows_warps_per_cta = k.tune.rows_warps;
  out->rows_ctas = k.rows_blocks;
  out->cols_warps_per_cta = k.tune.cols_warps;
  out->cols_prefetch = k.tune.cols_pf;
  out->cols_ctas = k.cols_blocks;
  return SGM_OK;
}

}  // extern "C"

// =============================================================================================
// Batched pyramid: every pair's full pyramid (reference FasterStereoCuda::Match,
// FasterStereoCuda.cpp:408-529) in one graph. The coarsest level of all pairs is a single-level
// batch (its buckets and autotuned kernels above), followed by its dilation and small-region
// removal; each finer 32-disparity level runs census, cost, the uint32 scanline scans (per width
// class bucket, lane split autotuned) and the median for all pairs, then hands its map to the
// next level as initial disparities.
// =============================================================================================
struct sgm_batch_pyr {
  struct Bucket {
    int wclass = 0;
    std::vector<int> members;
    int ids = 0, cost_prefix = 0, cost_items = 0, max_w = 0;
    int rows_prefix[5] = {}, rows_items[5] = {}, cols_prefix[5] = {}, cols_items[5] = {};
    int rows_lanes = 8, cols_lanes = 8, rows_blocks = 0, cols_blocks = 0;
  };
  struct Level {  // a 32-disparity level (index n < layers - 1)
    int n = 0;
    sgm_option_t opt{};
    std::vector<BatchPair> hdesc;
    BatchPair* ddesc = nullptr;
    int census_prefix = 0, census_items = 0, tile_prefix = 0, tile_items = 0;
    int row_prefix = 0, row_items = 0, pix_prefix = 0, pix_items = 0;
    int lrm_prefix = 0, lrm_items = 0;  // LR/median tiles (32 x kLrmRows)
    std::vector<Bucket> buckets;
    int queue0 = 0;
  };
  bool ready = false;
  int dev = 0, nsm = 148, layers = 1, word = 8;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> side;
  std::vector<cudaStream_t> side2;  // the bottom-to-top column pass of each 32-disparity bucket
  std::vector<cudaEvent_t> ev;
  std::vector<sgm_batch_pair_t> pairs;
  sgm_ext_options_t ext{};
  sgm_option_t copt{};  // coarsest level options (dilation / removal applied here)
  sgm_batch* coarse = nullptr;
  std::vector<Level> lv;
  int c_tile_prefix = 0, c_tile_items = 0, c_row_prefix = 0, c_row_items = 0, c_pix_prefix = 0, c_pix_items = 0;
  std::vector<int> dec_prefix, dec_items;  // per level >= 1: rows of the level (decimation)
  unsigned char* arena = nullptr;
  size_t arena_bytes = 0;
  int* dtab = nullptr;
  int* queues = nullptr;
  int nqueues = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t graph_kernels = 0;
  std::string err;

  void free_all() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    if (coarse) {
      coarse->free_all();
      delete coarse;
    }
    coarse = nullptr;
    for (auto& L : lv)
      if (L.ddesc) sgm_dev_free(L.ddesc);
    lv.clear();
    if (arena) sgm_dev_free(arena);
    if (dtab) sgm_dev_free(dtab);
    if (queues) sgm_dev_free(queues);
    arena = nullptr;
    dtab = nullptr;
    queues = nullptr;
    for (auto s : side) cudaStreamDestroy(s);
    side.clear();
    for (auto s : side2) cudaStreamDestroy(s);
    side2.clear();
    for (auto e : ev) cudaEventDestroy(e);
    ev.clear();
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    pairs.clear();
    dec_prefix.clear();
    dec_items.clear();
    ready = false;
  }
};

namespace {

int perr(sgm_batch_pyr* p, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  p->err = buf;
  return code;
}

#define PTRY(p, expr)                                                                         \
  do {                                                                                        \
    cudaError_t _st = (expr);                                                                 \
    if (_st != cudaSuccess)                                                                   \
      return perr(p, _st == cudaErrorMemoryAllocation ? SGM_ERR_NOMEM : SGM_ERR_CUDA, "%s failed: %s", #expr, \
                  cudaGetErrorString(_st));                                                   \
  } while (0)

using PBucket = sgm_batch_pyr::Bucket;
using PLevel = sgm_batch_pyr::Level;

template <typename F>
int psize_grid(sgm_batch_pyr* p, F* fn, int threads, int items, int warps, int* blocks) {
  PTRY(p, sgm::allow_max_dynamic_smem(fn));
  int occ = 0;
  PTRY(p, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, 0));
  *blocks = std::max(1, std::min(p->nsm * std::max(occ, 1), (items + warps - 1) / warps));
  return SGM_OK;
}

int init_rows(sgm_batch_pyr* p, PLevel& L, PBucket& k, cudaStream_t s, int* queue, bool prepare) {
  const int G = k.rows_lanes, li = lanes_index(G), n = (int)k.members.size();
  const int* ids = p->dtab + k.ids;
  const int* pre = p->dtab + k.rows_prefix[li];
  auto go = [&](auto fn) -> int {
    if (prepare) return psize_grid(p, fn, 128, k.rows_items[li], 4, &k.rows_blocks);
    fn<<<k.rows_blocks, 128, 0, s>>>(L.ddesc, ids, pre, n, queue);
    PTRY(p, cudaGetLastError());
    return SGM_OK;
  };
  return G == 2 ? go(kb_rows3_init<2, 8>) : G == 4 ? go(kb_rows3_init<4, 8>) : go(kb_rows3_init<8, 8>);
}

// PASS: 0 both column passes, 1 bottom-to-top only, 2 top-to-bottom + WTA only (the persistent
// grid is sized for PASS 0; the queue counts any grid).
template <int PASS = 0>
int init_cols(sgm_batch_pyr* p, PLevel& L, PBucket& k, cudaStream_t s, int* queue, bool prepare) {
  const int G = k.cols_lanes, li = lanes_index(G), n = (int)k.members.size();
  const int* ids = p->dtab + k.ids;
  const int* pre = p->dtab + k.cols_prefix[li];
  auto go = [&](auto fn) -> int {
    if (prepare) return psize_grid(p, fn, 128, k.cols_items[li], 4, &k.cols_blocks);
    fn<<<k.cols_blocks, 128, 0, s>>>(L.ddesc, ids, pre, n, queue);
    PTRY(p, cudaGetLastError());
    return SGM_OK;
  };
  if (prepare) return G == 2 ? go(kb_cols3_init<2, 1>) : G == 4 ? go(kb_cols3_init<4, 4>) : go(kb_cols3_init<8, 4>);
  return G == 2   ? go(kb_cols3_init<2, 1, PASS>)
         : G == 4 ? go(kb_cols3_init<4, 4, PASS>)
                  : go(kb_cols3_init<8, 4, PASS>);
}

int init_cost(sgm_batch_pyr* p, PLevel& L, PBucket& k, cudaStream_t s) {
  const size_t smem = (size_t)k.max_w * p->word;
  const int n = (int)k.members.size();
  if (p->word == 8) {
    PTRY(p, sgm::allow_max_dynamic_smem(kb_cost3_init<uint64_t>));
    kb_cost3_init<uint64_t><<<k.cost_items, 256, smem, s>>>(L.ddesc, p->dtab + k.ids, p->dtab + k.cost_prefix, n);
  } else {
    PTRY(p, sgm::allow_max_dynamic_smem(kb_cost3_init<uint32_t>));
    kb_cost3_init<uint32_t><<<k.cost_items, 256, smem, s>>>(L.ddesc, p->dtab + k.ids, p->dtab + k.cost_prefix, n);
  }
  PTRY(p, cudaGetLastError());
  return SGM_OK;
}

// Median (and LR when set) of one level into post (dilation next) or out.
int level_post(sgm_batch_pyr* p, const BatchPair* d, const int* tpre, int tiles, int n, const sgm_option_t& o,
               cudaStream_t s) {
  const dim3 blk(32, 8);
  const float thr = o.lr_threshold;
  if (o.do_lr_check && o.do_median_filter) kb_lr_median<true, true><<<tiles, blk, 0, s>>>(d, tpre, n, thr);
  else if (o.do_lr_check) kb_lr_median<true, false><<<tiles, blk, 0, s>>>(d, tpre, n, thr);
  else if (o.do_median_filter) kb_lr_median<false, true><<<tiles, blk, 0, s>>>(d, tpre, n, thr);
  else kb_lr_median<false, false><<<tiles, blk, 0, s>>>(d, tpre, n, thr);
  PTRY(p, cudaGetLastError());
  return SGM_OK;
}

// Dilation and small-region removal of one level, when its options ask for them (prof: each
// launch timed alone).
int level_filters(sgm_batch_pyr* p, const BatchPair* d, const sgm_option_t& o, int tpre, int tiles, int rpre, int rows,
                  int ppre, int pix, int n, cudaStream_t s, int64_t* kernels, bool prof = false) {
  auto T = [&](const char* name, auto launch) {
    timed(prof, s, name, [&] {
      launch();
      return SGM_OK;
    });
    (*kernels)++;
  };
  if (o.post_filter_type == 1)  // the LR/median stage wrote `post`
    T("gauss", [&] { kb_gauss<<<tiles, dim3(32, 8), 0, s>>>(d, p->dtab + tpre, n); });
  if (o.morphology_type == 2)
    T("dilation", [&] { kb_dilation<<<tiles, dim3(32, 8), 0, s>>>(d, p->dtab + tpre, n); });
  if (o.do_remove_peaks) {
    const int am = p->ext.peaks_abs_mode;
    T("cc_rows", [&] { kb_cc_rows<<<(rows + 7) / 8, dim3(32, 8), 0, s>>>(d, p->dtab + rpre, n, am); });
    T("cc_vert", [&] { kb_cc_vert<<<(pix + 255) / 256, 256, 0, s>>>(d, p->dtab + ppre, n, am); });
    T("cc_count", [&] { kb_cc_count<<<(pix + 255) / 256, 256, 0, s>>>(d, p->dtab + ppre, n); });
    T("cc_filter",
      [&] { kb_cc_filter<<<(pix + 255) / 256, 256, 0, s>>>(d, p->dtab + ppre, n, o.peaks_ratio_threshold); });
  }
  PTRY(p, cudaGetLastError());
  return SGM_OK;
}

int level_census(sgm_batch_pyr* p, const BatchPair* d, int cpre, int citems, int n, cudaStream_t s) {
  const int blocks = citems;  // one block per (pair, view, row block)
  if (p->word == 8) kb_census4<uint64_t, 4, 3><<<blocks, 128, 0, s>>>(d, p->dtab + cpre, n);
  else kb_census4<uint32_t, 2, 2><<<blocks, 128, 0, s>>>(d, p->dtab + cpre, n);
  PTRY(p, cudaGetLastError());
  return SGM_OK;
}

// Lane splits of each 32-disparity bucket, timed on this batch's shapes (noise images, zero
// initial disparities); every split gives the same result.
int pyr_autotune(sgm_batch_pyr* p) {
  const int npairs = (int)p->pairs.size();
  for (auto& L : p->lv) {
    int st0 = level_census(p, L.ddesc, L.census_prefix, L.census_items, npairs, p->stream);
    if (st0) return st0;
    for (size_t bi = 0; bi < L.buckets.size(); ++bi) {
      auto& k = L.buckets[bi];
      int* q = p->queues + L.queue0 + 3 * bi;
      int st = init_cost(p, L, k, p->stream);
      if (st) return st;
      float best = 1e30f;
      int bg = 8;
      for (int G : {2, 4, 8}) {
        k.rows_lanes = G;
        st = init_rows(p, L, k, nullptr, nullptr, true);
        if (st) return st;
        cudaEvent_t e0, e1;
        PTRY(p, cudaEventCreate(&e0));
        PTRY(p, cudaEventCreate(&e1));
        for (int r = 0; r < 2 && !st; ++r) {
          if (r == 1) cudaEventRecord(e0, p->stream);
          cudaMemsetAsync(q, 0, 2 * sizeof(int), p->stream);
          st = init_rows(p, L, k, p->stream, q, false);
        }
        cudaEventRecord(e1, p->stream);
        float ms = 0;
        if (!st && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st) return st;
        if (ms < best) { best = ms; bg = G; }
      }
      k.rows_lanes = bg;
      best = 1e30f;
      bg = 8;
      for (int G : {2, 4, 8}) {
        k.cols_lanes = G;
        st = init_cols(p, L, k, nullptr, nullptr, true);
        if (st) return st;
        cudaEvent_t e0, e1;
        PTRY(p, cudaEventCreate(&e0));
        PTRY(p, cudaEventCreate(&e1));
        for (int r = 0; r < 2 && !st; ++r) {
          if (r == 1) cudaEventRecord(e0, p->stream);
          cudaMemsetAsync(q + 1, 0, sizeof(int), p->stream);
          st = init_cols(p, L, k, p->stream, q + 1, false);
        }
        cudaEventRecord(e1, p->stream);
        float ms = 0;
        if (!st && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st) return st;
        if (ms < best) { best = ms; bg = G; }
      }
      k.cols_lanes = bg;
      st = init_rows(p, L, k, nullptr, nullptr, true);
      if (!st) st = init_cols(p, L, k, nullptr, nullptr, true);
      if (st) return st;
    }
  }
  return SGM_OK;
}

}  // namespace

namespace {

// census -> per-bucket [cost, rows, cols] -> LR/median of the coarsest level (the single-level
// batch's stages), then its dilation and small-region removal; then, for every finer level, the
// next-level initial disparities, census, per-bucket [cost, rows, cols], median.
int pyr_capture(sgm_batch_pyr* p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->exec = nullptr;
  p->graph = nullptr;
  cudaStream_t s = p->stream;
  sgm_batch* c = p->coarse;
  const int n = (int)p->pairs.size();
  const int Lc = p->layers - 1;
  PTRY(p, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int st = SGM_OK;
  int64_t kernels = 0;
  int evi = 0;
  auto fork_join = [&](int nb, auto body) {
    cudaEventRecord(p->ev[evi], s);
    const int fork = evi++;
    for (int i = 0; i < nb && !st; ++i) {
      cudaStream_t t = p->side[i];
      cudaStreamWaitEvent(t, p->ev[fork], 0);
      st = body(i, t);
      cudaEventRecord(p->ev[evi], t);
      cudaStreamWaitEvent(s, p->ev[evi], 0);
      ++evi;
    }
  };
  if (cudaMemsetAsync(c->queues, 0, c->nqueues * sizeof(int), s) != cudaSuccess ||
      (p->nqueues && cudaMemsetAsync(p->queues, 0, p->nqueues * sizeof(int), s) != cudaSuccess))
    st = perr(p, SGM_ERR_CUDA, "queue reset failed");
  // level images from the full-resolution images
  for (int lvl = 1; lvl < p->layers && !st; ++lvl) {
    const BatchPair* dst = lvl == Lc ? c->ddesc : p->lv[lvl].ddesc;
    kb_decimate<<<p->dec_items[lvl], 128, 0, s>>>(dst, p->lv[0].ddesc, p->dtab + p->dec_prefix[lvl], n, lvl);
    kernels++;
    if (cudaGetLastError() != cudaSuccess) st = perr(p, SGM_ERR_CUDA, "decimation launch failed");
  }
  // coarsest level
  if (!st) { st = launch_census(c, s); kernels++; }
  if (!st)
    fork_join((int)c->buckets.size(), [&](int i, cudaStream_t t) {
      const int ea = evi++, eb = evi++;
      return bucket_scans(c, c->buckets[i], t, p->side2[i], p->ev[ea], p->ev[eb], c->queues + 3 * i, &kernels);
    });
  if (!st) { st = launch_post(c, s); kernels++; }
  if (!st)
    st = level_filters(p, c->ddesc, p->copt, p->c_tile_prefix, p->c_tile_items, p->c_row_prefix, p->c_row_items,
                       p->c_pix_prefix, p->c_pix_items, n, s, &kernels);
  // finer levels
  for (int lvl = Lc - 1; lvl >= 0 && !st; --lvl) {
    PLevel& L = p->lv[lvl];
    const BatchPair* above = lvl == Lc - 1 ? c->ddesc : p->lv[lvl + 1].ddesc;
    kb_init_next<<<(L.row_items + 7) / 8, dim3(32, 8), 0, s>>>(L.ddesc, above, p->dtab + L.row_prefix, n);
    kernels++;
    if (cudaGetLastError() != cudaSuccess) st = perr(p, SGM_ERR_CUDA, "initial-disparity launch failed");
    if (!st) { st = level_census(p, L.ddesc, L.census_prefix, L.census_items, n, s); kernels++; }
    if (!st)
      fork_join((int)L.buckets.size(), [&](int i, cudaStream_t t) {
        // the bottom-to-top pass (cost volume only) on side2 beside the row scans
        int* q = p->queues + L.queue0 + 3 * i;
        int r = init_cost(p, L, L.buckets[i], t);
        cudaStream_t t2 = p->side2[i];
        cudaEventRecord(p->ev[evi], t);
        cudaStreamWaitEvent(t2, p->ev[evi++], 0);
        if (!r) r = init_cols<1>(p, L, L.buckets[i], t2, q + 1, false);
        if (!r) r = init_rows(p, L, L.buckets[i], t, q, false);
        cudaEventRecord(p->ev[evi], t2);
        cudaStreamWaitEvent(t, p->ev[evi++], 0);
        if (!r) r = init_cols<2>(p, L, L.buckets[i], t, q + 2, false);
        kernels += 4;
        return r;
      });
    if (!st) { st = level_post(p, L.ddesc, p->dtab + L.lrm_prefix, L.lrm_items, n, L.opt, s); kernels++; }
    if (!st)
      st = level_filters(p, L.ddesc, L.opt, L.tile_prefix, L.tile_items, L.row_prefix, L.row_items, L.pix_prefix,
                         L.pix_items, n, s, &kernels);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (st) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (ce != cudaSuccess) return perr(p, SGM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
  p->graph = g;
  PTRY(p, cudaGraphInstantiate(&p->exec, g, 0));
  p->graph_kernels = kernels;
  return SGM_OK;
}

// pyr_capture's work enqueued directly on s, one launch after another in a valid order (the
// column passes and the row scans of a bucket in sequence), each timed alone.
int pyr_run_timed(sgm_batch_pyr* p, cudaStream_t s) {
  sgm_batch* c = p->coarse;
  const int n = (int)p->pairs.size();
  const int Lc = p->layers - 1;
  if (cudaMemsetAsync(c->queues, 0, c->nqueues * sizeof(int), s) != cudaSuccess ||
      (p->nqueues && cudaMemsetAsync(p->queues, 0, p->nqueues * sizeof(int), s) != cudaSuccess))
    return perr(p, SGM_ERR_CUDA, "queue reset failed");
  int st = SGM_OK;
  int64_t kernels = 0;
  for (int lvl = 1; lvl < p->layers && !st; ++lvl) {
    const BatchPair* dst = lvl == Lc ? c->ddesc : p->lv[lvl].ddesc;
    st = timed(true, s, "decimate", [&] {
      kb_decimate<<<p->dec_items[lvl], 128, 0, s>>>(dst, p->lv[0].ddesc, p->dtab + p->dec_prefix[lvl], n, lvl);
      return cudaGetLastError() == cudaSuccess ? SGM_OK : perr(p, SGM_ERR_CUDA, "decimation launch failed");
    });
  }
  if (!st) st = timed(true, s, "census", [&] { return launch_census(c, s); });
  for (size_t i = 0; !st && i < c->buckets.size(); ++i) st = bucket_scans_timed(c, c->buckets[i], s, c->queues + 3 * i);
  if (!st) st = timed(true, s, "lr_median", [&] { return launch_post(c, s); });
  if (!st)
    st = level_filters(p, c->ddesc, p->copt, p->c_tile_prefix, p->c_tile_items, p->c_row_prefix, p->c_row_items,
                       p->c_pix_prefix, p->c_pix_items, n, s, &kernels, true);
  for (int lvl = Lc - 1; lvl >= 0 && !st; --lvl) {
    PLevel& L = p->lv[lvl];
    const BatchPair* above = lvl == Lc - 1 ? c->ddesc : p->lv[lvl + 1].ddesc;
    st = timed(true, s, "init_next_level", [&] {
      kb_init_next<<<(L.row_items + 7) / 8, dim3(32, 8), 0, s>>>(L.ddesc, above, p->dtab + L.row_prefix, n);
      return cudaGetLastError() == cudaSuccess ? SGM_OK : perr(p, SGM_ERR_CUDA, "initial-disparity launch failed");
    });
    if (!st)
      st = timed(true, s, "census", [&] { return level_census(p, L.ddesc, L.census_prefix, L.census_items, n, s); });
    for (size_t i = 0; !st && i < L.buckets.size(); ++i) {
      PBucket& k = L.buckets[i];
      int* q = p->queues + L.queue0 + 3 * i;
      st = timed(true, s, "cost", [&] { return init_cost(p, L, k, s); });
      if (!st) st = timed(true, s, "vpaths_bt_init", [&] { return init_cols<1>(p, L, k, s, q + 1, false); });
      if (!st) st = timed(true, s, "hpaths_init", [&] { return init_rows(p, L, k, s, q, false); });
      if (!st) st = timed(true, s, "vpaths_wta_init", [&] { return init_cols<2>(p, L, k, s, q + 2, false); });
    }
    if (!st)
      st = timed(true, s, "lr_median",
                 [&] { return level_post(p, L.ddesc, p->dtab + L.lrm_prefix, L.lrm_items, n, L.opt, s); });
    if (!st)
      st = level_filters(p, L.ddesc, L.opt, L.tile_prefix, L.tile_items, L.row_prefix, L.row_items, L.pix_prefix,
                         L.pix_items, n, s, &kernels, true);
  }
  return st;
}

}  // namespace

extern "C" {

int sgm_batch_pyr_create(sgm_batch_pyr_t* out) {
  if (!out) return SGM_ERR_ARG;
  *out = new sgm_batch_pyr();
  return SGM_OK;
}

int sgm_batch_pyr_destroy(sgm_batch_pyr_t p) {
  if (!p) return SGM_ERR_ARG;
  p->free_all();
  delete p;
  return SGM_OK;
}

const char* sgm_batch_pyr_last_error(sgm_batch_pyr_t p) { return p ? p->err.c_str() : ""; }

static int batch_pyr_init_impl(sgm_batch_pyr_t p, const sgm_batch_pair_t* pairs, int32_t count,
                               const sgm_pyr_option1_t* option, const sgm_level_override_t* ov,
                               const sgm_ext_options_t* ext) {
  if (!p) return SGM_ERR_ARG;
  if (!pairs || !option || count <= 0) return perr(p, SGM_ERR_ARG, "empty batch or null argument");
  if (count > 4096) return perr(p, SGM_ERR_ARG, "at most 4096 pairs per batch (got %d)", count);

  const int layers = std::max(1, option->num_layers);
  sgm_ext_options_t ex{};
  ex.tie_rule = ex.init_tie_rule = sgm::kTieRefB200;
  ex.p2_div0 = -1;
  if (ext) ex = *ext;
  if (layers > 1 && ex.init_tie_rule != sgm::kTieLowest && ex.init_tie_rule != sgm::kTieRefB200)
    return perr(p, SGM_ERR_UNSUPPORTED, "batched pyramids support initial-disparity tie rules 0 and 4");
  for (int i = 0; i < count; ++i) {
    if (pairs[i].width <= 0 || pairs[i].height <= 0 || pairs[i].disp_range <= 0)
      return perr(p, SGM_ERR_ARG, "pair %d: size or disparity range error", i);
    if ((pairs[i].width >> (layers - 1)) < 8 || (pairs[i].height >> (layers - 1)) < 8)
      return perr(p, SGM_ERR_ARG, "pair %d: too many layers for a %dx%d image", i, pairs[i].width, pairs[i].height);
  }
  p->free_all();
  p->pairs.assign(pairs, pairs + count);
  p->layers = layers;
  p->ext = ex;
  PTRY(p, cudaGetDevice(&p->dev));
  PTRY(p, cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, p->dev));
  PTRY(p, cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  const int Lc = layers - 1;
  auto o1_of = [&](int i) {
    sgm_pyr_option1_t o = *option;
    o.width = pairs[i].width;
    o.height = pairs[i].height;
    o.min_disp = pairs[i].min_disparity;
    o.max_disp = pairs[i].min_disparity + pairs[i].disp_range;
    return o;
  };
  // coarsest level: a single-level batch without its dilation / removal (applied here)
  std::vector<sgm_batch_pair_t> cp(count);
  sgm_option_t copt{};
  for (int i = 0; i < count; ++i) {
    const sgm_pyr_option1_t o = o1_of(i);
    int dmin = 0, dr = 0;
    level_options(&o, ov, Lc, layers, &copt, &dmin, &dr);
    cp[i] = {pairs[i].width >> Lc, pairs[i].height >> Lc, dmin, dr};
  }
  p->copt = copt;
  p->word = copt.cs_type == 1 ? 8 : 4;
  sgm_option_t cbatch = copt;  // the parent applies smoothing, dilation and removal
  cbatch.do_remove_peaks = false;
  cbatch.morphology_type = 0;
  cbatch.post_filter_type = 0;
  p->coarse = new sgm_batch();
  int st = sgm_batch_init(p->coarse, cp.data(), count, &cbatch, &ex);
  if (st) return perr(p, st, "coarsest level: %s", p->coarse->err.c_str());
  // finer levels: arena
  p->lv.resize(Lc);
  struct Sz { size_t img, cs, vol, n4, n2; };
  size_t total = 0;
  std::vector<std::vector<size_t>> off(Lc, std::vector<size_t>(count));
  const bool cdil = copt.morphology_type == 2, cpeaks = copt.do_remove_peaks;
  for (int lvl = 0; lvl < Lc; ++lvl) {
    int dmin = 0, dr = 0;
    const sgm_pyr_option1_t o0 = o1_of(0);
    level_options(&o0, ov, lvl, layers, &p->lv[lvl].opt, &dmin, &dr);
    p->lv[lvl].n = lvl;
    const sgm_option_t& lo = p->lv[lvl].opt;
    if (lo.do_lr_check) return perr(p, SGM_ERR_UNSUPPORTED, "LR check at an initial-disparity level");
    if (lo.post_filter_type == 1 && lo.morphology_type == 2)
      return perr(p, SGM_ERR_UNSUPPORTED, "smoothing and dilation at the same level");
    for (int i = 0; i < count; ++i) {
      const size_t N = (size_t)(pairs[i].width >> lvl) * (pairs[i].height >> lvl);
      off[lvl][i] = total;
      total += 2 * align256(N) + 2 * align256(N * p->word) + 4 * align256(N * sgm::kLevelRange) +
               3 * align256(N * 4) + align256(N * 2) + (lo.do_remove_peaks ? 2 * align256(N * 4) : 0);
    }
  }
  const bool cpf = copt.post_filter_type == 1;
  if (cpf && cdil) return perr(p, SGM_ERR_UNSUPPORTED, "smoothing and dilation at the same level");
  std::vector<size_t> coff(count);
  for (int i = 0; i < count; ++i) {
    const size_t N = (size_t)cp[i].width * cp[i].height;
    coff[i] = total;
    total += (cdil || cpf ? align256(N * 4) : 0) + (cpeaks ? 2 * align256(N * 4) : 0);
  }
  p->arena_bytes = total + p->coarse->arena_bytes;
  if (total) PTRY(p, sgm_dev_malloc(&p->arena, total));
  // coarsest-level descriptors: post-processing buffers
  int strips = ex.peaks_strips > 0 ? ex.peaks_strips : default_peaks_strips();
  for (int i = 0; i < count; ++i) {
    BatchPair& d = p->coarse->hdesc[i];
    unsigned char* q = p->arena + coff[i];
    const size_t N = (size_t)cp[i].width * cp[i].height;
    if (cdil || cpf) {
      d.post = reinterpret_cast<float*>(q);
      q += align256(N * 4);
      const int s2 = std::min(cp[i].width, cp[i].height);
      d.dil_wth = ((s2 < 360 ? 3 : (s2 < 720 ? 5 : 7)) - 1) / 2;
    }
    if (cpeaks) {
      d.label = reinterpret_cast<int*>(q);
      q += align256(N * 4);
      d.count = reinterpret_cast<int*>(q);
      d.peaks_tiles = cp[i].height / strips;
      d.peaks_rows = strips * d.peaks_tiles;
    }
  }
  PTRY(p, cudaMemcpy(p->coarse->ddesc, p->coarse->hdesc.data(), sizeof(BatchPair) * count, cudaMemcpyHostToDevice));
  // finer-level descriptors
  for (int lvl = 0; lvl < Lc; ++lvl) {
    PLevel& L = p->lv[lvl];
    const sgm_option_t& lo = L.opt;
    L.hdesc.assign(count, BatchPair{});
    for (int i = 0; i < count; ++i) {
      const int w = pairs[i].width >> lvl, h = pairs[i].height >> lvl;
      const size_t N = (size_t)w * h;
      unsigned char* q = p->arena + off[lvl][i];
      BatchPair& d = L.hdesc[i];
      d.img_l = q; q += align256(N);
      d.img_r = q; q += align256(N);
      d.cs_l = q; q += align256(N * p->word);
      d.cs_r = q; q += align256(N * p->word);
      d.cost = q; q += align256(N * sgm::kLevelRange);
      d.lr = q; q += align256(N * sgm::kLevelRange);
      d.rl = q; q += align256(N * sgm::kLevelRange);
      d.bt = q; q += align256(N * sgm::kLevelRange);
      d.wta = reinterpret_cast<float*>(q); q += align256(N * 4);
      d.post = nullptr;
      float* post = reinterpret_cast<float*>(q); q += align256(N * 4);
      d.out = reinterpret_cast<float*>(q); q += align256(N * 4);
      d.init = reinterpret_cast<const int16_t*>(q); q += align256(N * 2);
      if (lo.morphology_type == 2 || lo.post_filter_type == 1) {
        d.post = post;
        const int s2 = std::min(w, h);
        d.dil_wth = ((s2 < 360 ? 3 : (s2 < 720 ? 5 : 7)) - 1) / 2;
      }
      if (lo.do_remove_peaks) {
        d.label = reinterpret_cast<int*>(q); q += align256(N * 4);
        d.count = reinterpret_cast<int*>(q);
        d.peaks_tiles = h / strips;
        d.peaks_rows = strips * d.peaks_tiles;
      }
      d.P.W = w; d.P.H = h; d.P.min_d = 0; d.P.x0 = 0;
      d.P.p1 = (uint32_t)lo.p1; d.P.p2 = (uint32_t)lo.p2_init;
      d.P.vstride = N * sgm::kLevelRange;
      d.Q.uniqueness = lo.unique_threshold;
      d.Q.tie_rule = ex.init_tie_rule;
      d.Q.rows = (h / 4) * 4;
      d.Q.dmax_excl = sgm::kLevelRange - 1;
      d.Q.dstride = N;
      d.Q.image_border(w, h);
      d.nv = 1;
      d.IP.W = w; d.IP.H = h; d.IP.x0 = 0;
      d.IP.p1 = (uint32_t)lo.p1; d.IP.p1s = lo.p1; d.IP.p2s = lo.p2_init; d.IP.p2_div0 = ex.p2_div0;
      d.IP.invalid_cost = lo.cs_type == 1 ? 0xFFu : sgm::kInvalidCost;
      d.IP.vstride = N * sgm::kLevelRange;
    }
    PTRY(p, sgm_dev_malloc(&L.ddesc, sizeof(BatchPair) * count));
    PTRY(p, cudaMemcpy(L.ddesc, L.hdesc.data(), sizeof(BatchPair) * count, cudaMemcpyHostToDevice));
  }
  // item tables
  std::vector<int> tab;
  auto prefix_of = [&](const std::vector<int>& ids, auto per) {
    const int at = (int)tab.size();
    int acc = 0;
    for (int id : ids) { tab.push_back(acc); acc += per(id); }
    tab.push_back(acc);
    return std::make_pair(at, acc);
  };
  std::vector<int> all(count);
  for (int i = 0; i < count; ++i) all[i] = i;
  auto tiles_of = [](int w, int h) { return ((w + 31) / 32) * ((h + 7) / 8); };
  {
    auto t = prefix_of(all, [&](int i) { return tiles_of(cp[i].width, cp[i].height); });
    p->c_tile_prefix = t.first; p->c_tile_items = t.second;
    auto r = prefix_of(all, [&](int i) { return cp[i].height; });
    p->c_row_prefix = r.first; p->c_row_items = r.second;
    auto x = prefix_of(all, [&](int i) { return cp[i].width * cp[i].height; });
    p->c_pix_prefix = x.first; p->c_pix_items = x.second;
  }
  p->dec_prefix.assign(layers, 0);
  p->dec_items.assign(layers, 0);
  for (int lvl = 1; lvl < layers; ++lvl) {
    auto r = prefix_of(all, [&](int i) { return pairs[i].height >> lvl; });
    p->dec_prefix[lvl] = r.first; p->dec_items[lvl] = r.second;
  }
  int nq = 0;
  for (int lvl = 0; lvl < Lc; ++lvl) {
    PLevel& L = p->lv[lvl];
    auto hw = [&](int i) { return std::make_pair(pairs[i].width >> lvl, pairs[i].height >> lvl); };
    auto c = prefix_of(all, [&](int i) { return 2 * ((hw(i).second + sgm::kCensusRows - 1) / sgm::kCensusRows); });
    L.census_prefix = c.first; L.census_items = c.second;
    auto t = prefix_of(all, [&](int i) { return tiles_of(hw(i).first, hw(i).second); });
    L.tile_prefix = t.first; L.tile_items = t.second;
    auto lt = prefix_of(all, [&](int i) {
      return ((hw(i).first + 31) / 32) * ((hw(i).second + kLrmRows - 1) / kLrmRows);
    });
    L.lrm_prefix = lt.first; L.lrm_items = lt.second;
    auto r = prefix_of(all, [&](int i) { return hw(i).second; });
    L.row_prefix = r.first; L.row_items = r.second;
    auto x = prefix_of(all, [&](int i) { return hw(i).first * hw(i).second; });
    L.pix_prefix = x.first; L.pix_items = x.second;
    std::map<int, std::vector<int>> groups;
    for (int i = 0; i < count; ++i) groups[width_class(hw(i).first)].push_back(i);
    for (auto& gr : groups) {
      PBucket k;
      k.wclass = gr.first;
      k.members = gr.second;
      std::stable_sort(k.members.begin(), k.members.end(),
                       [&](int a, int b2) { return hw(a).first * 2 + hw(a).second > hw(b2).first * 2 + hw(b2).second; });
      k.ids = (int)tab.size();
      tab.insert(tab.end(), k.members.begin(), k.members.end());
      for (int i : k.members) k.max_w = std::max(k.max_w, hw(i).first);
      auto cc = prefix_of(k.members, [&](int i) { return hw(i).second; });
      k.cost_prefix = cc.first; k.cost_items = cc.second;
      for (int li = 1; li < 5; ++li) {
        const int per = 32 >> (li - 1);
        auto rp = prefix_of(k.members, [&](int i) { return (2 * hw(i).second + per - 1) / per; });
        k.rows_prefix[li] = rp.first; k.rows_items[li] = rp.second;
        auto vp = prefix_of(k.members, [&](int i) { return (hw(i).first + per - 1) / per; });
        k.cols_prefix[li] = vp.first; k.cols_items[li] = vp.second;
      }
      L.buckets.push_back(k);
    }
    L.queue0 = nq;
    nq += 3 * (int)L.buckets.size();  // rows, bottom-to-top, top-to-bottom + WTA
  }
  PTRY(p, sgm_dev_malloc(&p->dtab, tab.size() * sizeof(int)));
  PTRY(p, cudaMemcpy(p->dtab, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice));
  p->nqueues = nq;
  if (nq) PTRY(p, sgm_dev_malloc(&p->queues, nq * sizeof(int)));
  size_t nside = p->coarse->buckets.size();
  int nev = 1 + 3 * (int)p->coarse->buckets.size();
  for (auto& L : p->lv) {
    nside = std::max(nside, L.buckets.size());
    nev += 1 + 3 * (int)L.buckets.size();
  }
  for (size_t i = 0; i < nside; ++i) {
    cudaStream_t t;
    PTRY(p, cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
    p->side.push_back(t);
    PTRY(p, cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
    p->side2.push_back(t);
  }
  for (int i = 0; i < nev; ++i) {
    cudaEvent_t e;
    PTRY(p, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    p->ev.push_back(e);
  }
  // tune the 32-disparity levels on noise images with zero initial disparities, then capture
  for (int lvl = 0; lvl < Lc; ++lvl)
    for (int i = 0; i < count; ++i) {
      const size_t N = (size_t)(pairs[i].width >> lvl) * (pairs[i].height >> lvl);
      BatchPair& d = p->lv[lvl].hdesc[i];
      kb_fill_noise<<<64, 256, 0, p->stream>>>(const_cast<uint8_t*>(d.img_l), N, 31u + 2u * i);
      kb_fill_noise<<<64, 256, 0, p->stream>>>(const_cast<uint8_t*>(d.img_r), N, 32u + 2u * i);
      PTRY(p, cudaMemsetAsync(const_cast<int16_t*>(d.init), 0, N * 2, p->stream));
    }
  PTRY(p, cudaGetLastError());
  st = pyr_autotune(p);
  if (st) return st;
  st = pyr_capture(p);
  if (st) return st;
  PTRY(p, cudaStreamSynchronize(p->stream));
  p->ready = true;
  return SGM_OK;
}

int sgm_batch_pyr_init(sgm_batch_pyr_t p, const sgm_batch_pair_t* pairs, int32_t count,
                       const sgm_pyr_option1_t* option, const sgm_level_override_t* ov, const sgm_ext_options_t* ext) {
  const int st = batch_pyr_init_impl(p, pairs, count, option, ov, ext);
  if (st && p) p->free_all();  // a batch whose init failed keeps no device memory
  return st;
}

int sgm_batch_pyr_pair_buffers(sgm_batch_pyr_t p, int32_t index, uint8_t** d_left, uint8_t** d_right,
                               float** d_disp) {
  if (!p || !p->ready) return p ? perr(p, SGM_ERR_STATE, "batch not initialised") : SGM_ERR_ARG;
  if (index < 0 || index >= (int)p->pairs.size()) return perr(p, SGM_ERR_ARG, "pair index %d out of range", index);
  const BatchPair& d = p->layers > 1 ? p->lv[0].hdesc[index] : p->coarse->hdesc[index];
  if (d_left) *d_left = const_cast<uint8_t*>(d.img_l);
  if (d_right) *d_right = const_cast<uint8_t*>(d.img_r);
  if (d_disp) *d_disp = d.out;
  return SGM_OK;
}

int sgm_batch_pyr_run(sgm_batch_pyr_t p, void* stream) {
  if (!p || !p->ready) return p ? perr(p, SGM_ERR_STATE, "batch not initialised") : SGM_ERR_ARG;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
  if (sgm_prof_on()) return pyr_run_timed(p, s);  // per-launch timing: the same work without the graph
  const cudaError_t ce = cudaGraphLaunch(p->exec, s);
  if (ce != cudaSuccess) return perr(p, SGM_ERR_CUDA, "graph launch failed: %s", cudaGetErrorString(ce));
  return SGM_OK;
}

int sgm_batch_pyr_match(sgm_batch_pyr_t p, const uint8_t* const* left, const uint8_t* const* right,
                        float* const* disp) {
  if (!p || !p->ready) return p ? perr(p, SGM_ERR_STATE, "batch not initialised") : SGM_ERR_ARG;
  if (!left || !right || !disp) return perr(p, SGM_ERR_ARG, "null pointer argument");
  const int n = (int)p->pairs.size();
  cudaStream_t s = p->stream;
  for (int i = 0; i < n; ++i) {
    if (!left[i] || !right[i] || !disp[i]) return perr(p, SGM_ERR_ARG, "pair %d: null buffer", i);
    uint8_t *dl, *dr;
    sgm_batch_pyr_pair_buffers(p, i, &dl, &dr, nullptr);
    const size_t N = (size_t)p->pairs[i].width * p->pairs[i].height;
    PTRY(p, cudaMemcpyAsync(dl, left[i], N, cudaMemcpyHostToDevice, s));
    PTRY(p, cudaMemcpyAsync(dr, right[i], N, cudaMemcpyHostToDevice, s));
  }
  int st = sgm_batch_pyr_run(p, s);
  if (st) return st;
  for (int i = 0; i < n; ++i) {
    float* dd;
    sgm_batch_pyr_pair_buffers(p, i, nullptr, nullptr, &dd);
    const size_t N = (size_t)p->pairs[i].width * p->pairs[i].height;
    PTRY(p, cudaMemcpyAsync(disp[i], dd, N * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  PTRY(p, cudaStreamSynchronize(s));
  return SGM_OK;
}

int sgm_batch_pyr_info(sgm_batch_pyr_t p, sgm_batch_info_t* info) {
  if (!p || !info) return SGM_ERR_ARG;
  if (!p->ready) return perr(p, SGM_ERR_STATE, "batch not initialised");
  info->pairs = (int32_t)p->pairs.size();
  info->buckets = (int32_t)p->coarse->buckets.size();
  for (auto& L : p->lv) info->buckets += (int32_t)L.buckets.size();
  info->arena_bytes = p->arena_bytes;
  info->kernels_per_run = p->graph_kernels;
  return SGM_OK;
}

}  // extern "C"
