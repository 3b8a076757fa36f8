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
#include "sgm_kernels3.cuh"

void sgm_set_process_error(const char* msg);

namespace {

struct BatchPair {
  const uint8_t* img_l;
  const uint8_t* img_r;
  void* cs_l;
  void* cs_r;
  uint8_t* cost;
  uint8_t* lr;
  uint8_t* rl;
  uint8_t* bt;
  float* wta;  // [2][H][W]
  float* out;  // [H][W]
  sgm::PlainParams P;
  sgm::WtaParams Q;
  int nv;  // views (2 with the LR check)
};

// Largest b in [0, n) with prefix[b] <= item (prefix ascending, prefix[0] = 0).
__device__ __forceinline__ int find_pair(const int* __restrict__ prefix, int n, int item) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(prefix + mid) <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <typename Word, int CSW, int CSH>
__global__ void __launch_bounds__(256) kb_census(const BatchPair* __restrict__ pairs, const int* __restrict__ prefix,
                                                 int n) {
  const int item = blockIdx.x * blockDim.y + threadIdx.y;
  if (item >= __ldg(prefix + n)) return;
  const int b = find_pair(prefix, n, item);
  const BatchPair d = pairs[b];
  const int W = d.P.W, H = d.P.H;
  const int local = item - __ldg(prefix + b);
  const int view = local / H;
  const int y = local - view * H;
  const uint8_t* img = view ? d.img_r : d.img_l;
  Word* out = static_cast<Word*>(view ? d.cs_r : d.cs_l) + (size_t)y * W;
  for (int x = threadIdx.x; x < W; x += 32) out[x] = sgm::census_value<Word, CSW, CSH>(img, x, y, W, H, view == 1);
}

template <int K, typename Word>
__global__ void __launch_bounds__(256) kb_rows(const BatchPair* __restrict__ pairs, const int* __restrict__ ids,
                                               const int* __restrict__ prefix, int n, int* __restrict__ queue) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* base = smem_raw + (size_t)threadIdx.y * sgm::hpaths2_warp_smem<K, Word>();
  const int total = __ldg(prefix + n);
  for (;;) {
    int item = 0;
    if (threadIdx.x == 0) item = atomicAdd(queue, 1);
    item = __shfl_sync(sgm::kFull, item, 0);
    if (item >= total) break;
    const int b = find_pair(prefix, n, item);
    const BatchPair d = pairs[__ldg(ids + b)];
    const int local = item - __ldg(prefix + b);
    const int per_view = 2 * d.P.H;
    const int view = local / per_view;
    const int rem = local - view * per_view;
    sgm::hpaths2_warp<K, Word>(static_cast<const Word*>(d.cs_l), static_cast<const Word*>(d.cs_r), d.cost, d.lr,
                               d.rl, d.P, view, rem >> 1, rem & 1, base);
  }
}

template <int K, int PF>
__global__ void __launch_bounds__(256) kb_cols(const BatchPair* __restrict__ pairs, const int* __restrict__ ids,
                                               const int* __restrict__ prefix, int n, int* __restrict__ queue) {
  const int total = __ldg(prefix + n);
  for (;;) {
    int item = 0;
    if (threadIdx.x == 0) item = atomicAdd(queue, 1);
    item = __shfl_sync(sgm::kFull, item, 0);
    if (item >= total) break;
    const int b = find_pair(prefix, n, item);
    const BatchPair d = pairs[__ldg(ids + b)];
    const int local = item - __ldg(prefix + b);
    const int view = local / d.P.W;
    const int x = local - view * d.P.W;
    if constexpr (PF == 0)
      sgm::vpaths1_warp<K>(d.cost, d.lr, d.rl, d.bt, d.wta, d.P, d.Q, view, x);
    else
      sgm::vpaths2_warp<K, PF>(d.cost, d.lr, d.rl, d.bt, d.wta, d.P, d.Q, view, x, nullptr);
  }
}

template <int K, typename Word>
__global__ void __launch_bounds__(128) kb_cost3(const BatchPair* __restrict__ pairs, const int* __restrict__ ids,
                                                const int* __restrict__ prefix, int n) {
  __shared__ Word win[128 + 32 * K];
  const int item = blockIdx.x;
  const int b = find_pair(prefix, n, item);
  const BatchPair d = pairs[__ldg(ids + b)];
  const int local = item - __ldg(prefix + b);
  const int segs = (d.P.W + 127) / 128;
  const int row = local / segs;  // view * H + y
  const int seg = local - row * segs;
  const int view = row / d.P.H;
  sgm::cost3_block<K, Word>(static_cast<const Word*>(d.cs_l), static_cast<const Word*>(d.cs_r), d.cost, d.P, view,
                            row - view * d.P.H, seg * 128, win);
}

// Items of 32/G scanlines (pair, first scanline); lanes beyond the pair's scanlines idle.
template <int K, int G, int PF>
__global__ void __launch_bounds__(256) kb_rows3(const BatchPair* __restrict__ pairs, const int* __restrict__ ids,
                                                const int* __restrict__ prefix, int n, int* __restrict__ queue) {
  constexpr int S = 32 / G;
  const int lane = threadIdx.x;
  const int total = __ldg(prefix + n);
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(queue, 1);
    item = __shfl_sync(sgm::kFull, item, 0);
    if (item >= total) break;
    const int b = find_pair(prefix, n, item);
    const BatchPair d = pairs[__ldg(ids + b)];
    const int local = item - __ldg(prefix + b);
    sgm::hpaths3_lane<K, G, PF>(d.cost, d.lr, d.rl, d.P, d.nv, local * S + lane / G, lane % G);
  }
}

template <int K, int G, int PF>
__global__ void __launch_bounds__(256) kb_cols3(const BatchPair* __restrict__ pairs, const int* __restrict__ ids,
                                                const int* __restrict__ prefix, int n, int* __restrict__ queue) {
  constexpr int S = 32 / G;
  extern __shared__ uint32_t s_sum[];
  const int lane = threadIdx.x;
  uint32_t* colS = s_sum + ((size_t)threadIdx.y * S + lane / G) * (16 * K + 1);
  const int total = __ldg(prefix + n);
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(queue, 1);
    item = __shfl_sync(sgm::kFull, item, 0);
    if (item >= total) break;
    const int b = find_pair(prefix, n, item);
    const BatchPair d = pairs[__ldg(ids + b)];
    const int local = item - __ldg(prefix + b);
    const int per_view = (d.P.W + S - 1) / S;
    const int view = local / per_view;
    const int grp = local - view * per_view;
    sgm::vpaths3_lane<K, G, PF>(d.cost, d.lr, d.rl, d.bt, d.wta, d.P, d.Q, view, grp * S + lane / G, lane % G, colS);
    __syncwarp();
  }
}

template <bool LR, bool MED>
__global__ void __launch_bounds__(256) kb_lr_median(const BatchPair* __restrict__ pairs,
                                                    const int* __restrict__ prefix, int n, float thr) {
  __shared__ float tile[10][34];
  const int item = blockIdx.x;
  const int b = find_pair(prefix, n, item);
  const BatchPair d = pairs[b];
  const int local = item - __ldg(prefix + b);
  const int tiles_x = (d.P.W + 31) / 32;
  const int ty = local / tiles_x;
  const int tx = local - ty * tiles_x;
  sgm::lr_median_tile<LR, MED>(d.wta, d.wta + d.Q.dstride, nullptr, d.out, d.P.W, d.P.H, thr, tx * 32, ty * 8, tile);
}

// Deterministic noise for the autotuner's timing runs (overwritten by the caller's images).
__global__ void kb_fill_noise(uint8_t* p, size_t n, uint32_t seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    p[i] = (uint8_t)(h >> 24);
  }
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

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
  int census_prefix = 0, tile_prefix = 0;  // offsets into dtab
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
    if (arena) cudaFree(arena);
    if (ddesc) cudaFree(ddesc);
    if (dtab) cudaFree(dtab);
    if (queues) cudaFree(queues);
    arena = nullptr;
    ddesc = nullptr;
    dtab = nullptr;
    queues = nullptr;
    for (auto s : side) cudaStreamDestroy(s);
    side.clear();
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

template <int K>
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
    st = G == 4 ? go(kb_cols3<K, 4, pf_cols<K, 4>()>) : go(kb_cols3<K, 2, pf_cols<K, 2>()>);
  } else {
    st = G == 1 ? go(kb_cols3<K, 1, pf_cols<K, 1>()>) : G == 2 ? go(kb_cols3<K, 2, pf_cols<K, 2>()>)
       : G == 4 ? go(kb_cols3<K, 4, pf_cols<K, 4>()>) : go(kb_cols3<K, 8, pf_cols<K, 8>()>);
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

int cols(sgm_batch* b, sgm_batch::Bucket& k, cudaStream_t s, int* queue, bool prepare) {
  switch (k.K) {
    case 1: return cols_t<1>(b, k, s, queue, prepare);
    case 2: return cols_t<2>(b, k, s, queue, prepare);
    default: return cols_t<4>(b, k, s, queue, prepare);
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
int prepare_bucket(sgm_batch* b, sgm_batch::Bucket& k) {
  const int st = rows(b, k, nullptr, nullptr, true);
  return st ? st : cols(b, k, nullptr, nullptr, true);
}

int launch_census(sgm_batch* b, cudaStream_t s) {
  const int blocks = (b->census_items + 7) / 8;
  const int n = (int)b->pairs.size();
  if (b->word == 8)
    kb_census<uint64_t, 4, 3><<<blocks, dim3(32, 8), 0, s>>>(b->ddesc, b->dtab + b->census_prefix, n);
  else
    kb_census<uint32_t, 2, 2><<<blocks, dim3(32, 8), 0, s>>>(b->ddesc, b->dtab + b->census_prefix, n);
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
    int* q = b->queues + 2 * i;
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
    st = launch_rows(b, b->buckets[i], t, b->queues + 2 * i);
    if (!st) st = launch_cols(b, b->buckets[i], t, b->queues + 2 * i + 1);
    kernels += b->buckets[i].tune.rows_lanes ? 3 : 2;
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

int sgm_batch_init(sgm_batch_t b, const sgm_batch_pair_t* pairs, int32_t count, const sgm_option_t* option,
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
  BTRY(b, cudaMalloc(&b->arena, total));
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
    d.nv = nv;
  }
  BTRY(b, cudaMalloc(&b->ddesc, sizeof(BatchPair) * count));
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
  auto cp = prefix_of(all, [&](int i) { return 2 * pairs[i].height; });
  b->census_prefix = cp.first; b->census_items = cp.second;
  auto tp = prefix_of(all, [&](int i) { return ((pairs[i].width + 31) / 32) * ((pairs[i].height + 7) / 8); });
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
  BTRY(b, cudaMalloc(&b->dtab, tab.size() * sizeof(int)));
  BTRY(b, cudaMemcpy(b->dtab, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice));
  b->nqueues = 2 * (int)b->buckets.size();
  BTRY(b, cudaMalloc(&b->queues, b->nqueues * sizeof(int)));
  for (size_t i = 0; i < b->buckets.size(); ++i) {
    cudaStream_t t;
    BTRY(b, cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
    b->side.push_back(t);
  }
  for (size_t i = 0; i < b->buckets.size() + 1; ++i) {
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
