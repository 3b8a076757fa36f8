// Batched kernels: the single-pair device bodies (sgm_kernels.cuh, sgm_kernels3.cuh) applied to a
// table of pairs. Every kernel maps its block or warp item to (pair, item within the pair) with a
// prefix table over the pairs, so one launch covers pairs of different sizes; the scan kernels
// are persistent and take warp items from an atomic queue.
#pragma once
#include "sgm_kernels3.cuh"

namespace sgm {
namespace batch {

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
  // pyramid levels (zero / null in single-level batches)
  float* post;           // LR/median output when a dilation follows (the dilation writes `out`)
  int* label;            // small-region removal: labels and component sizes [H][W]
  int* count;
  int peaks_tiles;       // strip height; strips cover rows [0, peaks_rows)
  int peaks_rows;
  int dil_wth;           // dilation half window
  const int16_t* init;   // initial disparities of a 32-disparity level [H][W]
  sgm::InitParams IP;    // that level's recurrence parameters
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

// Census by tiles of kCensusRows rows (sgm::census4_tile): item = (pair, view, row block), the
// block walks the row block's 512-pixel tiles.
template <typename Word, int CSW, int CSH>
__global__ void __launch_bounds__(128, 4) kb_census4(const BatchPair* __restrict__ pairs, const int* __restrict__ prefix,
                                                  int n) {
  constexpr int RY = sgm::kCensusRows;
  __shared__ uint32_t tile[sgm::census4_tile_words<CSH, RY>()];
  const int item = blockIdx.x;
  const int b = find_pair(prefix, n, item);
  const BatchPair& d = pairs[b];
  const int W = d.P.W, H = d.P.H;
  const int nrb = (H + RY - 1) / RY;
  const int local = item - __ldg(prefix + b);
  const int view = local / nrb;
  const int by = (local - view * nrb) * RY;
  const uint8_t* img = view ? d.img_r : d.img_l;
  Word* out = static_cast<Word*>(view ? d.cs_r : d.cs_l);
  for (int bx = 0; bx < W; bx += 512) sgm::census4_tile<Word, CSW, CSH, RY>(img, out, W, H, view == 1, bx, by, tile);
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

template <int K, int G, int PF, int PASS = 0>
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
    sgm::vpaths3_lane<K, G, PF, PASS>(d.cost, d.lr, d.rl, d.bt, d.wta, d.P, d.Q, view, grp * S + lane / G, lane % G,
                                      colS);
    __syncwarp();
  }
}

// LR check + 3x3 median over tiles of 32 x kLrmRows pixels (one block of 32 x 8 threads, kLrmRows / 8
// pixels per thread): the per-pixel values of sgm::lr_median_tile (a pure function of the
// pixel's neighbourhood), with the tile's loads issued together and the pair lookup made once per
// kLrmRows / 8 tiles of 32 x 8. item = (pair, tile) in row-major tile order.
constexpr int kLrmRows = 32;
template <bool LR, bool MED>
__global__ void __launch_bounds__(256) kb_lr_median(const BatchPair* __restrict__ pairs,
                                                    const int* __restrict__ prefix, int n, float thr) {
  constexpr int TR = kLrmRows + 2, NR = kLrmRows / 8;
  __shared__ float tile[TR][34];
  const int item = blockIdx.x;
  const int b = find_pair(prefix, n, item);
  const BatchPair& d = pairs[b];
  const int local = item - __ldg(prefix + b);
  const int W = d.P.W, H = d.P.H;
  const float* __restrict__ dl = d.wta;
  const float* __restrict__ dr = d.wta + d.Q.dstride;
  float* __restrict__ out = d.post ? d.post : d.out;
  const int tiles_x = (W + 31) / 32;
  const int tyi = local / tiles_x;
  const int bx = (local - tyi * tiles_x) * 32, by = tyi * kLrmRows;
  const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
  for (int k = 0; k < (TR * 34 + 255) / 256; ++k) {
    const int i = k * 256 + ty * 32 + tx;
    if (i < TR * 34) {
      const int ly = i / 34, lx = i - ly * 34;
      const int gx = bx + lx - 1, gy = by + ly - 1;
      float v = sgm::kInvalidFloat;
      if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
        v = dl[(size_t)gy * W + gx];
        if (LR) v = sgm::lr_value(v, gx, dr + (size_t)gy * W, nullptr, W, thr);
      }
      tile[ly][lx] = v;
    }
  }
  __syncthreads();
  const int x = bx + tx;
  if (x >= W) return;
  int ylim = 2 * ((W - 1) / 2);
  ylim = ylim > H - 2 ? H - 2 : ylim;
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const int ry = ty + 8 * r, y = by + ry;
    if (y < H) {
      float v = tile[ry + 1][tx + 1];
      if (MED && x >= 1 && x <= W - 2 && y >= 1 && y <= ylim)
        v = sgm::median9(tile[ry][tx], tile[ry][tx + 1], tile[ry][tx + 2], tile[ry + 1][tx], tile[ry + 1][tx + 1],
                         tile[ry + 1][tx + 2], tile[ry + 2][tx], tile[ry + 2][tx + 1], tile[ry + 2][tx + 2]);
      out[(size_t)y * W + x] = v;
    }
  }
}

// Deterministic noise for the autotuner's timing runs (overwritten by the caller's images).
static __global__ void kb_fill_noise(uint8_t* p, size_t n, uint32_t seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    p[i] = (uint8_t)(h >> 24);
  }
}


// ------------------------------------------------------------------ pyramid levels
// Level images sampled from the full-resolution images (pair order shared by lv and l0); one
// block per level row.
static __global__ void kb_decimate(const BatchPair* __restrict__ lv, const BatchPair* __restrict__ l0,
                                   const int* __restrict__ rprefix, int n, int shift) {
  const int item = blockIdx.x;
  const int b = find_pair(rprefix, n, item);
  const int y = item - __ldg(rprefix + b);
  const int w = lv[b].P.W, W0 = l0[b].P.W;
  uint8_t* dl = const_cast<uint8_t*>(lv[b].img_l);
  uint8_t* dr = const_cast<uint8_t*>(lv[b].img_r);
  const uint8_t* sl = l0[b].img_l;
  const uint8_t* sr = l0[b].img_r;
  for (int x = threadIdx.x; x < w; x += blockDim.x) sgm::decimate_px(sl, sr, dl, dr, W0, w, shift, x, y);
}

// Dilation post -> out, one block per 32x8 tile.
static __global__ void __launch_bounds__(256) kb_dilation(const BatchPair* __restrict__ pairs,
                                                          const int* __restrict__ tprefix, int n) {
  const int item = blockIdx.x;
  const int b = find_pair(tprefix, n, item);
  const BatchPair d = pairs[b];
  const int local = item - __ldg(tprefix + b);
  const int tiles_x = (d.P.W + 31) / 32;
  const int ty = local / tiles_x, tx = local - ty * tiles_x;
  const int x = tx * 32 + threadIdx.x, y = ty * 8 + threadIdx.y;
  if (x < d.P.W && y < d.P.H) sgm::dilation_px<float>(d.post, d.out, d.P.W, d.P.H, d.dil_wth, x, y);
}

// Gauss smoothing post -> out (the pyramid's finest level with do_smooth), one block per tile.
static __global__ void __launch_bounds__(256) kb_gauss(const BatchPair* __restrict__ pairs,
                                                       const int* __restrict__ tprefix, int n) {
  const int item = blockIdx.x;
  const int b = find_pair(tprefix, n, item);
  const BatchPair d = pairs[b];
  const int local = item - __ldg(tprefix + b);
  const int tiles_x = (d.P.W + 31) / 32;
  const int ty = local / tiles_x, tx = local - ty * tiles_x;
  const int x = tx * 32 + threadIdx.x, y = ty * 8 + threadIdx.y;
  if (x < d.P.W && y < d.P.H) sgm::gauss_px(d.post, d.out, d.P.W, d.P.H, 1.5f, 2.0f, x, y);
}

// Small-region removal on `out`: row runs (one warp per row), vertical unions, sizes, filter.
static __global__ void __launch_bounds__(256) kb_cc_rows(const BatchPair* __restrict__ pairs,
                                                         const int* __restrict__ rprefix, int n, int abs_mode) {
  const int item = blockIdx.x * blockDim.y + threadIdx.y;
  if (item >= __ldg(rprefix + n)) return;
  const int b = find_pair(rprefix, n, item);
  const BatchPair d = pairs[b];
  sgm::cc_rows_warp(d.out, d.label, d.count, d.P.W, d.P.H, d.peaks_rows, abs_mode, item - __ldg(rprefix + b));
}

static __global__ void __launch_bounds__(256) kb_cc_vert(const BatchPair* __restrict__ pairs,
                                                         const int* __restrict__ pprefix, int n, int abs_mode) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= __ldg(pprefix + n)) return;
  const int b = find_pair(pprefix, n, i);
  const BatchPair d = pairs[b];
  if (d.peaks_tiles > 1)
    sgm::cc_vert_px(d.out, d.label, d.P.W, d.P.H, d.peaks_tiles, d.peaks_rows, abs_mode, i - __ldg(pprefix + b));
}

static __global__ void __launch_bounds__(256) kb_cc_count(const BatchPair* __restrict__ pairs,
                                                          const int* __restrict__ pprefix, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= __ldg(pprefix + n)) return;
  const int b = find_pair(pprefix, n, i);
  sgm::cc_count_px(pairs[b].label, pairs[b].count, i - __ldg(pprefix + b));
}

static __global__ void __launch_bounds__(256) kb_cc_filter(const BatchPair* __restrict__ pairs,
                                                           const int* __restrict__ pprefix, int n, float ratio) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= __ldg(pprefix + n)) return;
  const int b = find_pair(pprefix, n, i);
  const BatchPair d = pairs[b];
  if (d.peaks_tiles > 0) sgm::cc_filter_px(d.out, d.label, d.count, d.P.W, d.peaks_tiles, ratio, i - __ldg(pprefix + b));
}

// Initial disparities of the finer level `next` from the coarser level's `out`: one warp per
// (pair, row) item of rprefix (blocks of 32 x 8 threads), lanes along the row.
static __global__ void __launch_bounds__(256) kb_init_next(const BatchPair* __restrict__ next,
                                                           const BatchPair* __restrict__ cur,
                                                           const int* __restrict__ rprefix, int n) {
  const int item = blockIdx.x * blockDim.y + threadIdx.y;
  if (item >= __ldg(rprefix + n)) return;
  const int b = find_pair(rprefix, n, item);
  const int y = item - __ldg(rprefix + b);
  const int w = next[b].P.W, h = next[b].P.H;
  const float* src = cur[b].out;
  const long ncur = (long)cur[b].P.W * cur[b].P.H;
  int16_t* dst = const_cast<int16_t*>(next[b].init);
#pragma unroll 4
  for (int x = threadIdx.x; x < w; x += 32) sgm::init_next_px(src, ncur, dst, w, h, x, y);
}

// Cost volume of a 32-disparity level: one block per (pair, view, row); `ids` gives the pair order.
template <typename Word>
__global__ void __launch_bounds__(256) kb_cost3_init(const BatchPair* __restrict__ pairs, const int* __restrict__ ids,
                                                     const int* __restrict__ rprefix, int n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int item = blockIdx.x;
  const int b = find_pair(rprefix, n, item);
  const BatchPair d = pairs[__ldg(ids + b)];
  const int local = item - __ldg(rprefix + b);
  const int view = local / d.P.H;
  sgm::cost3_init_row<Word>(static_cast<const Word*>(d.cs_l), static_cast<const Word*>(d.cs_r), d.init, d.init, d.cost,
                            d.IP, local - view * d.P.H, view, reinterpret_cast<Word*>(smem_raw));
}

// Shared-memory set-up of the 32-disparity scan kernels (penalties are the same for every pair
// of a level): the P2' table and the padding of every scanline row.
template <int G>
__device__ __forceinline__ void init_scan_smem(uint32_t* p2tab, uint32_t* rows, const sgm::InitParams& P) {
  sgm::fill_p2_table(p2tab, P, threadIdx.x, blockDim.x);
  sgm::init_row_pad<G>(rows + threadIdx.x / G, P.p1, true, threadIdx.x % G);
  __syncthreads();
}

// Persistent scans of 32-disparity levels, 128-thread blocks; items of 32/G scanlines / columns.
// With two lanes per scanline the registers are held to five blocks per SM (96 each, no spill):
// 1-2 % more pairs/s than four blocks at 64-256 pyramids per batch.
template <int G, int PF>
__global__ void __launch_bounds__(128, G == 2 ? 5 : 1)
    kb_rows3_init(const BatchPair* __restrict__ pairs, const int* __restrict__ ids, const int* __restrict__ prefix,
                  int n, int* __restrict__ queue) {
  constexpr int S = 32 / G;
  __shared__ uint32_t p2tab[sgm::kP2Tab];
  __shared__ uint32_t rows[sgm::init_rs<G>() * sgm::kIRow];
  init_scan_smem<G>(p2tab, rows, pairs[__ldg(ids)].IP);
  uint32_t* row = rows + threadIdx.x / G;
  const int lane = threadIdx.x & 31;
  const int total = __ldg(prefix + n);
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(queue, 1);
    item = __shfl_sync(sgm::kFull, item, 0);
    if (item >= total) break;
    const int b = find_pair(prefix, n, item);
    const BatchPair d = pairs[__ldg(ids + b)];
    const int local = item - __ldg(prefix + b);
    sgm::hpaths3_init_lane<G, PF>(d.cost, d.init, d.init, d.lr, d.rl, d.IP, d.nv, local * S + lane / G, lane % G, row,
                                  p2tab);
  }
}

template <int G, int PF, int PASS = 0>
__global__ void __launch_bounds__(128, G == 2 ? 5 : 1)
    kb_cols3_init(const BatchPair* __restrict__ pairs, const int* __restrict__ ids, const int* __restrict__ prefix,
                  int n, int* __restrict__ queue) {
  constexpr int S = 32 / G;
  __shared__ uint32_t p2tab[sgm::kP2Tab];
  __shared__ uint32_t rows[sgm::init_rs<G>() * sgm::kIRow];
  __shared__ uint32_t sums[sgm::init_rs<G>() * (sgm::kLevelRange / 2)];
  init_scan_smem<G>(p2tab, rows, pairs[__ldg(ids)].IP);
  uint32_t* row = rows + threadIdx.x / G;
  uint32_t* colS = sums + threadIdx.x / G;
  const int lane = threadIdx.x & 31;
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
    sgm::vpaths3_init_lane<G, PF, PASS>(d.cost, d.lr, d.rl, d.init, d.init, d.bt, d.wta, d.IP, d.Q, view,
                                        grp * S + lane / G, lane % G, row, colS, p2tab);
    __syncwarp();
  }
}

}  // namespace batch
}  // namespace sgm
