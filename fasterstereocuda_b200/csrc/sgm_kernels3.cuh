// SGM kernels with one thread per scanline (sm_100a).
//
// A thread owns one path (a row in one direction, or a column) and keeps all D path costs of
// its current pixel in registers, two disparities per 32-bit word (u16x2: L(2k) in the low
// half, L(2k+1) in the high half). One recurrence step is then, per word,
//   x = min3(L(d-1), L(d+1), m + P2 - P1)      __vimin3_u16x2
//   t = min(x + P1, L(d))                      __viaddmin_u16x2
//   L'(d) = t + C(d) - m                       one 3-input add
// with the d-1 / d+1 words formed by byte permutes inside the thread: no shuffles, no warp
// reductions, and the minimum over d is a tree of SIMD minima. A scanline may also be split over
// G = 2, 4 or 8 neighbouring lanes (each holding D/G disparities; two shuffles carry the
// boundary words and a butterfly the minimum), trading instructions for parallelism. The WTA
// runs in the scanline's threads (keys S << 6 | d, sums kept in shared memory). Neighbouring
// scanlines sit in neighbouring lanes, so the column kernel's loads of one row are contiguous.
//
// Exactness: the reference's recurrence is uint32; here every value is held in 16 bits, which
// is exact while L <= 255 + P2 and m + P2 < 65536, i.e. for P1, P2 <= 16383 (checked on the
// host), and the min(x + P1, ...) form needs P2 >= P1 (host falls back otherwise).
// Results equal k_hpaths_plain / k_vpaths_wta_plain (reference kernels cited there).
#pragma once
#include "sgm_kernels.cuh"

namespace sgm {

constexpr uint32_t kMaxPenalty16 = 16383;

__device__ __forceinline__ uint32_t rep16(uint32_t v) { return v * 0x10001u; }
__device__ __forceinline__ uint32_t min16x2(uint32_t a, uint32_t b) { return __vimin3_u16x2(a, b, b); }
__device__ __forceinline__ uint32_t hmin16(uint32_t w) { return min(w & 0xFFFFu, w >> 16); }

// Bytes (b0 b1 b2 b3) of v -> u16x2 words (b0, b1) and (b2, b3).
__device__ __forceinline__ uint32_t widen_lo(uint32_t v) { return __byte_perm(v, 0u, 0x4140); }
__device__ __forceinline__ uint32_t widen_hi(uint32_t v) { return __byte_perm(v, 0u, 0x4342); }
// Low bytes of the four halves of (w0, w1) -> one 32-bit word of u8 path costs.
__device__ __forceinline__ uint32_t narrow(uint32_t w0, uint32_t w1) { return __byte_perm(w0, w1, 0x6420); }

// Raw per-thread slices: NR 32-bit words (4*NR bytes, 4-, 8- or 16*n-byte aligned).
template <int NR>
__device__ __forceinline__ void ld_slice(const uint8_t* __restrict__ p, uint32_t (&r)[NR]) {
  if constexpr (NR == 1) {
    r[0] = __ldcg(reinterpret_cast<const unsigned int*>(p));
  } else if constexpr (NR == 2) {
    const uint2 q = __ldcg(reinterpret_cast<const uint2*>(p));
    r[0] = q.x; r[1] = q.y;
  } else {
#pragma unroll
    for (int v = 0; v < NR / 4; ++v) {
      const uint4 q = __ldcg(reinterpret_cast<const uint4*>(p) + v);
      r[4 * v] = q.x; r[4 * v + 1] = q.y; r[4 * v + 2] = q.z; r[4 * v + 3] = q.w;
    }
  }
}

template <int NR>
__device__ __forceinline__ void st_slice(uint8_t* __restrict__ p, const uint32_t (&r)[NR]) {
  if constexpr (NR == 1) {
    *reinterpret_cast<uint32_t*>(p) = r[0];
  } else if constexpr (NR == 2) {
    *reinterpret_cast<uint2*>(p) = make_uint2(r[0], r[1]);
  } else {
#pragma unroll
    for (int v = 0; v < NR / 4; ++v)
      reinterpret_cast<uint4*>(p)[v] = make_uint4(r[4 * v], r[4 * v + 1], r[4 * v + 2], r[4 * v + 3]);
  }
}

// Bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned, inside one allocation) into L2.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// A row scan reads one short slice per row and step, so its loads of one DRAM page are spread
// over many steps. Every 16 steps the scanline's first lane prefetches the row's next 16 pixels
// (steps s0 + 8 .. s0 + 23, clamped to the scanline) into L2 in one request.
// With many pairs in flight: +3.5 % pyramid, +7.5 % plain pairs/s (a single pair's scans alone
// run ~10 % faster without it).
template <int BYTES_PER_PX>
__device__ __forceinline__ void prefetch_row_ahead(const uint8_t* row, int xs, int dx, int s0, int len, int g) {
  if (g == 0 && (s0 & 15) == 0) {
    const int a = s0 + 8, n = min(16, len - a);
    if (n > 0) {
      const int x_lo = dx > 0 ? xs + a : xs - a - (n - 1);
      prefetch_l2(row + (size_t)x_lo * BYTES_PER_PX, (uint32_t)(n * BYTES_PER_PX));
    }
  }
}

// bytes -> u16x2 words (NT = 2*NR) and back (low bytes)
template <int NR>
__device__ __forceinline__ void widen_slice(const uint32_t (&r)[NR], uint32_t (&w)[2 * NR]) {
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    w[2 * i] = widen_lo(r[i]);
    w[2 * i + 1] = widen_hi(r[i]);
  }
}
template <int NR>
__device__ __forceinline__ void narrow_slice(const uint32_t (&w)[2 * NR], uint32_t (&r)[NR]) {
#pragma unroll
  for (int i = 0; i < NR; ++i) r[i] = narrow(w[2 * i], w[2 * i + 1]);
}

// Minimum over the u16x2 words (a log-depth tree), then over the G threads of the scanline.
template <int NT, int G>
__device__ __forceinline__ uint32_t group_min16(const uint32_t (&v)[NT]) {
  uint32_t t[NT];
#pragma unroll
  for (int k = 0; k < NT; ++k) t[k] = v[k];
  // ternary tree of 3-input SIMD minima
#pragma unroll
  for (int st = 1; st < NT; st *= 3) {
#pragma unroll
    for (int k = 0; k + st < NT; k += 3 * st)
      t[k] = k + 2 * st < NT ? __vimin3_u16x2(t[k], t[k + st], t[k + 2 * st]) : min16x2(t[k], t[k + st]);
  }
  uint32_t r = hmin16(t[0]);
#pragma unroll
  for (int o = 1; o < G; o *= 2) r = min(r, __shfl_xor_sync(kFull, r, o, G));
  return r;
}

template <int G>
__device__ __forceinline__ uint32_t group_min(uint32_t r) {
#pragma unroll
  for (int o = 1; o < G; o *= 2) r = min(r, __shfl_xor_sync(kFull, r, o, G));
  return r;
}

// First pixel of a path: L = C. Returns m = min_d C(d) over the scanline's G threads.
template <int NT, int G>
__device__ __forceinline__ uint32_t first_g(uint32_t (&L)[NT], const uint32_t (&c)[NT]) {
#pragma unroll
  for (int k = 0; k < NT; ++k) L[k] = c[k];
  return group_min16<NT, G>(c);
}

// One recurrence step of a scanline held by G threads (thread g owns words g*NT .. g*NT+NT-1);
// returns the new minimum. p1x2 = rep16(P1), p2m1 = P2 - P1. Every lane of the warp calls it.
template <int NT, int G>
__device__ __forceinline__ uint32_t step_g(uint32_t (&L)[NT], const uint32_t (&c)[NT], uint32_t m, uint32_t p1x2,
                                          uint32_t p2m1, int g) {
  uint32_t left_nb = 0, right_nb = 0;
  if constexpr (G > 1) {
    left_nb = __shfl_up_sync(kFull, L[NT - 1], 1, G);
    right_nb = __shfl_down_sync(kFull, L[0], 1, G);
  }
  const bool first = g == 0, last = g == G - 1;
  const uint32_t l4 = rep16(m + p2m1);
  const uint32_t mm = rep16(m);
  uint32_t nl[NT];
#pragma unroll
  for (int k = 0; k < NT; ++k) {
    uint32_t lw, rw;
    if (k > 0) lw = __byte_perm(L[k - 1], L[k], 0x5432);
    else lw = first ? ((L[0] << 16) | 0xFFFFu) : __byte_perm(left_nb, L[0], 0x5432);
    if (k < NT - 1) rw = __byte_perm(L[k], L[k + 1], 0x5432);
    else rw = last ? ((L[k] >> 16) | 0xFFFF0000u) : __byte_perm(L[k], right_nb, 0x5432);
    const uint32_t x = __vimin3_u16x2(lw, rw, l4);
    uint32_t t = __viaddmin_u16x2(x, p1x2, L[k]);
    if (k == 0 && first) t = min16x2(t, 0xFFFF0000u | kInvalidCost);            // d = 0: left candidate 127
    if (k == NT - 1 && last) t = min16x2(t, (kInvalidCost << 16) | 0xFFFFu);    // d = D-1: right candidate 127
    nl[k] = t + c[k] - mm;
  }
#pragma unroll
  for (int k = 0; k < NT; ++k) L[k] = nl[k];
  return group_min16<NT, G>(nl);
}

// ---------------------------------------------------------------------------------------------
// Cost volume of both views (reference Kernel_CostCompute cusgm_cc.cu:118-172 / 238-293):
// view 0: C(x,d) = popc(cl[x] ^ cr[x-min_d-d]), view 1: C(x,d) = popc(cr[x] ^ cl[x+min_d+d]),
// an out-of-range partner index reads element 0 of the partner row; with 5x5 census the last
// pixel of every D-pixel block of view 1 keeps its view-0 cost (cusgm_cc.cu:288).
// One thread per pixel, 128 pixels of one row per CTA, partner words staged in shared memory.
// Columns x < max(0, min_d) are not written (no path reads them).
// ---------------------------------------------------------------------------------------------
// 128 pixels [bx, bx + 128) of row y, view `view`, by a 128-thread block (every thread calls it).
// D costs of one pixel: popc(a ^ wp[STEP * d]) packed four per word, 16-byte stores.
template <int D, typename Word, int STEP>
__device__ __forceinline__ void cost3_px(const Word a, const Word* wp, uint8_t* __restrict__ out) {
#pragma unroll
  for (int v = 0; v < D / 16; ++v) {
    uint32_t q[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      uint32_t c[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) c[b] = popc_word((Word)(a ^ wp[STEP * (16 * v + 4 * j + b)]));
      q[j] = __byte_perm(__byte_perm(c[0], c[1], 0x0040u), __byte_perm(c[2], c[3], 0x0040u), 0x5410u);
    }
    reinterpret_cast<uint4*>(out)[v] = make_uint4(q[0], q[1], q[2], q[3]);
  }
}

template <int K, typename Word>
__device__ __forceinline__ void cost3_block(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                            uint8_t* __restrict__ cost, const PlainParams& P, int view, int y, int bx,
                                            Word* win) {
  constexpr int D = 32 * K;
  const int W = P.W;
  const Word* own = (view == 0 ? cs_l : cs_r) + (size_t)y * W;
  const Word* oth = (view == 0 ? cs_r : cs_l) + (size_t)y * W;
  const Word oth0 = oth[0];
  // view 0: window index i <-> partner position bx - min_d - (D-1) + i;
  // view 1: i <-> bx + min_d + i
  const int ws = view == 0 ? bx - P.min_d - (D - 1) : bx + P.min_d;
  for (int i = threadIdx.x; i < 128 + D - 1; i += 128) {
    const int pos = ws + i;
    win[i] = (pos >= 0 && pos < W) ? oth[pos] : oth0;
  }
  __syncthreads();
  const int x = bx + threadIdx.x;
  if (x >= W || x < P.x0) return;
  const Word a = own[x];
  bool lr_cost = false;
  if (view == 1 && sizeof(Word) == 4) {
    const int blk = P.x0 + ((x - P.x0) / D) * D;
    lr_cost = (x == blk + min(D, W - blk) - 1);
  }
  uint8_t* out = cost + (size_t)view * P.vstride + ((size_t)y * W + x) * D;
  if (!lr_cost) {
    // partner of disparity d: view 0 at win[t + D-1 - d], view 1 at win[t + d] (immediate offsets)
    if (view == 0) cost3_px<D, Word, -1>(a, win + threadIdx.x + (D - 1), out);
    else cost3_px<D, Word, 1>(a, win + threadIdx.x, out);
  } else {  // 5x5 right view: this pixel keeps its left-to-right cost
    const Word* g_own = cs_r + (size_t)y * W;
    const Word own0 = g_own[0];
    const Word l = cs_l[(size_t)y * W + x];
    for (int v = 0; v < D / 16; ++v) {
      uint32_t q[4];
      for (int j = 0; j < 4; ++j) {
        uint32_t packed = 0;
        for (int b = 0; b < 4; ++b) {
          const int d = 16 * v + 4 * j + b;
          const int pos = x - P.min_d - d;
          const Word p = (pos >= 0 && pos < W) ? g_own[pos] : own0;
          packed |= popc_word((Word)(l ^ p)) << (8 * b);
        }
        q[j] = packed;
      }
      reinterpret_cast<uint4*>(out)[v] = make_uint4(q[0], q[1], q[2], q[3]);
    }
  }
}

template <int K, typename Word>
__global__ void __launch_bounds__(128) k_cost3(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                               uint8_t* __restrict__ cost, PlainParams P) {
  __shared__ Word win[128 + 32 * K];
  cost3_block<K, Word>(cs_l, cs_r, cost, P, blockIdx.z, blockIdx.y, blockIdx.x * 128, win);
}

// ---------------------------------------------------------------------------------------------
// Regions of interest (StereoCuda::Match with StereoROI_T). A view's region -- columns
// [rx0, rx0 + rw), rows [ry0, ry0 + rh) -- is matched as a sub-image of its own: its cost is
// stored compactly as [rh][rw][D] and the scan kernels run on that sub-volume, so every path
// starts at the region's edge as the reference's ROI scans do (xoffset / xEnd / yoffset / yend,
// cusgm_ca.cu:1478-1598 launched at :3991-3999).
// ---------------------------------------------------------------------------------------------
// Costs of 128 region pixels of one row (partners from the whole image, as in the full volume:
// cusgm_cc.cu:118-172 / 238-293 with the ROI offsets of :478-488). 5x5 census, view 1: the last
// pixel of every D-pixel block counted from the ROI's x (bx) is not written by the reference's
// right-view kernel, so it keeps the left view's cost there (cusgm_cc.cu:288).
template <int K, typename Word>
__global__ void __launch_bounds__(128) k_cost_roi(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                                  uint8_t* __restrict__ cost, PlainParams P, int view, int rx0,
                                                  int ry0, int rw, int bx) {
  constexpr int D = 32 * K;
  __shared__ Word win[128 + D];
  const int W = P.W;
  const int y = ry0 + blockIdx.y;
  const int xb = rx0 + blockIdx.x * 128;
  const Word* own = (view == 0 ? cs_l : cs_r) + (size_t)y * W;
  const Word* oth = (view == 0 ? cs_r : cs_l) + (size_t)y * W;
  const Word oth0 = oth[0];
  const int ws = view == 0 ? xb - P.min_d - (D - 1) : xb + P.min_d;
  for (int i = threadIdx.x; i < 128 + D - 1; i += 128) {
    const int pos = ws + i;
    win[i] = (pos >= 0 && pos < W) ? oth[pos] : oth0;
  }
  __syncthreads();
  const int xr = blockIdx.x * 128 + threadIdx.x;  // column inside the region
  if (xr >= rw) return;
  const int x = rx0 + xr;
  uint8_t* out = cost + ((size_t)blockIdx.y * rw + xr) * D;
  bool lr_cost = false;
  if (view == 1 && sizeof(Word) == 4) {
    const int blk = bx + ((x - bx) / D) * D;
    lr_cost = (x == blk + min(D, W - blk) - 1);
  }
  if (!lr_cost) {
    if (view == 0) cost3_px<D, Word, -1>(own[x], win + threadIdx.x + (D - 1), out);
    else cost3_px<D, Word, 1>(own[x], win + threadIdx.x, out);
  } else {  // the left view's cost of this pixel
    const Word* g_r = cs_r + (size_t)y * W;
    const Word r0 = g_r[0];
    const Word l = cs_l[(size_t)y * W + x];
    for (int v = 0; v < D / 16; ++v) {
      uint32_t q[4];
      for (int j = 0; j < 4; ++j) {
        uint32_t packed = 0;
        for (int b = 0; b < 4; ++b) {
          const int pos = x - P.min_d - (16 * v + 4 * j + b);
          packed |= popc_word((Word)(l ^ ((pos >= 0 && pos < W) ? g_r[pos] : r0))) << (8 * b);
        }
        q[j] = packed;
      }
      reinterpret_cast<uint4*>(out)[v] = make_uint4(q[0], q[1], q[2], q[3]);
    }
  }
}

// Full disparity map of a view from its region's map: the region's values, INVALID elsewhere.
static __global__ void k_roi_scatter(const float* __restrict__ region, float* __restrict__ full, int W, int H,
                                     int rx0, int ry0, int rw, int rh) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const int xr = x - rx0, yr = y - ry0;
  const bool in = xr >= 0 && xr < rw && yr >= 0 && yr < rh;
  full[(size_t)y * W + x] = in ? region[(size_t)yr * rw + xr] : kInvalidFloat;
}

// ---------------------------------------------------------------------------------------------
// Horizontal paths, G threads per scanline (view, direction, row): scanline index i -> group
// i / H (view = group >> 1, dir = group & 1), y = i % H. Reads the cost volume, writes the
// left-to-right (dir 0) or right-to-left (dir 1) path volume; the cost of step s + PF is loaded
// at step s. Same results as the lane-per-disparity row kernels (reference
// Kernel_Aggregate_Horizontal_Warpfor*, cusgm_ca.cu:1343-1770).
// ---------------------------------------------------------------------------------------------
// Scanline i (lane g of its G lanes); every lane of the warp calls it with the same trip count.
// i >= nviews*2*H: the lane follows the last scanline without storing (the shuffles need it).
template <int K, int G, int PF>
__device__ __forceinline__ void hpaths3_lane(const uint8_t* __restrict__ cost, uint8_t* __restrict__ lr,
                                             uint8_t* __restrict__ rl, const PlainParams& P, int nviews, int i,
                                             int g) {
  constexpr int D = 32 * K, NT = D / 2 / G, NR = NT / 2, SB = D / G;  // SB: bytes per thread slice
  const int H = P.H, W = P.W;
  const int nscan = nviews * 2 * H;
  const bool valid = i < nscan;
  if (!valid) i = nscan - 1;
  const int grp = i / H;
  const int y = i - grp * H;
  const int view = grp >> 1, dir = grp & 1;
  const int x0 = P.x0;
  const int len = W - x0;
  if (len <= 0) return;  // uniform over the grid
  const size_t vo = (size_t)view * P.vstride + (size_t)y * W * D + (size_t)g * SB;
  const uint8_t* crow = cost + vo;
  uint8_t* orow = (dir == 0 ? lr : rl) + vo;
  const uint32_t p1x2 = rep16(P.p1), p2m1 = P.p2 - P.p1;
  const int xs = dir == 0 ? x0 : W - 1;
  const int dx = dir == 0 ? 1 : -1;
  uint32_t L[NT], c[NT], out[NR];
  uint32_t ring[PF][NR];
#pragma unroll
  for (int j = 0; j < PF; ++j)
    if (j < len) ld_slice<NR>(crow + (size_t)(xs + j * dx) * D, ring[j]);
  uint32_t m = 0;
  static_assert(16 % PF == 0, "blocks of PF steps start every 16 steps");
  for (int s0 = 0; s0 < len; s0 += PF) {
    prefetch_row_ahead<D>(crow - (size_t)g * SB, xs, dx, s0, len, g);
#pragma unroll
    for (int j = 0; j < PF; ++j) {
      const int s = s0 + j;
      if (s < len) {
        const int x = xs + s * dx;
        widen_slice<NR>(ring[j], c);
        if (s + PF < len) ld_slice<NR>(crow + (size_t)(x + PF * dx) * D, ring[j]);
        m = s == 0 ? first_g<NT, G>(L, c) : step_g<NT, G>(L, c, m, p1x2, p2m1, g);
        narrow_slice<NR>(L, out);
        if (valid) st_slice<NR>(orow + (size_t)x * D, out);
      }
    }
  }
}

template <int K, int G, int PF>
// five CTAs per SM (at most 96 registers) where a lane holds at most 32 disparities and G >= 2:
// many concurrent pairs are occupancy-bound (plain 1242x375x64: +5 % pairs/s over the
// unconstrained 113-128 registers); wider slices would spill
__global__ void __launch_bounds__(128, (G >= 2 && 32 * K / G <= 32) ? 5 : 1)
    k_hpaths3(const uint8_t* __restrict__ cost, uint8_t* __restrict__ lr,
                                                 uint8_t* __restrict__ rl, PlainParams P, int nviews) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  hpaths3_lane<K, G, PF>(cost, lr, rl, P, nviews, t / G, threadIdx.x % G);
}

// ---------------------------------------------------------------------------------------------
// Vertical paths + 4-path sum + WTA, G threads per column: a bottom-to-top pass storing its path
// costs, then top-to-bottom summing the four u8 path costs and selecting the disparity inside
// the column's threads. Same results as k_vpaths_wta_plain (reference
// Kernel_Aggregate_Vertical_Warpfor*, cusgm_ca.cu:1410-1888, WTA cusgm_ca.cu:3514-3809).
// Shared memory: D/2 + 1 words per column (the sums, read back for S(d*-1), S(d*+1) and the
// reference tie rule), i.e. vpaths3_col_smem<K>() bytes per column.
// ---------------------------------------------------------------------------------------------
template <int K>
__host__ __device__ constexpr size_t vpaths3_col_smem() { return (size_t)(16 * K + 1) * 4; }

// Column xc of view `view` (lane g of its G lanes); colS: this column's D/2 + 1 words of shared
// memory. Every lane of the warp calls it (same H); xc >= W: the lane follows column W-1 without
// storing.
// PASS: 0 both passes, 1 the bottom-to-top pass only, 2 the top-to-bottom pass only (reads the
// stored bottom-to-top volume), so that the two can be launched around the row scans.
template <int K, int G, int PF, int PASS = 0>
__device__ __forceinline__ void vpaths3_lane(const uint8_t* __restrict__ cost, const uint8_t* __restrict__ lr,
                                             const uint8_t* __restrict__ rl, uint8_t* __restrict__ bt,
                                             float* __restrict__ disp, const PlainParams& P, const WtaParams& Q,
                                             int view, int xc, int g, uint32_t* colS) {
  constexpr int D = 32 * K, NW = D / 2, NT = NW / G, NR = NT / 2, SB = D / G;
  uint32_t* myS = colS + g * NT;
  const int W = P.W, H = P.H;
  const bool valid = xc < W;
  const int x = valid ? xc : W - 1;            // idle lanes follow the last column, without stores
  const bool computed = valid && x >= P.x0;    // columns left of x0 are INVALID
  const bool col_ok = computed && x >= Q.xlo && x <= Q.xhi;
  float* dout = disp + (size_t)view * Q.dstride + x;
  const size_t vo = (size_t)view * P.vstride + (size_t)x * D + (size_t)g * SB;
  const size_t rs = (size_t)W * D;
  const uint8_t* cv = cost + vo;
  uint8_t* btv = bt + vo;
  const uint32_t p1x2 = rep16(P.p1), p2m1 = P.p2 - P.p1;
  uint32_t L[NT], c[NT], out[NR];
  uint32_t ring[PF][NR];
  uint32_t m = 0;
  if constexpr (PASS != 2) {  // bottom-to-top pass (stores its path costs)
    // bottom -> top
#pragma unroll
    for (int j = 0; j < PF; ++j)
      if (j < H) ld_slice<NR>(cv + (size_t)(H - 1 - j) * rs, ring[j]);
    for (int s0 = 0; s0 < H; s0 += PF) {
#pragma unroll
      for (int j = 0; j < PF; ++j) {
        const int s = s0 + j;
        if (s < H) {
          const int y = H - 1 - s;
          widen_slice<NR>(ring[j], c);
          if (s + PF < H) ld_slice<NR>(cv + (size_t)(y - PF) * rs, ring[j]);
          m = s == 0 ? first_g<NT, G>(L, c) : step_g<NT, G>(L, c, m, p1x2, p2m1, g);
          narrow_slice<NR>(L, out);
          if (computed) st_slice<NR>(btv + (size_t)y * rs, out);
        }
      }
    }
  }
  if constexpr (PASS != 1) {  // top-to-bottom pass with the 4-path sum and the WTA
    // top -> bottom + sum + WTA; the other three paths of row y + PF are loaded at row y
    const uint8_t* lrv = lr + vo;
    const uint8_t* rlv = rl + vo;
    uint32_t ra[PF][NR], rb[PF][NR], re[PF][NR];
#pragma unroll
    for (int j = 0; j < PF; ++j) {
      if (j < H) {
        ld_slice<NR>(cv + (size_t)j * rs, ring[j]);
        ld_slice<NR>(btv + (size_t)j * rs, ra[j]);
        ld_slice<NR>(lrv + (size_t)j * rs, rb[j]);
        ld_slice<NR>(rlv + (size_t)j * rs, re[j]);
      }
    }
    for (int y0 = 0; y0 < H; y0 += PF) {
#pragma unroll
      for (int j = 0; j < PF; ++j) {
        const int y = y0 + j;
        if (y < H) {
          uint32_t wa[NT], wb[NT], we[NT];
          widen_slice<NR>(ring[j], c);
          widen_slice<NR>(ra[j], wa);
          widen_slice<NR>(rb[j], wb);
          widen_slice<NR>(re[j], we);
          if (y + PF < H) {
            const size_t o = (size_t)(y + PF) * rs;
            ld_slice<NR>(cv + o, ring[j]);
            ld_slice<NR>(btv + o, ra[j]);
            ld_slice<NR>(lrv + o, rb[j]);
            ld_slice<NR>(rlv + o, re[j]);
          }
          m = y == 0 ? first_g<NT, G>(L, c) : step_g<NT, G>(L, c, m, p1x2, p2m1, g);
          if (y >= Q.ylo && y <= Q.yhi && y < Q.rows) {  // uniform over the warp
            // S = the four u8 path costs summed (< 1024). Keys S << 6 | (d mod 64) per block of
            // disparities: D = 32 one block; D = 64: d < 32 (A) and d >= 32 (B), the reference's two
            // stores; D = 128: d < 64 and d >= 64.
            constexpr int SPLIT = D == 32 ? 64 : (D == 64 ? 32 : 64);  // first d of the second block
            uint32_t acc0 = 0xFFFFFFFFu, acc1 = 0xFFFFFFFFu;
            if constexpr (G > 1) {
              // every d of this lane lies in one block: one tree of SIMD minima
              uint32_t key[NT];
              const uint32_t dl = (uint32_t)((g * SB) & 63) * 0x10001u + 0x10000u;  // (d, d+1) mod 64 of word 0
#pragma unroll
              for (int k = 0; k < NT; ++k) {
                const uint32_t sk = (L[k] & 0x00FF00FFu) + wa[k] + wb[k] + we[k];
                myS[k] = sk;
                key[k] = sk * 64u + dl + (uint32_t)(2 * k) * 0x10001u;
              }
              uint32_t t = key[0];
              if constexpr (NT > 1) {
#pragma unroll
                for (int st = 1; st < NT; st *= 3) {
#pragma unroll
                  for (int k = 0; k + st < NT; k += 3 * st)
                    key[k] = k + 2 * st < NT ? __vimin3_u16x2(key[k], key[k + st], key[k + 2 * st])
                                             : min16x2(key[k], key[k + st]);
                }
                t = key[0];
              }
              if (g * SB < SPLIT) acc0 = t;
              else acc1 = t;
            } else {
#pragma unroll
              for (int k = 0; k < NT; ++k) {
                const uint32_t sk = (L[k] & 0x00FF00FFu) + wa[k] + wb[k] + we[k];
                myS[k] = sk;
                const uint32_t d0 = (uint32_t)(2 * (g * NT + k));
                const uint32_t key = sk * 64u + ((d0 & 63u) | (((d0 + 1u) & 63u) << 16));
                if ((int)d0 < SPLIT) acc0 = min16x2(acc0, key);
                else acc1 = min16x2(acc1, key);
              }
            }
            const uint32_t k0 = group_min<G>(hmin16(acc0)), k1 = group_min<G>(hmin16(acc1));
            __syncwarp();
            uint32_t sm;
            int ds;
            if constexpr (D == 32) {
              sm = k0 >> 6;
              ds = (int)(k0 & 63);
            } else if constexpr (D == 64) {
              const uint32_t SA = k0 >> 6, SB2 = k1 >> 6;
              sm = min(SA, SB2);
              ds = (int)(min(k0, k1) & 63);  // lowest d among the minima
              // A non-empty: odd rows take A; even rows take B = {t : S(t+32) == m, S(t) != m}
              // when non-empty, which needs the minimum in both blocks (rare); computed by every
              // lane of a warp where one column needs it (the shuffles must not diverge)
              if (Q.tie_rule == kTieRefB200 && (y & 1) == 0 && __any_sync(kFull, SA == SB2)) {
                const uint32_t mm = rep16(sm);
                uint32_t ax = 0xFFFFFFFFu;
#pragma unroll
                for (int k = 0; k < NT; ++k) {
                  const int w = g * NT + k;  // word index; B words are 16..31
                  if (w >= 16) {
                    const uint32_t z = colS[w - 16] - mm + 0x7FFF7FFFu;  // half >= 0x8000 iff S(t) != m
                    const uint32_t eq = ~z & 0x80008000u;               // bit 15 of a half iff S(t) == m
                    const uint32_t hx = myS[k] + (eq >> 5);              // excluded lanes get + 1024
                    const uint32_t t0 = (uint32_t)(2 * (w - 16));
                    ax = min16x2(ax, hx * 32u + (t0 | ((t0 + 1u) << 16)));
                  }
                }
                const uint32_t kx = group_min<G>(hmin16(ax));
                if (SA == sm) {
                  ds = (int)(k0 & 63);
                  if ((y & 1) == 0 && (kx >> 5) == sm) ds = 32 + (int)(kx & 31);
                }
              }
            } else {
              const uint32_t s0 = k0 >> 6, s1 = k1 >> 6;
              sm = min(s0, s1);
              ds = s0 <= s1 ? (int)(k0 & 63) : 64 + (int)(k1 & 63);
            }
            float dv = kInvalidFloat;
            if (col_ok && ds > 0 && ds < Q.dmax_excl) {
              const uint32_t w1 = colS[(ds - 1) >> 1];
              const float c1 = (float)(((ds - 1) & 1) ? (w1 >> 16) : (w1 & 0xFFFFu));
              const float c2 = (float)sm;
              float c3;
              if (ds + 1 < D) {
                const uint32_t w3 = colS[(ds + 1) >> 1];
                c3 = (float)(((ds + 1) & 1) ? (w3 >> 16) : (w3 & 0xFFFFu));
              } else {
                c3 = (float)ds;
              }
              const float d12 = __fsub_rn(c1, c2), d32 = __fsub_rn(c3, c2);
              const float uq = d12 < d32 ? d12 : d32;
              if (!(uq <= __fmul_rn(c2, __fsub_rn(1.0f, Q.uniqueness))))
                dv = __fadd_rn((float)(ds + P.min_d), subpix_bias(c1, c2, c3));
            }
            __syncwarp();
            if (valid && g == 0) dout[(size_t)y * W] = dv;
          } else if (valid && g == 0) {
            dout[(size_t)y * W] = kInvalidFloat;
          }
        }
      }
    }
  }
}

// five CTAs per SM (at most 96 registers) where a lane holds at most 32 disparities and G >= 2:
// many concurrent pairs are occupancy-bound (plain 1242x375x64: +5 % pairs/s over the
// unconstrained 113-128 registers); wider slices would spill
template <int K, int G, int PF, int PASS = 0>
__global__ void __launch_bounds__(128, (G >= 2 && 32 * K / G <= 32) ? 5 : 1)
    k_vpaths3(const uint8_t* __restrict__ cost, const uint8_t* __restrict__ lr,
                                                 const uint8_t* __restrict__ rl, uint8_t* __restrict__ bt,
                                                 float* __restrict__ disp, PlainParams P, WtaParams Q) {
  extern __shared__ uint32_t s_sum[];
  vpaths3_lane<K, G, PF, PASS>(cost, lr, rl, bt, disp, P, Q, blockIdx.y, (blockIdx.x * blockDim.x + threadIdx.x) / G,
                         threadIdx.x % G, s_sum + (threadIdx.x / G) * (16 * K + 1));
}

}  // namespace sgm

namespace sgm {

// =============================================================================================
// Initial-disparity levels (D = 32) with one thread (or G lanes) per scanline.
//
// The realigned recurrence (reference cusgm_ca.cu:1181-1338): with s = base - last_base,
//   L'(d) = C(d) + min(L(d), L(d+s-1)+P1, L(d+s+1)+P1, m+P2') - m        (uint32)
// where an index outside [0, 32) gives the candidate 127 and P2' = max(P1, P2/|last_base-base+1|).
// After a pixel with an INVALID base the reference sets m = 127 whatever the path costs are, and
// a realignment by more than the range makes every neighbour candidate 127, so t - m can wrap and
// later steps see wrapped values.
//
// 16-bit form. Read every uint32 value v of the reference as the signed integer r with
// v = r mod 2^32. While every value compared in a step has r in [-2^15, 2^15), the unsigned order
// of v equals that of r mod 2^16 and sums agree modulo 2^16 (so in the stored low byte): the
// recurrence can run on u16x2 words (two disparities per word, wrapping SIMD adds). With P1 >= 0,
// every P2' <= kNarrowP2 and C <= 255:
//   m >= 0: the candidate m + P2' is non-negative, so t is in [0, m + P2'] and L' in [-m, 255+P2'];
//   m <  0: m is the least of values that are all negative, so every L is in [m, -1]; t is the
//           least non-negative candidate (<= max(127, P2')) or a negative >= m, and L' is in
//           [0, 382 + P2' + |m|].
// So |m| grows by at most 382 + P2max per step, and a step that starts from |m| = M compares
// values below M + 382 + 2*P2max. The kernels check |m| <= kNarrowM once per block of up to
// kNarrowBlock steps: a block that starts there stays below kNarrowM + 8*(382 + P2max) + P2max
// = 29671 < 2^15 for P2max = kNarrowP2 = 2047. A scanline runs in 16 bits while the check
// holds (the sign-extended 16-bit minimum is exact) and otherwise continues in 32 bits from the
// sign-extended state, which is exact too. The switch is needed: realignments beyond the range
// alternating with cost-255 pixels can grow |m| by up to 255 every two steps.
// The shifted neighbours come from the scanline's old costs written to a shared-memory row padded
// with 127 - P1 (127 after + P1, modulo 2^16 or 2^32 for any P1); shifts beyond +-33 read padding
// only. 32-bit layout: kIPad words, 32 words, kIPad words. 16-bit layout (the first kIRow16 words
// of the same row): 17 words (34 halves), 16 words, 18 words.
// =============================================================================================
constexpr int kIPad = 34;                      // padding words on each side of a scanline row
constexpr int kIRow = kIPad + 32 + kIPad + 1;  // words per scanline row (odd: fewer bank conflicts)

// byte j of the slice -> word j (one byte permute each)
template <int ND>
__device__ __forceinline__ void unpack_bytes(const uint32_t (&r)[ND / 4], uint32_t (&c)[ND]) {
#pragma unroll
  for (int j = 0; j < ND; ++j) c[j] = __byte_perm(r[j >> 2], 0u, 0x4440u | (unsigned)(j & 3));
}
// low bytes of four words -> one word (three byte permutes)
template <int ND>
__device__ __forceinline__ void pack_bytes(const uint32_t (&L)[ND], uint32_t (&r)[ND / 4]) {
#pragma unroll
  for (int i = 0; i < ND / 4; ++i)
    r[i] = __byte_perm(__byte_perm(L[4 * i], L[4 * i + 1], 0x0040u), __byte_perm(L[4 * i + 2], L[4 * i + 3], 0x0040u),
                       0x5410u);
}

template <int ND, int G>
__device__ __forceinline__ uint32_t group_min32(const uint32_t (&v)[ND]) {
  uint32_t t[ND];
#pragma unroll
  for (int k = 0; k < ND; ++k) t[k] = v[k];
#pragma unroll
  for (int st = 1; st < ND; st *= 2) {
#pragma unroll
    for (int k = 0; k + st < ND; k += 2 * st) t[k] = min(t[k], t[k + st]);
  }
  return group_min<G>(t[0]);
}

// P2' for k = |last_base - base + 1| (table for k < kP2Tab).
__device__ __forceinline__ uint32_t p2_prime(const uint32_t* tab, int k, const InitParams& P) {
  return p2_term(tab, k, P);
}

// Shared-memory rows of a 128-thread block are stored scanline-minor: word w of the scanline
// at row[w * init_rs<G>()]. The stride 128/G + 2 is twice an odd number, so the G lanes of the
// 32/G scanlines of a warp that access the same word index (the same shift) hit 32 different
// banks.
template <int G>
__host__ __device__ constexpr int init_rs() { return 128 / G + 2; }

// One realigned step of the scanline held by G lanes (lane g owns d = g*ND .. g*ND+ND-1); every
// lane of the warp calls it. `row`: this scanline's kIRow words (padding already written).
template <int ND, int G>
__device__ __forceinline__ uint32_t init_step32(uint32_t (&L)[ND], const uint32_t (&c)[ND], uint32_t m, int s,
                                                uint32_t p2t, uint32_t p1, uint32_t* row, int g) {
#pragma unroll
  for (int j = 0; j < ND; ++j) row[(kIPad + g * ND + j) * init_rs<G>()] = L[j];
  __syncwarp();
  const int sc = s < -33 ? -33 : (s > 33 ? 33 : s);
  const uint32_t* src = row + (kIPad + g * ND + sc - 1) * init_rs<G>();  // word j: old L(g*ND + j + s - 1)
  uint32_t w[ND + 2];
#pragma unroll
  for (int j = 0; j < ND + 2; ++j) w[j] = src[j * init_rs<G>()];
  __syncwarp();
  const uint32_t l4 = m + p2t;
  uint32_t nl[ND];
#pragma unroll
  for (int j = 0; j < ND; ++j) {
    const uint32_t t = min(__vimin3_u32(L[j], w[j] + p1, w[j + 2] + p1), l4);
    nl[j] = c[j] + (t - m);
  }
#pragma unroll
  for (int j = 0; j < ND; ++j) L[j] = nl[j];
  return group_min32<ND, G>(nl);
}

constexpr int kINPad = 17;                         // 16-bit layout: padding words on the left
constexpr int kIRow16 = kINPad + 16 + kINPad + 1;  // 51 words; the last one is read at odd shifts
constexpr int32_t kNarrowP2 = 2047, kNarrowM = 8192;
constexpr int kNarrowBlock = 8;  // steps between two checks of |m| (the prefetch depth)

// Penalties that keep a 16-bit step exact (P2' = max(P1, P2 / k) or max(P1, p2_div0)).
__device__ __forceinline__ bool init_narrow_ok(const InitParams& P) {
  return P.p1s >= 0 && P.p1s <= kNarrowP2 && P.p2s <= kNarrowP2 && P.p2_div0 <= kNarrowP2;
}
__device__ __forceinline__ uint32_t sext16(uint32_t v) { return (uint32_t)(int32_t)(int16_t)(uint16_t)v; }
__device__ __forceinline__ bool narrow_m_ok(uint32_t m) {
  return (int32_t)m <= kNarrowM && (int32_t)m >= -kNarrowM;
}

// Padding of one scanline row for the 16-bit or the 32-bit layout, by the scanline's G lanes.
template <int G>
__device__ __forceinline__ void init_row_pad(uint32_t* row, uint32_t p1, bool narrow16, int g) {
  const uint32_t pad = kInvalidCost - p1;
  if (narrow16) {
    const uint32_t w = rep16(pad & 0xFFFFu);
    for (int k = g; k < kINPad; k += G) row[k * init_rs<G>()] = w;
    for (int k = g; k < kINPad + 1; k += G) row[(kINPad + 16 + k) * init_rs<G>()] = w;
  } else {
    for (int k = g; k < kIPad; k += G) {
      row[k * init_rs<G>()] = pad;
      row[(kIPad + 32 + k) * init_rs<G>()] = pad;
    }
  }
}

// One realigned step in 16 bits: L[0 .. ND/2) are this lane's u16x2 words (d = g*ND + 2k in the
// low half), r its ND raw cost bytes; writes the new words to nl and returns the new minimum,
// sign-extended. Every lane of the warp calls it. Requires p2t <= kNarrowP2 and |m| within the
// bound of its block (see above).
template <int ND, int G>
__device__ __forceinline__ uint32_t init_step16(const uint32_t (&L)[ND], uint32_t (&nl)[ND / 2],
                                                const uint32_t (&r)[ND / 4], uint32_t m, int s, uint32_t p2t,
                                                uint32_t p1, uint32_t* row, int g) {
  constexpr int NW = ND / 2;
#pragma unroll
  for (int k = 0; k < NW; ++k) row[(kINPad + g * NW + k) * init_rs<G>()] = L[k];
  __syncwarp();
  const int sc = s < -33 ? -33 : (s > 33 ? 33 : s);
  const int o = 2 * kINPad + g * ND + sc - 1;  // half index of old L(g*ND + s - 1), in [0, 98 - ND]
  const uint32_t* src = row + (o >> 1) * init_rs<G>();
  const uint32_t sel = (o & 1) ? 0x5432u : 0x3210u;
  uint32_t wd[NW + 2];
#pragma unroll
  for (int k = 0; k < NW + 2; ++k) wd[k] = src[k * init_rs<G>()];
  __syncwarp();
  // __viaddmin_u16x2(a, b, c) = min((a + b) mod 2^16, c) per half; with c = 0xFFFF it is the
  // wrapping add (the wrap of the add is what the exactness argument needs; the wrapping tests
  // of these kernels reach it)
  const uint32_t l4 = rep16((m + p2t) & 0xFFFFu);
  const uint32_t p1x2 = rep16(p1 & 0xFFFFu);
  const uint32_t negm = rep16((0u - m) & 0xFFFFu);
  uint32_t a[NW + 1];  // min(old L(d + s - 1) + P1, m + P2') for the word's two d
#pragma unroll
  for (int k = 0; k < NW + 1; ++k) a[k] = __viaddmin_u16x2(__byte_perm(wd[k], wd[k + 1], sel), p1x2, l4);
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    const uint32_t c2 = (k & 1) ? widen_hi(r[k >> 1]) : widen_lo(r[k >> 1]);
    const uint32_t cm = __viaddmin_u16x2(c2, negm, 0xFFFFFFFFu);  // C - m
    nl[k] = __viaddmin_u16x2(__vimin3_u16x2(L[k], a[k], a[k + 1]), cm, 0xFFFFFFFFu);
  }
  return sext16(group_min16<NW, G>(nl));
}

// 16-bit words -> one uint32 per disparity (in place, sign-extended: exact, see above).
template <int ND>
__device__ __forceinline__ void widen_state(uint32_t (&L)[ND]) {
#pragma unroll
  for (int k = ND / 2 - 1; k >= 0; --k) {
    const uint32_t w = L[k];
    L[2 * k + 1] = sext16(w >> 16);
    L[2 * k] = sext16(w & 0xFFFFu);
  }
}

// Stored path costs (low bytes) of the state, in either form.
template <int ND>
__device__ __forceinline__ void pack_state(const uint32_t (&L)[ND], bool wide, uint32_t (&out)[ND / 4]) {
  if (wide) {
    pack_bytes<ND>(L, out);
  } else {
#pragma unroll
    for (int i = 0; i < ND / 4; ++i) out[i] = narrow(L[2 * i], L[2 * i + 1]);
  }
}

// First pixel of a scanline: L = C. Returns min C over the scanline.
template <int ND, int G>
__device__ __forceinline__ uint32_t init_first(uint32_t (&L)[ND], const uint32_t (&r)[ND / 4], bool wide) {
  if (wide) {
    uint32_t c[ND];
    unpack_bytes<ND>(r, c);
#pragma unroll
    for (int k = 0; k < ND; ++k) L[k] = c[k];
    return group_min32<ND, G>(c);
  }
  uint32_t w[ND / 2];
  widen_slice<ND / 4>(r, w);
#pragma unroll
  for (int k = 0; k < ND / 2; ++k) L[k] = w[k];
  return group_min16<ND / 2, G>(w);
}

// One step of a scanline; keeps the result only for a valid base (else m = 127, L unchanged).
// 16-bit form (L[0 .. ND/2) are u16x2 words):
template <int ND, int G>
__device__ __forceinline__ void init_advance16(uint32_t (&L)[ND], const uint32_t (&r)[ND / 4], uint32_t& m,
                                               int& last_base, int base, const InitParams& P,
                                               const uint32_t* p2tab, uint32_t* row, int g) {
  uint32_t nl[ND / 2];
  // P2' only matters for a valid base (an INVALID one discards the step)
  const uint32_t p2t = base != kInvalidShort ? p2_prime(p2tab, abs(last_base - base + 1), P) : 0u;
  const uint32_t mn = init_step16<ND, G>(L, nl, r, m, base - last_base, p2t,
                                         P.p1, row, g);
  if (base != kInvalidShort) {
#pragma unroll
    for (int k = 0; k < ND / 2; ++k) L[k] = nl[k];
    m = mn;
    last_base = base;
  } else {
    m = kInvalidCost;
  }
}
// 32-bit form (one uint32 per disparity; the row holds the 32-bit padding):
template <int ND, int G>
__device__ __forceinline__ void init_advance32(uint32_t (&L)[ND], const uint32_t (&r)[ND / 4], uint32_t& m,
                                               int& last_base, int base, const InitParams& P,
                                               const uint32_t* p2tab, uint32_t* row, int g) {
  uint32_t c[ND], Lk[ND];
  unpack_bytes<ND>(r, c);
#pragma unroll
  for (int k = 0; k < ND; ++k) Lk[k] = L[k];
  const uint32_t p2t = base != kInvalidShort ? p2_prime(p2tab, abs(last_base - base + 1), P) : 0u;
  const uint32_t mn = init_step32<ND, G>(Lk, c, m, base - last_base, p2t,
                                         P.p1, row, g);
  if (base != kInvalidShort) {
#pragma unroll
    for (int k = 0; k < ND; ++k) L[k] = Lk[k];
    m = mn;
    last_base = base;
  } else {
    m = kInvalidCost;
  }
}

// Between scanlines the row holds the 16-bit padding. A scanline that continues in 32 bits
// (from step `from`; 0: from its first pixel) widens its state and switches the padding, and
// switches it back at its end. Warp-uniform.
template <int ND, int G>
__device__ __forceinline__ void init_go_wide(uint32_t (&L)[ND], int from, const InitParams& P, uint32_t* row,
                                             int g) {
  if (from > 0) widen_state<ND>(L);
  __syncwarp();
  init_row_pad<G>(row, P.p1, false, g);
  __syncwarp();
}
template <int G>
__device__ __forceinline__ void init_go_narrow(const InitParams& P, uint32_t* row, int g) {
  __syncwarp();
  init_row_pad<G>(row, P.p1, true, g);
  __syncwarp();
}

// WTA of one pixel of an initial-disparity level from the u16x2 sums of its four paths
// (reference Kernel_ComputeDisparityByWTA for initial disparities). ok: the pixel may be valid.
// Keys S*32 + d (S <= 1020) fit 16 bits: their minimum is the lowest d of least S. Rule
// kTieRefB200: the lowest tied d whose uniqueness test passes; kTieLowest: the lowest tied d.
template <int G>
__device__ __forceinline__ float init_candidate(const uint32_t* colS, int d, uint32_t sm, int base,
                                                const WtaParams& Q) {
  if (d <= 1 || d >= kLevelRange - 1) return kInvalidFloat;
  const uint32_t w1 = colS[((d - 1) >> 1) * init_rs<G>()], w3 = colS[((d + 1) >> 1) * init_rs<G>()];
  const float c1 = (float)((d - 1) & 1 ? w1 >> 16 : w1 & 0xFFFFu), c2 = (float)sm,
              c3 = (float)((d + 1) & 1 ? w3 >> 16 : w3 & 0xFFFFu);
  const float d12 = __fsub_rn(c1, c2), d32 = __fsub_rn(c3, c2);
  const float uq = d12 < d32 ? d12 : d32;
  if (uq <= __fmul_rn(c2, __fsub_rn(1.0f, Q.uniqueness))) return kInvalidFloat;
  return __fadd_rn((float)(d + base), subpix_bias(c1, c2, c3));
}
template <int ND, int G>
__device__ __forceinline__ void init_wta_pixel(const uint32_t (&S2)[ND / 2], uint32_t* colS, int g, int base,
                                               bool ok, const WtaParams& Q, bool store, float* dst) {
  constexpr int NW = ND / 2;
  const uint32_t d0 = (uint32_t)(g * ND) * 0x10001u + 0x10000u;  // (d, d + 1) of word 0
  uint32_t key[NW];
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    colS[(g * NW + k) * init_rs<G>()] = S2[k];
    key[k] = (S2[k] << 5) + d0 + (uint32_t)(2 * k) * 0x10001u;
  }
  const uint32_t kmin = group_min16<NW, G>(key);
  __syncwarp();
  const uint32_t sm = kmin >> 5;
  const int ds = (int)(kmin & 31u);
  float dv = init_candidate<G>(colS, ds, sm, base, Q);  // the same in every lane of the group
  if (Q.tie_rule == kTieRefB200) {
    // while the candidate fails: the next tied d, i.e. the least key above kcur and below
    // (sm + 1) * 32 (keys <= kcur wrap to >= 2^15 in key - kcur - 1)
    const uint32_t lim = (sm + 1u) << 5;
    uint32_t kcur = kmin;
    for (;;) {
      const bool need = dv == kInvalidFloat && kcur + 1u < lim;
      if (!__any_sync(kFull, need)) break;
      const uint32_t neg = rep16((0u - (kcur + 1u)) & 0xFFFFu);
      uint32_t u[NW];
#pragma unroll
      for (int k = 0; k < NW; ++k) u[k] = __viaddmin_u16x2(key[k], neg, 0xFFFFFFFFu);
      const uint32_t nk = group_min16<NW, G>(u) + kcur + 1u;
      if (need) {
        kcur = nk < lim ? nk : lim;
        if (nk < lim) dv = init_candidate<G>(colS, (int)(nk & 31u), sm, base, Q);
      }
    }
  }
  if (!ok) dv = kInvalidFloat;
  __syncwarp();
  if (store && g == 0) *dst = dv;
}

// Cost volume of an initial-disparity level (reference cusgm_cc.cu:173-237 / 294-360):
// view 0: pos = x - d - base, C = (popc(own ^ oth[pos]) + CostAdjust(d)) & 0xFF for 0 < pos < W,
// else the invalid cost; view 1: pos = x + d + base, partner oth[pos] for 0 < pos < W else oth[0].
// One CTA per (row, view); the partner row's census words in shared memory (W words).
// Row y of view `view` by one block (every thread calls it); oth_s: W words of shared memory.
// The 32 costs of one pixel at an initial-disparity level. View 0: partner x - d - base, valid
// iff 0 < pos < W, else the invalid cost; view 1: partner x + d + base, oth[0] when out of range.
// The valid disparities form one interval, taken as a bit mask once per pixel; partner loads use
// immediate offsets from oth_s + x -/+ base (made only for valid d).
template <typename Word, bool V0>
__device__ __forceinline__ void cost3_init_px(const Word a, const Word* oth_s, int x, int base, int W,
                                              uint32_t invalid, uint8_t* __restrict__ dst) {
  // valid d: view 0  x-base-W < d < x-base;  view 1  -x-base < d < W-x-base
  const int lo = V0 ? x - base - W + 1 : 1 - x - base;
  const int hi = V0 ? x - base - 1 : W - 1 - x - base;
  const int l = max(lo, 0), h = min(hi, kLevelRange - 1);
  const uint32_t mask = l <= h ? (0xFFFFFFFFu >> (31 - h)) & (0xFFFFFFFFu << l) : 0u;
  const Word* p = oth_s + (V0 ? x - base : x + base);
  const Word oth0 = oth_s[0];
  uint32_t q[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    uint32_t c[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int d = 4 * i + b;
      const bool ok = (mask >> d) & 1u;
      if (V0) {
        c[b] = ok ? ((popc_word((Word)(a ^ p[-d])) + cost_adjust(d)) & 0xFFu) : invalid;
      } else {
        const Word o = ok ? p[d] : oth0;
        c[b] = (popc_word((Word)(a ^ o)) + cost_adjust(d)) & 0xFFu;
      }
    }
    q[i] = __byte_perm(__byte_perm(c[0], c[1], 0x0040u), __byte_perm(c[2], c[3], 0x0040u), 0x5410u);
  }
  uint4* o = reinterpret_cast<uint4*>(dst);
  o[0] = make_uint4(q[0], q[1], q[2], q[3]);
  o[1] = make_uint4(q[4], q[5], q[6], q[7]);
}

template <typename Word>
__device__ __forceinline__ void cost3_init_row(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                               const int16_t* __restrict__ init_l, const int16_t* __restrict__ init_r,
                                               uint8_t* __restrict__ cost, const InitParams& P, int y, int view,
                                               Word* oth_s) {
  const int W = P.W;
  const Word* own = (view == 0 ? cs_l : cs_r) + (size_t)y * W;
  const Word* oth = (view == 0 ? cs_r : cs_l) + (size_t)y * W;
  const int16_t* ib = (view == 0 ? init_l : init_r) + (size_t)y * W;
  for (int i = threadIdx.x; i < W; i += blockDim.x) oth_s[i] = oth[i];
  __syncthreads();
  uint8_t* crow = cost + (size_t)view * P.vstride + (size_t)y * W * kLevelRange;
  for (int x = P.x0 + threadIdx.x; x < W; x += blockDim.x) {
    const int base = ib[x];
    uint8_t* dst = crow + (size_t)x * kLevelRange;
    if (view == 0) cost3_init_px<Word, true>(own[x], oth_s, x, base, W, P.invalid_cost, dst);
    else cost3_init_px<Word, false>(own[x], oth_s, x, base, W, P.invalid_cost, dst);
  }
}

template <typename Word>
__global__ void __launch_bounds__(256) k_cost3_init(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                                    const int16_t* __restrict__ init_l,
                                                    const int16_t* __restrict__ init_r, uint8_t* __restrict__ cost,
                                                    InitParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cost3_init_row<Word>(cs_l, cs_r, init_l, init_r, cost, P, blockIdx.x, blockIdx.y, reinterpret_cast<Word*>(smem_raw));
}

// Horizontal paths of an initial-disparity level, G lanes per scanline (view, dir, y) with the
// scanline index as in hpaths3_lane. INVALID bases are skipped (m := 127, L and last_base kept);
// the first pixel sets last_base whatever its base.
template <int G, int PF>
__device__ __forceinline__ void hpaths3_init_lane(const uint8_t* __restrict__ cost,
                                                  const int16_t* __restrict__ init_l,
                                                  const int16_t* __restrict__ init_r, uint8_t* __restrict__ lr,
                                                  uint8_t* __restrict__ rl, const InitParams& P, int nviews, int i,
                                                  int g, uint32_t* row, const uint32_t* p2tab) {
  constexpr int ND = kLevelRange / G, NR = ND / 4;
  const int H = P.H, W = P.W;
  const int nscan = nviews * 2 * H;
  const bool valid = i < nscan;
  if (!valid) i = nscan - 1;
  const int grp = i / H;
  const int y = i - grp * H;
  const int view = grp >> 1, dir = grp & 1;
  const int len = W - P.x0;
  if (len <= 0) return;
  const size_t vo = (size_t)view * P.vstride + (size_t)y * W * kLevelRange + (size_t)g * ND;
  const uint8_t* crow = cost + vo;
  uint8_t* orow = (dir == 0 ? lr : rl) + vo;
  const int16_t* ib = (view == 0 ? init_l : init_r) + (size_t)y * W;
  const int xs = dir == 0 ? P.x0 : W - 1;
  const int dx = dir == 0 ? 1 : -1;
  uint32_t L[ND], out[NR];
  uint32_t m = 0;
  int last_base = 0;
  // 16-bit steps with a PF-deep prefetch ring up to s_wide, 32-bit steps (plain loads) after it
  int s_wide = init_narrow_ok(P) ? len : 0;
  static_assert(PF <= kNarrowBlock, "the 16-bit bound holds for kNarrowBlock steps");
  static_assert(16 % PF == 0, "blocks of PF steps start every 16 steps");
  if (s_wide > 0) {
    uint32_t ring[PF][NR];
    int rbase[PF];
#pragma unroll
    for (int j = 0; j < PF; ++j) {
      if (j < len) {
        ld_slice<NR>(crow + (size_t)(xs + j * dx) * kLevelRange, ring[j]);
        rbase[j] = ib[xs + j * dx];
      }
    }
    for (int s0 = 0; s0 < s_wide; s0 += PF) {
      prefetch_row_ahead<kLevelRange>(crow - (size_t)g * ND, xs, dx, s0, len, g);
#pragma unroll
      for (int j = 0; j < PF; ++j) {
        const int s = s0 + j;
        if (s < s_wide) {
          const int x = xs + s * dx;
          uint32_t r[NR];
#pragma unroll
          for (int k = 0; k < NR; ++k) r[k] = ring[j][k];
          const int base = rbase[j];
          if (s + PF < len) {
            ld_slice<NR>(crow + (size_t)(x + PF * dx) * kLevelRange, ring[j]);
            rbase[j] = ib[x + PF * dx];
          }
          if (s == 0) {
            m = init_first<ND, G>(L, r, false);
            last_base = base;
          } else {
            // every lane steps (the exchange and the minimum are warp-wide); kept for a valid base
            init_advance16<ND, G>(L, r, m, last_base, base, P, p2tab, row, g);
          }
#pragma unroll
          for (int i = 0; i < NR; ++i) out[i] = narrow(L[2 * i], L[2 * i + 1]);
          if (valid) st_slice<NR>(orow + (size_t)x * kLevelRange, out);
        }
      }
      if (__any_sync(kFull, !narrow_m_ok(m))) s_wide = min(len, s0 + PF);  // 32 bits after this block
    }
  }
  if (s_wide < len) {
    init_go_wide<ND, G>(L, s_wide, P, row, g);
    for (int s = s_wide; s < len; ++s) {
      const int x = xs + s * dx;
      uint32_t r[NR];
      ld_slice<NR>(crow + (size_t)x * kLevelRange, r);
      const int base = ib[x];
      if (s == 0) {
        m = init_first<ND, G>(L, r, true);
        last_base = base;
      } else {
        init_advance32<ND, G>(L, r, m, last_base, base, P, p2tab, row, g);
      }
      pack_bytes<ND>(L, out);
      if (valid) st_slice<NR>(orow + (size_t)x * kLevelRange, out);
    }
    init_go_narrow<G>(P, row, g);
  }
}

template <int G, int PF>
__global__ void __launch_bounds__(128) k_hpaths3_init(const uint8_t* __restrict__ cost,
                                                      const int16_t* __restrict__ init_l,
                                                      const int16_t* __restrict__ init_r, uint8_t* __restrict__ lr,
                                                      uint8_t* __restrict__ rl, InitParams P, int nviews) {
  __shared__ uint32_t p2tab[kP2Tab];
  __shared__ uint32_t rows[init_rs<G>() * kIRow];
  fill_p2_table(p2tab, P, threadIdx.x, blockDim.x);
  uint32_t* row = rows + threadIdx.x / G;
  init_row_pad<G>(row, P.p1, true, threadIdx.x % G);
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  hpaths3_init_lane<G, PF>(cost, init_l, init_r, lr, rl, P, nviews, t / G, threadIdx.x % G, row, p2tab);
}

// Vertical paths + sum + WTA of an initial-disparity level, G lanes per column. last_base starts
// from row 0's base in both directions (reference behaviour). WTA (reference
// Kernel_ComputeDisparityByWTA for initial disparities): d in [2, 30]; tie rule kTieRefB200 =
// the lowest tied d whose uniqueness test passes (every tied lane writes its own result, a valid
// one wins), kTieLowest = the lowest tied d, then tested.
// PASS as in vpaths3_lane.
template <int G, int PF, int PASS = 0>
__device__ __forceinline__ void vpaths3_init_lane(const uint8_t* __restrict__ cost, const uint8_t* __restrict__ lr,
                                                  const uint8_t* __restrict__ rl, const int16_t* __restrict__ init_l,
                                                  const int16_t* __restrict__ init_r, uint8_t* __restrict__ bt,
                                                  float* __restrict__ disp, const InitParams& P, const WtaParams& Q,
                                                  int view, int xc, int g, uint32_t* row, uint32_t* colS,
                                                  const uint32_t* p2tab) {
  constexpr int ND = kLevelRange / G, NR = ND / 4, NW = ND / 2;
  const int W = P.W, H = P.H;
  const bool valid = xc < W;
  const int x = valid ? xc : W - 1;
  const bool computed = valid && x >= P.x0;
  const bool col_ok = computed && x >= 5 && x <= W - 5;
  float* dout = disp + (size_t)view * Q.dstride + x;
  const int16_t* ib = (view == 0 ? init_l : init_r) + x;
  const size_t vo = (size_t)view * P.vstride + (size_t)x * kLevelRange + (size_t)g * ND;
  const size_t rs = (size_t)W * kLevelRange;
  const uint8_t* cv = cost + vo;
  uint8_t* btv = bt + vo;
  const bool narrow_ok = init_narrow_ok(P);
  uint32_t L[ND], out[NR];
  uint32_t m = 0;
  const int base0 = ib[0];
  int last_base = base0;
  if constexpr (PASS != 2) {  // bottom-to-top pass (stores its path costs)
    // bottom -> top: 16-bit steps with a prefetch ring up to s_wide, then 32-bit steps
    int s_wide = narrow_ok ? H : 0;
    static_assert(PF <= kNarrowBlock, "the 16-bit bound holds for kNarrowBlock steps");
    if (s_wide > 0) {
      uint32_t ring[PF][NR];
      int rbase[PF];
#pragma unroll
      for (int j = 0; j < PF; ++j) {
        if (j < H) {
          ld_slice<NR>(cv + (size_t)(H - 1 - j) * rs, ring[j]);
          rbase[j] = ib[(size_t)(H - 1 - j) * W];
        }
      }
      for (int s0 = 0; s0 < s_wide; s0 += PF) {
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const int s = s0 + j;
          if (s < s_wide) {
            const int y = H - 1 - s;
            uint32_t r[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) r[k] = ring[j][k];
            const int base = rbase[j];
            if (s + PF < H) {
              ld_slice<NR>(cv + (size_t)(y - PF) * rs, ring[j]);
              rbase[j] = ib[(size_t)(y - PF) * W];
            }
            if (s == 0) m = init_first<ND, G>(L, r, false);
            else init_advance16<ND, G>(L, r, m, last_base, base, P, p2tab, row, g);
            if ((s == 0 || base != kInvalidShort) && computed) {
#pragma unroll
              for (int i = 0; i < NR; ++i) out[i] = narrow(L[2 * i], L[2 * i + 1]);
              st_slice<NR>(btv + (size_t)y * rs, out);
            }
          }
        }
        if (__any_sync(kFull, !narrow_m_ok(m))) s_wide = min(H, s0 + PF);
      }
    }
    if (s_wide < H) {
      init_go_wide<ND, G>(L, s_wide, P, row, g);
      for (int s = s_wide; s < H; ++s) {
        const int y = H - 1 - s;
        uint32_t r[NR];
        ld_slice<NR>(cv + (size_t)y * rs, r);
        const int base = ib[(size_t)y * W];
        if (s == 0) m = init_first<ND, G>(L, r, true);
        else init_advance32<ND, G>(L, r, m, last_base, base, P, p2tab, row, g);
        if ((s == 0 || base != kInvalidShort) && computed) {
          pack_bytes<ND>(L, out);
          st_slice<NR>(btv + (size_t)y * rs, out);
        }
      }
      init_go_narrow<G>(P, row, g);
    }
  }
  if constexpr (PASS != 1) {  // top-to-bottom pass with the 4-path sum and the WTA
    // top -> bottom + sum + WTA (a new scanline)
    const uint8_t* lrv = lr + vo;
    const uint8_t* rlv = rl + vo;
    last_base = base0;
    int y_wide = narrow_ok ? H : 0;
    if (y_wide > 0) {
      uint32_t ring[PF][NR], ra[PF][NR], rb[PF][NR], re[PF][NR];
      int rbase[PF];
#pragma unroll
      for (int j = 0; j < PF; ++j) {
        if (j < H) {
          const size_t o = (size_t)j * rs;
          ld_slice<NR>(cv + o, ring[j]);
          ld_slice<NR>(btv + o, ra[j]);
          ld_slice<NR>(lrv + o, rb[j]);
          ld_slice<NR>(rlv + o, re[j]);
          rbase[j] = ib[(size_t)j * W];
        }
      }
      for (int y0 = 0; y0 < y_wide; y0 += PF) {
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const int y = y0 + j;
          if (y < y_wide) {
            uint32_t r[NR], S2[NW];
#pragma unroll
            for (int k = 0; k < NR; ++k) {
              r[k] = ring[j][k];
              // sums of the three stored paths, two disparities per word (each half <= 765)
              S2[2 * k] = widen_lo(ra[j][k]) + widen_lo(rb[j][k]) + widen_lo(re[j][k]);
              S2[2 * k + 1] = widen_hi(ra[j][k]) + widen_hi(rb[j][k]) + widen_hi(re[j][k]);
            }
            const int base = rbase[j];
            if (y + PF < H) {
              const size_t o = (size_t)(y + PF) * rs;
              ld_slice<NR>(cv + o, ring[j]);
              ld_slice<NR>(btv + o, ra[j]);
              ld_slice<NR>(lrv + o, rb[j]);
              ld_slice<NR>(rlv + o, re[j]);
              rbase[j] = ib[(size_t)(y + PF) * W];
            }
            if (y == 0) m = init_first<ND, G>(L, r, false);
            else init_advance16<ND, G>(L, r, m, last_base, base, P, p2tab, row, g);
            const bool skipped = y > 0 && base == kInvalidShort;
            if (y >= 5 && y <= H - 5 && y < Q.rows) {  // uniform over the warp
#pragma unroll
              for (int k = 0; k < NW; ++k) S2[k] += L[k] & 0x00FF00FFu;  // + this path (<= 1020 per half)
              init_wta_pixel<ND, G>(S2, colS, g, base, col_ok && base != kInvalidShort && !skipped, Q, valid,
                                    dout + (size_t)y * W);
            } else if (valid && g == 0) {
              dout[(size_t)y * W] = kInvalidFloat;
            }
          }
        }
        if (__any_sync(kFull, !narrow_m_ok(m))) y_wide = min(H, y0 + PF);
      }
    }
    if (y_wide < H) {
      init_go_wide<ND, G>(L, y_wide, P, row, g);
      for (int y = y_wide; y < H; ++y) {
        const size_t o = (size_t)y * rs;
        uint32_t r[NR], S2[NW];
        ld_slice<NR>(cv + o, r);
        {
          uint32_t qa[NR], qb[NR], qe[NR];
          ld_slice<NR>(btv + o, qa);
          ld_slice<NR>(lrv + o, qb);
          ld_slice<NR>(rlv + o, qe);
#pragma unroll
          for (int k = 0; k < NR; ++k) {
            S2[2 * k] = widen_lo(qa[k]) + widen_lo(qb[k]) + widen_lo(qe[k]);
            S2[2 * k + 1] = widen_hi(qa[k]) + widen_hi(qb[k]) + widen_hi(qe[k]);
          }
        }
        const int base = ib[(size_t)y * W];
        if (y == 0) m = init_first<ND, G>(L, r, true);
        else init_advance32<ND, G>(L, r, m, last_base, base, P, p2tab, row, g);
        const bool skipped = y > 0 && base == kInvalidShort;
        if (y >= 5 && y <= H - 5 && y < Q.rows) {
#pragma unroll
          for (int k = 0; k < NW; ++k) S2[k] += (L[2 * k] & 0xFFu) | ((L[2 * k + 1] & 0xFFu) << 16);
          init_wta_pixel<ND, G>(S2, colS, g, base, col_ok && base != kInvalidShort && !skipped, Q, valid,
                                dout + (size_t)y * W);
        } else if (valid && g == 0) {
          dout[(size_t)y * W] = kInvalidFloat;
        }
      }
      init_go_narrow<G>(P, row, g);
    }
  }
}

template <int G, int PF, int PASS = 0>
__global__ void __launch_bounds__(128) k_vpaths3_init(const uint8_t* __restrict__ cost,
                                                      const uint8_t* __restrict__ lr, const uint8_t* __restrict__ rl,
                                                      const int16_t* __restrict__ init_l,
                                                      const int16_t* __restrict__ init_r, uint8_t* __restrict__ bt,
                                                      float* __restrict__ disp, InitParams P, WtaParams Q) {
  __shared__ uint32_t p2tab[kP2Tab];
  __shared__ uint32_t rows[init_rs<G>() * kIRow];
  __shared__ uint32_t sums[init_rs<G>() * (kLevelRange / 2)];
  fill_p2_table(p2tab, P, threadIdx.x, blockDim.x);
  uint32_t* row = rows + threadIdx.x / G;
  init_row_pad<G>(row, P.p1, true, threadIdx.x % G);
  __syncthreads();
  const int xc = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  vpaths3_init_lane<G, PF, PASS>(cost, lr, rl, init_l, init_r, bt, disp, P, Q, blockIdx.y, xc, threadIdx.x % G, row,
                           sums + threadIdx.x / G, p2tab);
}

}  // namespace sgm
