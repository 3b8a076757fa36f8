// SGM stereo kernels for sm_100a.
//
// Data layout in HBM (dense, no pitch):
//   images        u8   [H][W]                 per view
//   census        u32/u64 [H][W]              per view (5x5 -> u32, 9x7 -> u64)
//   volumes       u8   [view][H][W][D]        cost, left->right, right->left, bottom->top path costs
//   disparity     f32  [view][H][W]
// Views: 0 = left image matched against the right one, 1 = right image against the left
// (the second view exists only when the left-right check is on).
//
// Warp mapping of the path scans: one warp owns one scanline; lane l holds the K = D/32
// contiguous disparities d = l*K + j, so the d-1 / d+1 neighbours cross lanes only at j = 0
// and j = K-1 (two shuffles per step), and the per-step minimum is one REDUX (__reduce_min_sync).
#pragma once
#include "sgm_common.cuh"

namespace sgm {

// ---------------------------------------------------------------------------------------------
// Census transform (reference SgmStereoCuda/cusgm_cc.cu:30-106). Both views in one launch
// (blockIdx.z). Left border value 0, right border value 0xFFFFFFFF (zero-extended).
// ---------------------------------------------------------------------------------------------
template <typename Word, int CSW, int CSH>
__device__ __forceinline__ Word census_value(const uint8_t* __restrict__ img, int x, int y, int W, int H, bool right) {
  Word v = 0;
  if (x < CSW || x >= W - CSW || y < CSH || y >= H - CSH) {
    v = right ? (Word)0xFFFFFFFFu : (Word)0;
  } else {
    const uint8_t c = __ldg(img + (size_t)y * W + x);
#pragma unroll
    for (int dy = -CSH; dy <= CSH; ++dy) {
      const uint8_t* row = img + (size_t)(y + dy) * W + x;
#pragma unroll
      for (int dx = -CSW; dx <= CSW; ++dx) v = (Word)((v << 1) | (Word)(__ldg(row + dx) < c));
    }
  }
  return v;
}

template <typename Word, int CSW, int CSH>
__global__ void __launch_bounds__(128) k_census(const uint8_t* __restrict__ img_l, const uint8_t* __restrict__ img_r,
                                                Word* __restrict__ cs_l, Word* __restrict__ cs_r, int W, int H) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const bool right = blockIdx.z == 1;
  if (x >= W) return;
  (right ? cs_r : cs_l)[(size_t)y * W + x] = census_value<Word, CSW, CSH>(right ? img_r : img_l, x, y, W, H, right);
}

// Census of 4 consecutive pixels per thread with byte-parallel compares (same values as
// census_value). A 128-thread block covers 512 pixels of RY rows; the rows y-CSH .. y+RY-1+CSH,
// columns x0-4 .. x0+515 are staged in shared memory (`tile`, census4_tile_words<CSH, RY>()
// words). For each window offset the thread compares the 4-byte window of its pixels' neighbours
// with their 4 centres at once:
//   a < c (unsigned, per byte)  <=>  top bit of (~a & c) | (~(a ^ c) & ~((a | 0x80) - (c & 0x7f)))
// (the subtraction cannot borrow across bytes), and collects offset k's bit of pixel p in byte p
// of word k / 8 at bit 7 - k % 8; a byte transpose then yields each pixel's MSB-first word.
constexpr int kCensus4Stride = 131;  // words per staged row (130 used)
constexpr int kCensusRows = 8;      // output rows per block (RY)
template <int CSH, int RY>
__host__ __device__ constexpr int census4_tile_words() { return (RY + 2 * CSH) * kCensus4Stride; }

template <typename Word, int CSW, int CSH, int RY>
__device__ __forceinline__ void census4_tile(const uint8_t* __restrict__ img, Word* __restrict__ cs, int W, int H,
                                             bool right, int bx, int by, uint32_t* tile) {
  static_assert(CSW <= 4, "the window spans x0-4 .. x0+7");
  constexpr int TR = RY + 2 * CSH, NC = 2 * CSW + 1, NB = (2 * CSH + 1) * NC, NG = (NB + 7) / 8;
  static_assert(NG == (int)sizeof(Word) || NG == 4 || NG == 8, "census word of NB bits");
  // stage: word w of row r holds pixels bx - 4 + 4w .. +3 of image row by + r - CSH (0 outside);
  // the first barrier lets a block call this for several tiles in a row
  __syncthreads();
  for (int i = threadIdx.x; i < TR * 130; i += 128) {
    const int r = i / 130, w = i - r * 130;
    const int yy = by + r - CSH, xx = bx - 4 + 4 * w;
    uint32_t v = 0;
    if (yy >= 0 && yy < H) {
      const uint8_t* row = img + (size_t)yy * W;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (xx + j >= 0 && xx + j < W) v |= (uint32_t)__ldg(row + xx + j) << (8 * j);
    }
    tile[r * kCensus4Stride + w] = v;
  }
  __syncthreads();
  const int t = threadIdx.x, x0 = bx + 4 * t;
  if (x0 >= W) return;
  const uint32_t* tw = tile + t;
#pragma unroll 1
  for (int oy = 0; oy < RY; ++oy) {
    const int y = by + oy;
    if (y >= H) break;
    const uint32_t c = tw[(oy + CSH) * kCensus4Stride + 1], c7 = c & 0x7F7F7F7Fu;
    uint32_t acc[NG];
#pragma unroll
    for (int g = 0; g < NG; ++g) acc[g] = 0;
#pragma unroll
    for (int dy = 0; dy <= 2 * CSH; ++dy) {
#pragma unroll
      for (int dx = -CSW; dx <= CSW; ++dx) {
        const int k = dy * NC + dx + CSW, s = 4 + dx;
        const uint32_t* w = tw + (oy + dy) * kCensus4Stride;  // shared: words x0-4, x0, x0+4
        uint32_t a;
        if (s == 0) a = w[0];
        else if (s == 4) a = w[1];
        else if (s == 8) a = w[2];  // the compiler loads each of the row's 3 words once
        else if (s < 4) a = __byte_perm(w[0], w[1], (uint32_t)(s | (s + 1) << 4 | (s + 2) << 8 | (s + 3) << 12));
        else a = __byte_perm(w[1], w[2], (uint32_t)((s - 4) | (s - 3) << 4 | (s - 2) << 8 | (s - 1) << 12));
        const uint32_t d = (a | 0x80808080u) - c7;
        const uint32_t lt = (~a & c) | (~(a ^ c) & ~d);  // top bit of each byte: a < c
        acc[k >> 3] |= (lt >> (k & 7)) & (0x80808080u >> (k & 7));
      }
    }
    Word* out = cs + (size_t)y * W;
    const bool row_border = y < CSH || y >= H - CSH;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int x = x0 + p;
      if (x >= W) break;
      const uint32_t sel = (uint32_t)(p | (p + 4) << 4);
      Word v;
      if constexpr (NG == 8) {
        const uint32_t hi = __byte_perm(__byte_perm(acc[3], acc[2], sel), __byte_perm(acc[1], acc[0], sel), 0x5410);
        const uint32_t lo = __byte_perm(__byte_perm(acc[7], acc[6], sel), __byte_perm(acc[5], acc[4], sel), 0x5410);
        v = (Word)(((((uint64_t)hi) << 32) | lo) >> (64 - NB));
      } else {
        const uint32_t w32 = __byte_perm(__byte_perm(acc[3], acc[2], sel), __byte_perm(acc[1], acc[0], sel), 0x5410);
        v = (Word)(w32 >> (32 - NB));
      }
      if (row_border || x < CSW || x >= W - CSW) v = right ? (Word)0xFFFFFFFFu : (Word)0;
      out[x] = v;
    }
  }
}

// Both views in one launch (blockIdx.z), RY rows and 512 pixels per block.
template <typename Word, int CSW, int CSH, int RY>
__global__ void __launch_bounds__(128, 4) k_census4(const uint8_t* __restrict__ img_l, const uint8_t* __restrict__ img_r,
                                                 Word* __restrict__ cs_l, Word* __restrict__ cs_r, int W, int H) {
  __shared__ uint32_t tile[census4_tile_words<CSH, RY>()];
  const bool right = blockIdx.z == 1;
  census4_tile<Word, CSW, CSH, RY>(right ? img_r : img_l, right ? cs_r : cs_l, W, H, right, blockIdx.x * 512,
                                   blockIdx.y * RY, tile);
}

// ---------------------------------------------------------------------------------------------
// Recurrence step shared by every plain scan (reference cusgm_ca.cu:1517-1564 and its 32/128
// twins): L_p(d) = C_p(d) + min(L_q(d), L_q(d-1)+P1, L_q(d+1)+P1, m_q+P2) - m_q, uint32,
// with 127 as the candidate beyond d = 0 and d = D-1. Returns the new warp-wide minimum.
// ---------------------------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ uint32_t plain_step(uint32_t (&L)[K], const uint32_t (&c)[K], uint32_t m, uint32_t p1,
                                               uint32_t p2, int lane) {
  const uint32_t left_nb = __shfl_up_sync(kFull, L[K - 1], 1);
  const uint32_t right_nb = __shfl_down_sync(kFull, L[0], 1);
  const uint32_t l4 = m + p2;
  uint32_t nl[K];
  uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const uint32_t a = j > 0 ? L[j - 1] + p1 : (lane > 0 ? left_nb + p1 : kInvalidCost);
    const uint32_t b = j < K - 1 ? L[j + 1] + p1 : (lane < 31 ? right_nb + p1 : kInvalidCost);
    const uint32_t t = min(min(min(L[j], a), b), l4);
    nl[j] = c[j] + (t - m);
    mn = min(mn, nl[j]);
  }
#pragma unroll
  for (int j = 0; j < K; ++j) L[j] = nl[j];
  return __reduce_min_sync(kFull, mn);
}

template <int K>
__device__ __forceinline__ void store_u8(uint8_t* p, const uint32_t (&v)[K]) {
  if constexpr (K == 1) {
    *p = (uint8_t)v[0];
  } else if constexpr (K == 2) {
    *reinterpret_cast<uint16_t*>(p) = (uint16_t)((v[0] & 0xFFu) | ((v[1] & 0xFFu) << 8));
  } else if constexpr (K == 4) {
    *reinterpret_cast<uint32_t*>(p) = (v[0] & 0xFFu) | ((v[1] & 0xFFu) << 8) | ((v[2] & 0xFFu) << 16) | (v[3] << 24);
  } else {
    uint2 w;
    w.x = (v[0] & 0xFFu) | ((v[1] & 0xFFu) << 8) | ((v[2] & 0xFFu) << 16) | (v[3] << 24);
    w.y = (v[4] & 0xFFu) | ((v[5] & 0xFFu) << 8) | ((v[6] & 0xFFu) << 16) | (v[7] << 24);
    *reinterpret_cast<uint2*>(p) = w;
  }
}

// K bytes read through L2 (ld.global.cg): for data other warps of the same kernel write
// (adjacent columns share cache lines, so the read-only path could hold a stale line).
template <int K>
__device__ __forceinline__ void load_u8_cg(const uint8_t* p, uint32_t (&v)[K]) {
  if constexpr (K == 1) {
    v[0] = __ldcg(p);
  } else if constexpr (K == 2) {
    const uint32_t w = __ldcg(reinterpret_cast<const uint16_t*>(p));
    v[0] = w & 0xFFu;
    v[1] = w >> 8;
  } else if constexpr (K == 4) {
    const uint32_t w = __ldcg(reinterpret_cast<const uint32_t*>(p));
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = (w >> (8 * j)) & 0xFFu;
  } else {
    const uint2 w = __ldcg(reinterpret_cast<const uint2*>(p));
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      v[j] = (w.x >> (8 * j)) & 0xFFu;
      v[4 + j] = (w.y >> (8 * j)) & 0xFFu;
    }
  }
}

template <int K>
__device__ __forceinline__ void load_u8(const uint8_t* p, uint32_t (&v)[K]) {
  if constexpr (K == 1) {
    v[0] = __ldg(p);
  } else if constexpr (K == 2) {
    const uint32_t w = __ldg(reinterpret_cast<const uint16_t*>(p));
    v[0] = w & 0xFFu;
    v[1] = w >> 8;
  } else if constexpr (K == 4) {
    const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(p));
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = (w >> (8 * j)) & 0xFFu;
  } else {
    const uint2 w = __ldg(reinterpret_cast<const uint2*>(p));
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      v[j] = (w.x >> (8 * j)) & 0xFFu;
      v[4 + j] = (w.y >> (8 * j)) & 0xFFu;
    }
  }
}

struct PlainParams {
  int W, H;
  int min_d;   // minimum disparity
  int x0;      // first column of every scan, max(0, min_d)
  uint32_t p1, p2;
  size_t vstride;  // elements between the views of a volume (H*W*D)
};

// ---------------------------------------------------------------------------------------------
// Horizontal scans (left->right and right->left) of the plain path, with the Hamming cost
// computed on the fly from census rows staged in shared memory.
// Reference: Kernel_CostCompute cusgm_cc.cu:118-172/238-293 and
// Kernel_Aggregate_Horizontal_Warpfor{32,64,128} cusgm_ca.cu:1343-1770.
// One CTA = R rows x 2 directions (2R warps). The left->right warp also stores the cost volume.
// View 0: C(x,d) = popc(cl[x] ^ cr[x-min_d-d]); view 1: C(x,d) = popc(cr[x] ^ cl[x+min_d+d]);
// an out-of-range partner index reads element 0 of the partner row. With 5x5 census the
// reference's right-to-left cost kernel leaves the last pixel of every D-pixel block holding
// the left-to-right cost (cusgm_cc.cu:288); view 1 reproduces that.
// ---------------------------------------------------------------------------------------------
template <int K, typename Word>
__global__ void __launch_bounds__(256) k_hpaths_plain(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                                      uint8_t* __restrict__ cost, uint8_t* __restrict__ lr,
                                                      uint8_t* __restrict__ rl, PlainParams P) {
  constexpr int D = 32 * K;
  const int view = blockIdx.y;
  const int lane = threadIdx.x;
  const int wid = threadIdx.y;
  const int R = blockDim.y >> 1;
  const int row = wid >> 1;
  const int dir = wid & 1;
  const int y = blockIdx.x * R + row;
  const int W = P.W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Word* own = reinterpret_cast<Word*>(smem_raw) + (size_t)row * 2 * W;
  Word* oth = own + W;
  if (y < P.H) {
    const Word* g_own = (view == 0 ? cs_l : cs_r) + (size_t)y * W;
    const Word* g_oth = (view == 0 ? cs_r : cs_l) + (size_t)y * W;
    for (int i = dir * 32 + lane; i < W; i += 64) {
      own[i] = g_own[i];
      oth[i] = g_oth[i];
    }
  }
  __syncthreads();
  if (y >= P.H) return;
  const int x0 = P.x0;
  const int len = W - x0;
  if (len <= 0) return;
  const size_t vo = (size_t)view * P.vstride;
  uint8_t* out = (dir == 0 ? lr : rl) + vo;
  uint8_t* cvol = cost + vo;
  const int dbase = lane * K;
  const bool stale5 = (view == 1) && (sizeof(Word) == 4);
  uint32_t L[K];
  uint32_t m = 0;
  for (int s = 0; s < len; ++s) {
    const int x = dir == 0 ? x0 + s : W - 1 - s;
    uint32_t c[K];
    bool lr_cost = false;
    if (stale5) {
      const int blk = x0 + ((x - x0) / D) * D;
      const int iend = min(D, W - blk);
      lr_cost = (x == blk + iend - 1);
    }
    if (!lr_cost) {
      const Word a = own[x];
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const int d = dbase + j;
        const int pos = view == 0 ? x - P.min_d - d : x + P.min_d + d;
        c[j] = popc_word((Word)(a ^ ((pos >= 0 && pos < W) ? oth[pos] : oth[0])));
      }
    } else {  // view 1, 5x5: left-to-right cost of this pixel (own = right census, oth = left census)
      const Word a = oth[x];
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const int pos = x - P.min_d - (dbase + j);
        c[j] = popc_word((Word)(a ^ ((pos >= 0 && pos < W) ? own[pos] : own[0])));
      }
    }
    const size_t off = ((size_t)y * W + x) * D + dbase;
    if (s == 0) {
      uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
      for (int j = 0; j < K; ++j) {
        L[j] = c[j];
        mn = min(mn, c[j]);
      }
      m = __reduce_min_sync(kFull, mn);
    } else {
      m = plain_step<K>(L, c, m, P.p1, P.p2, lane);
    }
    store_u8<K>(out + off, L);
    if (dir == 0) store_u8<K>(cvol + off, c);
  }
}

// ---------------------------------------------------------------------------------------------
// Horizontal scans, second form. Each warp walks its row in chunks of 32 pixels:
//   1. the census words the chunk needs (32 own words and the D+31 partner words, out-of-range
//      partners replaced by element 0 of the row) are staged in the warp's shared window;
//   2. every lane computes the D costs of one pixel of the chunk (off the serial chain);
//   3. the 32 recurrence steps read their costs from shared memory;
//   4. the chunk's path costs (and, for the left-to-right warp, its costs) leave with coalesced
//      16-byte stores.
// Same results as k_hpaths_plain (reference kernels listed there). Shared memory per warp:
// window (D+64 words) + cost chunk (32 x (D+4) bytes) + path chunk (32 x D bytes).
// ---------------------------------------------------------------------------------------------
template <int K, typename Word>
__host__ __device__ constexpr size_t hpaths2_warp_smem() {
  return (size_t)(32 * K + 64) * sizeof(Word) + 32 * (32 * K + 4) + 32 * (32 * K);
}

// One scanline (view, y) in one direction (dir 0: left->right, 1: right->left), by one warp;
// `base` is the warp's hpaths2_warp_smem<K, Word>() bytes of shared memory (16-byte aligned).
template <int K, typename Word>
__device__ __forceinline__ void hpaths2_warp(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                             uint8_t* __restrict__ cost, uint8_t* __restrict__ lr,
                                             uint8_t* __restrict__ rl, const PlainParams& P, int view, int y, int dir,
                                             unsigned char* base) {
  constexpr int D = 32 * K;
  constexpr int CST = D + 4;  // padded row stride of the cost chunk (bank-conflict free prologue)
  const int lane = threadIdx.x & 31;
  const int W = P.W;
  Word* win = reinterpret_cast<Word*>(base);                   // [D + 64]: own[32], partner[D + 31]
  uint8_t* cbuf = base + (size_t)(D + 64) * sizeof(Word);      // [32][CST]
  uint8_t* pbuf = cbuf + 32 * CST;                             // [32][D]
  const int x0 = P.x0;
  const int len = W - x0;
  if (len <= 0) return;
  const size_t vo = (size_t)view * P.vstride;
  const Word* g_own = (view == 0 ? cs_l : cs_r) + (size_t)y * W;
  const Word* g_oth = (view == 0 ? cs_r : cs_l) + (size_t)y * W;
  const Word oth0 = g_oth[0];
  uint8_t* out = (dir == 0 ? lr : rl) + vo + (size_t)y * W * D;
  uint8_t* cout = cost + vo + (size_t)y * W * D;
  const bool stale5 = (view == 1) && (sizeof(Word) == 4);
  const Word own0 = g_own[0];
  uint32_t L[K];
  uint32_t m = 0;
  const int nchunks = (len + 31) >> 5;
  for (int c = 0; c < nchunks; ++c) {
    const int s0 = c << 5;
    const int n = min(32, len - s0);
    const int xa = dir == 0 ? x0 + s0 : W - (s0 + n);  // lowest pixel of the chunk
    // 1. census window
    const int ws = view == 0 ? xa - P.min_d - (D - 1) : xa + P.min_d;
    __syncwarp();
    for (int i = lane; i < D + 31; i += 32) {
      const int pos = ws + i;
      win[32 + i] = (pos >= 0 && pos < W) ? g_oth[pos] : oth0;
    }
    win[lane] = lane < n ? g_own[xa + lane] : (Word)0;
    __syncwarp();
    // 2. costs of pixel xa + lane for every d
    if (lane < n) {
      const int x = xa + lane;
      const Word a = win[lane];
      bool lr_cost = false;
      if (stale5) {
        const int blk = x0 + ((x - x0) / D) * D;
        lr_cost = (x == blk + min(D, W - blk) - 1);
      }
      uint32_t* crow = reinterpret_cast<uint32_t*>(cbuf + lane * CST);
#pragma unroll 4
      for (int d4 = 0; d4 < D; d4 += 4) {
        uint32_t packed = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int d = d4 + q;
          Word partner;
          if (!lr_cost) {
            // view 0: pos = x - min_d - d -> window index (x - xa) + (D - 1) - d
            // view 1: pos = x + min_d + d -> window index (x - xa) + d
            partner = win[32 + (view == 0 ? lane + (D - 1) - d : lane + d)];
          } else {  // 5x5 right view: this pixel keeps its left-to-right cost
            const int pos = x - P.min_d - d;
            partner = (pos >= 0 && pos < W) ? g_own[pos] : own0;
          }
          const Word own_word = lr_cost ? g_oth[x] : a;
          packed |= popc_word((Word)(own_word ^ partner)) << (8 * q);
        }
        crow[d4 >> 2] = packed;
      }
    }
    __syncwarp();
    // 3. recurrence over the chunk
    for (int i = 0; i < n; ++i) {
      const int s = s0 + i;
      const int px = dir == 0 ? i : n - 1 - i;  // buffer row of this step's pixel
      const uint8_t* cr = cbuf + px * CST + lane * K;
      uint32_t cv[K];
#pragma unroll
      for (int j = 0; j < K; ++j) cv[j] = cr[j];
      if (s == 0) {
        uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < K; ++j) {
          L[j] = cv[j];
          mn = min(mn, cv[j]);
        }
        m = __reduce_min_sync(kFull, mn);
      } else {
        m = plain_step<K>(L, cv, m, P.p1, P.p2, lane);
      }
      store_u8<K>(pbuf + px * D + lane * K, L);
    }
    __syncwarp();
    // 4. write the chunk: n pixels x D bytes contiguous in both volumes
    const int bytes = n * D;
    uint8_t* og = out + (size_t)xa * D;
    for (int b = lane * 16; b < bytes; b += 32 * 16)
      *reinterpret_cast<uint4*>(og + b) = *reinterpret_cast<const uint4*>(pbuf + b);
    if (dir == 0) {  // costs: 4-byte words (the padded chunk rows are only 4-byte aligned)
      uint32_t* cg = reinterpret_cast<uint32_t*>(cout + (size_t)xa * D);
      const uint32_t* cb = reinterpret_cast<const uint32_t*>(cbuf);
      for (int w = lane; w < bytes / 4; w += 32) {
        const int row = w / (D / 4), col = w - row * (D / 4);
        cg[w] = cb[row * (CST / 4) + col];
      }
    }
  }
  __syncwarp();
}

template <int K, typename Word>
__global__ void __launch_bounds__(256) k_hpaths_plain2(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                                       uint8_t* __restrict__ cost, uint8_t* __restrict__ lr,
                                                       uint8_t* __restrict__ rl, PlainParams P) {
  const int wid = threadIdx.y;
  const int R = blockDim.y >> 1;
  const int y = blockIdx.x * R + (wid >> 1);
  if (y >= P.H) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  hpaths2_warp<K, Word>(cs_l, cs_r, cost, lr, rl, P, blockIdx.y, y, wid & 1,
                        smem_raw + (size_t)wid * hpaths2_warp_smem<K, Word>());
}

struct WtaParams {
  float uniqueness;
  int tie_rule;
  int rows;        // rows the reference's WTA launch covers
  int dmax_excl;   // d* must be < dmax_excl (D for the warp kernels, D-1 for the generic one)
  size_t dstride;  // elements between the views of the disparity maps (H*W)
  // Pixels the thread-per-scanline WTA may make valid: x in [xlo, xhi], y in [ylo, yhi], in the
  // launch's coordinates. The reference's border (x < 5, y < 5, x > W-5, y > H-5 INVALID,
  // cusgm_ca.cu:3630) is in image coordinates; a region of interest scanned as its own sub-image
  // starting at (gx, gy) shifts it.
  int xlo, xhi, ylo, yhi;
  __host__ __device__ void image_border(int W, int H, int gx = 0, int gy = 0) {
    xlo = 5 - gx;
    xhi = W - 5 - gx;
    ylo = 5 - gy;
    yhi = H - 5 - gy;
  }
};

// Winner-take-all + uniqueness + subpixel on the summed path costs of one pixel.
// Reference Kernel_ComputeDisparityByWTA_Warpfor{32,64,128} cusgm_ca.cu:3514-3809 and the
// generic kernel :3149-3232. Returns the disparity (valid in every lane).
template <int K>
__device__ __forceinline__ float wta_pixel(const uint32_t (&S)[K], int lane, int min_d_or_base, const WtaParams& Q,
                                           int dmin_excl, int y) {
  constexpr int D = 32 * K;
  uint32_t lm = S[0];
#pragma unroll
  for (int j = 1; j < K; ++j) lm = min(lm, S[j]);
  const uint32_t m = __reduce_min_sync(kFull, lm);
  uint32_t bal[K];
#pragma unroll
  for (int j = 0; j < K; ++j) bal[j] = __ballot_sync(kFull, S[j] == m);
  const int ds = pick_tie<K>(bal, Q.tie_rule, y);
  // neighbours of d*: S(d*-1) and S(d*+1) live in lanes (d*-1)/K and (d*+1)/K
  const int dl = ds - 1 < 0 ? 0 : ds - 1;
  const int dr = ds + 1 >= D ? D - 1 : ds + 1;
  uint32_t vl = S[0], vr = S[0];
#pragma unroll
  for (int j = 1; j < K; ++j) {
    if ((dl % K) == j) vl = S[j];
    if ((dr % K) == j) vr = S[j];
  }
  const uint32_t s1 = __shfl_sync(kFull, vl, dl / K);
  const uint32_t s3 = __shfl_sync(kFull, vr, dr / K);
  if (ds <= dmin_excl || ds >= Q.dmax_excl) return kInvalidFloat;
  const float c1 = (float)s1;
  const float c2 = (float)m;
  const float c3 = (ds + 1 < D) ? (float)s3 : (float)ds;
  const float d12 = __fsub_rn(c1, c2), d32 = __fsub_rn(c3, c2);
  const float uq = d12 < d32 ? d12 : d32;
  if (uq <= __fmul_rn(c2, __fsub_rn(1.0f, Q.uniqueness))) return kInvalidFloat;
  return __fadd_rn((float)(ds + min_d_or_base), subpix_bias(c1, c2, c3));
}

// WTA at an initial-disparity level under the reference's measured behaviour (every tied lane
// stores its own result, cusgm_ca.cu:3488-3509): the lowest tied lane with a valid disparity wins.
__device__ __forceinline__ float wta_pixel_init_ref(uint32_t S, int lane, int base, const WtaParams& Q) {
  const uint32_t m = __reduce_min_sync(kFull, S);
  const uint32_t c1u = __shfl_up_sync(kFull, S, 1);
  const uint32_t c3u = __shfl_down_sync(kFull, S, 1);
  float v = kInvalidFloat;
  if (S == m && lane > 1 && lane < kLevelRange - 1) {
    const float c1 = (float)c1u, c2 = (float)m, c3 = (float)c3u;
    const float d12 = __fsub_rn(c1, c2), d32 = __fsub_rn(c3, c2);
    const float uq = d12 < d32 ? d12 : d32;
    if (!(uq <= __fmul_rn(c2, __fsub_rn(1.0f, Q.uniqueness))))
      v = __fadd_rn((float)(lane + base), subpix_bias(c1, c2, c3));
  }
  const uint32_t ok = __ballot_sync(kFull, v != kInvalidFloat);
  return __shfl_sync(kFull, v, ok ? __ffs(ok) - 1 : 0);
}

// ---------------------------------------------------------------------------------------------
// Vertical scans (bottom->top, then top->bottom) fused with the 4-path sum and the WTA.
// Reference Kernel_Aggregate_Vertical_Warpfor{32,64,128} cusgm_ca.cu:1410-1888 and the WTA
// kernels above. One warp per column; 8 columns per CTA. Columns left of x0 are INVALID.
// ---------------------------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void vpaths1_warp(const uint8_t* __restrict__ cost, const uint8_t* __restrict__ lr,
                                             const uint8_t* __restrict__ rl, uint8_t* __restrict__ bt,
                                             float* __restrict__ disp, const PlainParams& P, const WtaParams& Q,
                                             int view, int x) {
  constexpr int D = 32 * K;
  const int lane = threadIdx.x & 31;
  const int W = P.W, H = P.H;
  float* dout = disp + (size_t)view * Q.dstride;
  if (x < P.x0) {
    for (int y = lane; y < H; y += 32) dout[(size_t)y * W + x] = kInvalidFloat;
    return;
  }
  const size_t vo = (size_t)view * P.vstride;
  const uint8_t* cv = cost + vo;
  uint8_t* btv = bt + vo;
  const int dbase = lane * K;
  uint32_t L[K], c[K];
  uint32_t m = 0;
  // bottom -> top
  for (int s = 0; s < H; ++s) {
    const int y = H - 1 - s;
    const size_t off = ((size_t)y * W + x) * D + dbase;
    load_u8<K>(cv + off, c);
    if (s == 0) {
      uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
      for (int j = 0; j < K; ++j) { L[j] = c[j]; mn = min(mn, c[j]); }
      m = __reduce_min_sync(kFull, mn);
    } else {
      m = plain_step<K>(L, c, m, P.p1, P.p2, lane);
    }
    store_u8<K>(btv + off, L);
  }
  __syncwarp();
  // top -> bottom, summing the four paths and selecting the disparity
  const uint8_t* lrv = lr + vo;
  const uint8_t* rlv = rl + vo;
  const bool col_ok = x >= 5 && x <= W - 5;
  for (int y = 0; y < H; ++y) {
    const size_t off = ((size_t)y * W + x) * D + dbase;
    load_u8<K>(cv + off, c);
    if (y == 0) {
      uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
      for (int j = 0; j < K; ++j) { L[j] = c[j]; mn = min(mn, c[j]); }
      m = __reduce_min_sync(kFull, mn);
    } else {
      m = plain_step<K>(L, c, m, P.p1, P.p2, lane);
    }
    float dv = kInvalidFloat;
    if (col_ok && y >= 5 && y <= H - 5 && y < Q.rows) {
      uint32_t a[K], b[K], e[K], S[K];
      load_u8_cg<K>(btv + off, a);
      load_u8<K>(lrv + off, b);
      load_u8<K>(rlv + off, e);
#pragma unroll
      for (int j = 0; j < K; ++j) S[j] = (L[j] & 0xFFu) + a[j] + b[j] + e[j];
      dv = wta_pixel<K>(S, lane, P.min_d, Q, 0, y);
    }
    if (lane == 0) dout[(size_t)y * W + x] = dv;
  }
  __syncwarp();
}

template <int K>
__global__ void __launch_bounds__(256) k_vpaths_wta_plain(const uint8_t* __restrict__ cost,
                                                          const uint8_t* __restrict__ lr,
                                                          const uint8_t* __restrict__ rl, uint8_t* __restrict__ bt,
                                                          float* __restrict__ disp, PlainParams P, WtaParams Q) {
  const int x = blockIdx.x * blockDim.y + threadIdx.y;
  if (x >= P.W) return;
  vpaths1_warp<K>(cost, lr, rl, bt, disp, P, Q, blockIdx.y, x);
}

// Packed K bytes of one lane (K disparities) as loaded from a [..][D] u8 volume.
template <int K> struct PackOf { using T = uint32_t; };
template <> struct PackOf<8> { using T = uint2; };

template <int K>
__device__ __forceinline__ typename PackOf<K>::T ld_pack_cg(const uint8_t* p) {
  if constexpr (K == 1) return __ldcg(p);
  else if constexpr (K == 2) return __ldcg(reinterpret_cast<const uint16_t*>(p));
  else if constexpr (K == 4) return __ldcg(reinterpret_cast<const uint32_t*>(p));
  else return __ldcg(reinterpret_cast<const uint2*>(p));
}

template <int K>
__device__ __forceinline__ typename PackOf<K>::T ld_pack(const uint8_t* p) {
  if constexpr (K == 1) return __ldg(p);
  else if constexpr (K == 2) return __ldg(reinterpret_cast<const uint16_t*>(p));
  else if constexpr (K == 4) return __ldg(reinterpret_cast<const uint32_t*>(p));
  else return __ldg(reinterpret_cast<const uint2*>(p));
}

// The same K bytes read from shared memory with an access of exactly their size (the address
// is aligned to K bytes only).
template <int K>
__device__ __forceinline__ typename PackOf<K>::T ld_pack_shared(const uint8_t* p) {
  if constexpr (K == 1) return *p;
  else if constexpr (K == 2) return *reinterpret_cast<const uint16_t*>(p);
  else if constexpr (K == 4) return *reinterpret_cast<const uint32_t*>(p);
  else return *reinterpret_cast<const uint2*>(p);
}

template <int K>
__device__ __forceinline__ void unpack(const typename PackOf<K>::T& w, uint32_t (&v)[K]) {
  if constexpr (K == 8) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      v[j] = (w.x >> (8 * j)) & 0xFFu;
      v[4 + j] = (w.y >> (8 * j)) & 0xFFu;
    }
  } else {
#pragma unroll
    for (int j = 0; j < K; ++j) v[j] = (w >> (8 * j)) & 0xFFu;
  }
}

// ---------------------------------------------------------------------------------------------
// Vertical scans + WTA, second form: the per-row loads of the serial chain come from a
// PF-deep register ring filled PF rows ahead, and the bottom->top path costs of the CTA's
// columns stay in shared memory (bt_smem) when H*C*D fits, so the top->bottom pass reads them
// without a global round trip. One warp per column, C = blockDim.y columns per CTA.
// Same results as k_vpaths_wta_plain (reference kernels listed there).
// ---------------------------------------------------------------------------------------------
// One column (view, x) by one warp. bt_col: this column's H x D bytes of shared memory for the
// bottom->top path costs, or nullptr to keep them in the global volume bt.
template <int K, int PF>
__device__ __forceinline__ void vpaths2_warp(const uint8_t* __restrict__ cost, const uint8_t* __restrict__ lr,
                                             const uint8_t* __restrict__ rl, uint8_t* __restrict__ bt,
                                             float* __restrict__ disp, const PlainParams& P, const WtaParams& Q,
                                             int view, int x, uint8_t* bt_col) {
  using Pk = typename PackOf<K>::T;
  constexpr int D = 32 * K;
  const int lane = threadIdx.x & 31;
  const int W = P.W, H = P.H;
  const bool bt_smem = bt_col != nullptr;
  float* dout = disp + (size_t)view * Q.dstride;
  if (x < P.x0) {
    for (int y = lane; y < H; y += 32) dout[(size_t)y * W + x] = kInvalidFloat;
    return;
  }
  const size_t vo = (size_t)view * P.vstride;
  const uint8_t* cv = cost + vo + (size_t)x * D + lane * K;
  const uint8_t* lrv = lr + vo + (size_t)x * D + lane * K;
  const uint8_t* rlv = rl + vo + (size_t)x * D + lane * K;
  const size_t rs = (size_t)W * D;  // row stride of a volume
  uint8_t* btp;
  size_t bts;
  if (bt_smem) {
    btp = bt_col + lane * K;
    bts = D;
  } else {
    btp = bt + vo + (size_t)x * D + lane * K;
    bts = rs;
  }
  uint32_t L[K], c[K];
  uint32_t m = 0;
  // bottom -> top
  Pk ring[PF];
#pragma unroll
  for (int i = 0; i < PF; ++i) {
    const int y = H - 1 - i;
    if (y >= 0) ring[i] = ld_pack<K>(cv + (size_t)y * rs);
  }
  for (int s0 = 0; s0 < H; s0 += PF) {
#pragma unroll
    for (int i = 0; i < PF; ++i) {
      const int s = s0 + i;
      if (s < H) {
        const int y = H - 1 - s;
        unpack<K>(ring[i], c);
        if (s + PF < H) ring[i] = ld_pack<K>(cv + (size_t)(y - PF) * rs);
        if (s == 0) {
          uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
          for (int j = 0; j < K; ++j) { L[j] = c[j]; mn = min(mn, c[j]); }
          m = __reduce_min_sync(kFull, mn);
        } else {
          m = plain_step<K>(L, c, m, P.p1, P.p2, lane);
        }
        store_u8<K>(btp + (size_t)y * bts, L);
      }
    }
  }
  __syncwarp();
  // top -> bottom + sum + WTA (the bottom->top costs join the ring when they live in global memory)
  Pk rc[PF], ra[PF], rb[PF], re[PF];
#pragma unroll
  for (int i = 0; i < PF; ++i) {
    if (i < H) {
      rc[i] = ld_pack<K>(cv + (size_t)i * rs);
      ra[i] = ld_pack<K>(lrv + (size_t)i * rs);
      rb[i] = ld_pack<K>(rlv + (size_t)i * rs);
      if (!bt_smem) re[i] = ld_pack_cg<K>(btp + (size_t)i * bts);
    }
  }
  const bool col_ok = x >= 5 && x <= W - 5;
  for (int y0 = 0; y0 < H; y0 += PF) {
#pragma unroll
    for (int i = 0; i < PF; ++i) {
      const int y = y0 + i;
      if (y < H) {
        uint32_t a[K], b[K], e[K];
        unpack<K>(rc[i], c);
        unpack<K>(ra[i], a);
        unpack<K>(rb[i], b);
        if (!bt_smem) unpack<K>(re[i], e);
        if (y + PF < H) {
          rc[i] = ld_pack<K>(cv + (size_t)(y + PF) * rs);
          ra[i] = ld_pack<K>(lrv + (size_t)(y + PF) * rs);
          rb[i] = ld_pack<K>(rlv + (size_t)(y + PF) * rs);
          if (!bt_smem) re[i] = ld_pack_cg<K>(btp + (size_t)(y + PF) * bts);
        }
        if (y == 0) {
          uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
          for (int j = 0; j < K; ++j) { L[j] = c[j]; mn = min(mn, c[j]); }
          m = __reduce_min_sync(kFull, mn);
        } else {
          m = plain_step<K>(L, c, m, P.p1, P.p2, lane);
        }
        float dv = kInvalidFloat;
        if (col_ok && y >= 5 && y <= H - 5 && y < Q.rows) {
          uint32_t S[K];
          if (bt_smem) unpack<K>(ld_pack_shared<K>(btp + (size_t)y * bts), e);
#pragma unroll
          for (int j = 0; j < K; ++j) S[j] = (L[j] & 0xFFu) + e[j] + a[j] + b[j];
          dv = wta_pixel<K>(S, lane, P.min_d, Q, 0, y);
        }
        if (lane == 0) dout[(size_t)y * W + x] = dv;
      }
    }
  }
}

template <int K, int PF>
__global__ void __launch_bounds__(256) k_vpaths_wta_plain2(const uint8_t* __restrict__ cost,
                                                           const uint8_t* __restrict__ lr,
                                                           const uint8_t* __restrict__ rl, uint8_t* __restrict__ bt,
                                                           float* __restrict__ disp, PlainParams P, WtaParams Q,
                                                           int bt_smem) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int x = blockIdx.x * blockDim.y + threadIdx.y;
  if (x >= P.W) return;
  vpaths2_warp<K, PF>(cost, lr, rl, bt, disp, P, Q, blockIdx.y, x,
                      bt_smem ? smem_raw + (size_t)threadIdx.y * P.H * (32 * K) : nullptr);
}

// ---------------------------------------------------------------------------------------------
// Initial-disparity (pyramid) levels, D = 32: cost with CostAdjust and the per-pixel offset,
// recurrence realigned by base - last_base (reference cusgm_cc.cu:173-237/294-360,
// cusgm_ca.cu:1181-1338). All arithmetic uint32 as in the reference.
// ---------------------------------------------------------------------------------------------
struct InitParams {
  int W, H, x0;
  uint32_t p1;
  int32_t p1s, p2s, p2_div0;
  uint32_t invalid_cost;  // 0xFF (9x7) or 127 (5x5)
  size_t vstride;
};

// max(P1, P2 / k) for k = |last_base - base + 1|; k < kP2Tab from a shared-memory table.
constexpr int kP2Tab = 64;
__device__ __forceinline__ void fill_p2_table(uint32_t* tab, const InitParams& P, int tid, int nthreads) {
  for (int k = tid; k < kP2Tab; k += nthreads) {
    const int32_t q = k ? P.p2s / k : P.p2_div0;
    tab[k] = (uint32_t)(P.p1s > q ? P.p1s : q);
  }
}
__device__ __forceinline__ uint32_t p2_term(const uint32_t* tab, int k, const InitParams& P) {
  if (k < kP2Tab) return tab[k];
  if (P.p2s >= 0 && k > P.p2s) return (uint32_t)(P.p1s > 0 ? P.p1s : 0);  // P2 / k == 0
  const int32_t q = P.p2s / k;
  return (uint32_t)(P.p1s > q ? P.p1s : q);
}

// One realigned step. Returns the new minimum; L is replaced.
__device__ __forceinline__ uint32_t init_step(uint32_t& L, uint32_t c, uint32_t m, int base, int last_base, int lane,
                                              const InitParams& P, const uint32_t* p2tab) {
  const int i1 = lane + base - 1 - last_base;
  const int i2 = lane + base + 1 - last_base;
  const uint32_t v1 = __shfl_sync(kFull, L, i1 & 31);
  const uint32_t v2 = __shfl_sync(kFull, L, i2 & 31);
  const uint32_t a = (i1 >= 0 && i1 < kLevelRange) ? v1 + P.p1 : kInvalidCost;
  const uint32_t b = (i2 >= 0 && i2 < kLevelRange) ? v2 + P.p1 : kInvalidCost;
  const uint32_t l4 = m + p2_term(p2tab, abs(last_base - base + 1), P);
  const uint32_t t = min(min(min(L, a), b), l4);
  L = c + (t - m);
  return __reduce_min_sync(kFull, L);
}

template <typename Word>
__device__ __forceinline__ uint32_t init_cost(const Word* own, const Word* oth, int x, int d, int base, int W,
                                              int view, uint32_t invalid_cost, uint32_t adj) {
  if (view == 0) {
    const int pos = x - d - base;
    return (pos > 0 && pos < W) ? ((popc_word((Word)(own[x] ^ oth[pos])) + adj) & 0xFFu) : invalid_cost;
  }
  const int pos = x + d + base;
  return (popc_word((Word)(own[x] ^ ((pos > 0 && pos < W) ? oth[pos] : oth[0]))) + adj) & 0xFFu;
}

template <typename Word>
__global__ void __launch_bounds__(256) k_hpaths_init(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                                     const int16_t* __restrict__ init_l,
                                                     const int16_t* __restrict__ init_r, uint8_t* __restrict__ cost,
                                                     uint8_t* __restrict__ lr, uint8_t* __restrict__ rl, InitParams P) {
  constexpr int D = kLevelRange;
  const int view = blockIdx.y;
  const int lane = threadIdx.x;
  const int wid = threadIdx.y;
  const int R = blockDim.y >> 1;
  const int row = wid >> 1;
  const int dir = wid & 1;
  const int y = blockIdx.x * R + row;
  const int W = P.W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Word* own = reinterpret_cast<Word*>(smem_raw) + (size_t)row * 2 * W;
  Word* oth = own + W;
  int16_t* ibase = reinterpret_cast<int16_t*>(reinterpret_cast<Word*>(smem_raw) + (size_t)R * 2 * W) + (size_t)row * W;
  __shared__ uint32_t p2tab[kP2Tab];
  fill_p2_table(p2tab, P, threadIdx.y * 32 + lane, blockDim.x * blockDim.y);
  if (y < P.H) {
    const Word* g_own = (view == 0 ? cs_l : cs_r) + (size_t)y * W;
    const Word* g_oth = (view == 0 ? cs_r : cs_l) + (size_t)y * W;
    const int16_t* g_init = (view == 0 ? init_l : init_r) + (size_t)y * W;
    for (int i = dir * 32 + lane; i < W; i += 64) {
      own[i] = g_own[i];
      oth[i] = g_oth[i];
      ibase[i] = g_init[i];
    }
  }
  __syncthreads();
  if (y >= P.H) return;
  const int len = W - P.x0;
  if (len <= 0) return;
  const size_t vo = (size_t)view * P.vstride;
  uint8_t* out = (dir == 0 ? lr : rl) + vo;
  uint8_t* cvol = cost + vo;
  uint32_t L = 0, m = 0;
  int last_base = 0;
  const uint32_t adj = cost_adjust(lane);
  for (int s = 0; s < len; ++s) {
    const int x = dir == 0 ? P.x0 + s : W - 1 - s;
    const int base = ibase[x];
    const uint32_t c = init_cost<Word>(own, oth, x, lane, base, W, view, P.invalid_cost, adj);
    const size_t off = ((size_t)y * W + x) * D + lane;
    if (dir == 0) cvol[off] = (uint8_t)c;
    if (s == 0) {
      L = c;
      m = __reduce_min_sync(kFull, c);
      last_base = base;
      out[off] = (uint8_t)L;
      continue;
    }
    if (base == kInvalidShort) {
      m = kInvalidCost;
      continue;
    }
    m = init_step(L, c, m, base, last_base, lane, P, p2tab);
    last_base = base;
    out[off] = (uint8_t)L;
  }
}

// Horizontal scans at initial-disparity levels, second form: as k_hpaths_init, with the costs of
// 32 pixels computed per chunk by a prologue (lane = pixel) and the chunk's path costs and costs
// written with coalesced stores. Census rows and bases of the CTA's rows are staged whole (each
// pixel's partner window depends on its own base). Pixels skipped for an INVALID base leave
// unspecified bytes in the path volumes; nothing reads them (the WTA rejects those pixels first).
constexpr int kInitCst = kLevelRange + 4;  // padded cost-chunk row stride
__host__ __device__ constexpr size_t hinit2_warp_smem() { return 32 * kInitCst + 32 * kLevelRange; }

template <typename Word>
__global__ void __launch_bounds__(256) k_hpaths_init2(const Word* __restrict__ cs_l, const Word* __restrict__ cs_r,
                                                      const int16_t* __restrict__ init_l,
                                                      const int16_t* __restrict__ init_r, uint8_t* __restrict__ cost,
                                                      uint8_t* __restrict__ lr, uint8_t* __restrict__ rl,
                                                      InitParams P) {
  constexpr int D = kLevelRange;
  const int view = blockIdx.y;
  const int lane = threadIdx.x;
  const int wid = threadIdx.y;
  const int R = blockDim.y >> 1;
  const int row = wid >> 1;
  const int dir = wid & 1;
  const int y = blockIdx.x * R + row;
  const int W = P.W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t p2tab[kP2Tab];
  fill_p2_table(p2tab, P, wid * 32 + lane, blockDim.x * blockDim.y);
  // each staged row (own words, partner words, bases) starts on a 16-byte boundary
  const size_t row_bytes = ((size_t)W * (2 * sizeof(Word) + 2) + 15) & ~size_t(15);
  const size_t rows_bytes = (size_t)R * row_bytes;
  Word* own = reinterpret_cast<Word*>(smem_raw + (size_t)row * row_bytes);
  Word* oth = own + W;
  int16_t* ibase = reinterpret_cast<int16_t*>(oth + W);
  uint8_t* cbuf = smem_raw + rows_bytes + (size_t)wid * hinit2_warp_smem();
  uint8_t* pbuf = cbuf + 32 * kInitCst;
  if (y < P.H) {
    const Word* g_own = (view == 0 ? cs_l : cs_r) + (size_t)y * W;
    const Word* g_oth = (view == 0 ? cs_r : cs_l) + (size_t)y * W;
    const int16_t* g_init = (view == 0 ? init_l : init_r) + (size_t)y * W;
    for (int i = dir * 32 + lane; i < W; i += 64) {
      own[i] = g_own[i];
      oth[i] = g_oth[i];
      ibase[i] = g_init[i];
    }
  }
  __syncthreads();
  if (y >= P.H) return;
  const int len = W - P.x0;
  if (len <= 0) return;
  const size_t vo = (size_t)view * P.vstride;
  uint8_t* out = (dir == 0 ? lr : rl) + vo + (size_t)y * W * D;
  uint8_t* cout = cost + vo + (size_t)y * W * D;
  uint32_t L = 0, m = 0;
  int last_base = 0;
  const int nchunks = (len + 31) >> 5;
  for (int c = 0; c < nchunks; ++c) {
    const int s0 = c << 5;
    const int n = min(32, len - s0);
    const int xa = dir == 0 ? P.x0 + s0 : W - (s0 + n);
    __syncwarp();
    if (lane < n) {  // costs of pixel xa + lane
      const int x = xa + lane;
      const int bx = ibase[x];
      uint32_t* crow = reinterpret_cast<uint32_t*>(cbuf + lane * kInitCst);
#pragma unroll
      for (int d4 = 0; d4 < D; d4 += 4) {
        uint32_t packed = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          packed |= init_cost<Word>(own, oth, x, d4 + q, bx, W, view, P.invalid_cost, cost_adjust(d4 + q)) << (8 * q);
        crow[d4 >> 2] = packed;
      }
    }
    __syncwarp();
    for (int i = 0; i < n; ++i) {
      const int s = s0 + i;
      const int px = dir == 0 ? i : n - 1 - i;
      const int x = xa + px;
      const int base = ibase[x];
      const uint32_t cv = cbuf[px * kInitCst + lane];
      if (s == 0) {
        L = cv;
        m = __reduce_min_sync(kFull, cv);
        last_base = base;
      } else if (base == kInvalidShort) {
        m = kInvalidCost;
        continue;
      } else {
        m = init_step(L, cv, m, base, last_base, lane, P, p2tab);
        last_base = base;
      }
      pbuf[px * D + lane] = (uint8_t)L;
    }
    __syncwarp();
    const int bytes = n * D;
    uint8_t* og = out + (size_t)xa * D;
    for (int b = lane * 16; b < bytes; b += 32 * 16)
      *reinterpret_cast<uint4*>(og + b) = *reinterpret_cast<const uint4*>(pbuf + b);
    if (dir == 0) {
      uint32_t* cg = reinterpret_cast<uint32_t*>(cout + (size_t)xa * D);
      const uint32_t* cb = reinterpret_cast<const uint32_t*>(cbuf);
      for (int w = lane; w < bytes / 4; w += 32) {
        const int r2 = w / (D / 4), col = w - r2 * (D / 4);
        cg[w] = cb[r2 * (kInitCst / 4) + col];
      }
    }
  }
}

// Vertical scans + WTA at initial-disparity levels (reference cusgm_ca.cu:1263-1338 and
// Kernel_ComputeDisparityByWTA_Warpfor32 with init, :3425-3512). Both vertical scans start
// last_base from row 0 (:1291). disp = d* + base + bias; d* <= 1 or d* >= 31 -> INVALID.
static __global__ void __launch_bounds__(256) k_vpaths_wta_init(const uint8_t* __restrict__ cost,
                                                         const uint8_t* __restrict__ lr,
                                                         const uint8_t* __restrict__ rl,
                                                         const int16_t* __restrict__ init_l,
                                                         const int16_t* __restrict__ init_r, uint8_t* __restrict__ bt,
                                                         float* __restrict__ disp, InitParams P, WtaParams Q) {
  constexpr int D = kLevelRange;
  const int view = blockIdx.y;
  const int lane = threadIdx.x;
  const int x = blockIdx.x * blockDim.y + threadIdx.y;
  const int W = P.W, H = P.H;
  if (x >= W) return;
  float* dout = disp + (size_t)view * Q.dstride;
  if (x < P.x0) {
    for (int y = lane; y < H; y += 32) dout[(size_t)y * W + x] = kInvalidFloat;
    return;
  }
  __shared__ uint32_t p2tab[kP2Tab];
  for (int k = lane; k < kP2Tab; k += 32) {
    const int32_t q = k ? P.p2s / k : P.p2_div0;
    p2tab[k] = (uint32_t)(P.p1s > q ? P.p1s : q);
  }
  __syncwarp();
  const int16_t* ib = view == 0 ? init_l : init_r;
  const size_t vo = (size_t)view * P.vstride;
  const uint8_t* cv = cost + vo;
  uint8_t* btv = bt + vo;
  uint32_t L = 0, m = 0;
  int last_base = ib[x];  // row 0 for both directions
  for (int s = 0; s < H; ++s) {
    const int y = H - 1 - s;
    const size_t off = ((size_t)y * W + x) * D + lane;
    const uint32_t c = cv[off];
    if (s == 0) {
      L = c;
      m = __reduce_min_sync(kFull, c);
      btv[off] = (uint8_t)L;
      continue;
    }
    const int base = ib[(size_t)y * W + x];
    if (base == kInvalidShort) { m = kInvalidCost; continue; }
    m = init_step(L, c, m, base, last_base, lane, P, p2tab);
    last_base = base;
    btv[off] = (uint8_t)L;
  }
  __syncwarp();
  const uint8_t* lrv = lr + vo;
  const uint8_t* rlv = rl + vo;
  const bool col_ok = x >= 5 && x <= W - 5;
  last_base = ib[x];
  for (int y = 0; y < H; ++y) {
    const size_t off = ((size_t)y * W + x) * D + lane;
    const uint32_t c = cv[off];
    const int base = ib[(size_t)y * W + x];
    bool skipped = false;
    if (y == 0) {
      L = c;
      m = __reduce_min_sync(kFull, c);
    } else if (base == kInvalidShort) {
      m = kInvalidCost;
      skipped = true;
    } else {
      m = init_step(L, c, m, base, last_base, lane, P, p2tab);
      last_base = base;
    }
    float dv = kInvalidFloat;
    if (col_ok && y >= 5 && y <= H - 5 && y < Q.rows && base != kInvalidShort && !skipped) {
      uint32_t S[1];
      S[0] = (L & 0xFFu) + __ldcg(btv + off) + lrv[off] + rlv[off];
      dv = Q.tie_rule == kTieRefB200 ? wta_pixel_init_ref(S[0], lane, base, Q) : wta_pixel<1>(S, lane, base, Q, 1, y);
    }
    if (lane == 0) dout[(size_t)y * W + x] = dv;
  }
}

// Vertical scans + WTA at initial-disparity levels, second form (prefetch ring, bottom->top
// path costs in shared memory); same results as k_vpaths_wta_init.
template <int PF>
__global__ void __launch_bounds__(256) k_vpaths_wta_init2(const uint8_t* __restrict__ cost,
                                                          const uint8_t* __restrict__ lr,
                                                          const uint8_t* __restrict__ rl,
                                                          const int16_t* __restrict__ init_l,
                                                          const int16_t* __restrict__ init_r,
                                                          uint8_t* __restrict__ bt, float* __restrict__ disp,
                                                          InitParams P, WtaParams Q, int bt_smem) {
  constexpr int D = kLevelRange;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t p2tab[kP2Tab];
  fill_p2_table(p2tab, P, threadIdx.y * 32 + threadIdx.x, blockDim.x * blockDim.y);
  __syncthreads();
  const int view = blockIdx.y;
  const int lane = threadIdx.x;
  const int x = blockIdx.x * blockDim.y + threadIdx.y;
  const int W = P.W, H = P.H;
  if (x >= W) return;
  float* dout = disp + (size_t)view * Q.dstride;
  if (x < P.x0) {
    for (int y = lane; y < H; y += 32) dout[(size_t)y * W + x] = kInvalidFloat;
    return;
  }
  const int16_t* ib = (view == 0 ? init_l : init_r) + x;
  const size_t vo = (size_t)view * P.vstride;
  const size_t rs = (size_t)W * D;
  const uint8_t* cv = cost + vo + (size_t)x * D + lane;
  const uint8_t* lrv = lr + vo + (size_t)x * D + lane;
  const uint8_t* rlv = rl + vo + (size_t)x * D + lane;
  uint8_t* btp;
  size_t bts;
  if (bt_smem) {
    btp = smem_raw + (size_t)threadIdx.y * H * D + lane;
    bts = D;
  } else {
    btp = bt + vo + (size_t)x * D + lane;
    bts = rs;
  }
  uint32_t L = 0, m = 0;
  int last_base = ib[0];  // row 0 for both directions
  uint32_t rc[PF];
  int rbase[PF];
#pragma unroll
  for (int i = 0; i < PF; ++i) {
    const int y = H - 1 - i;
    if (y >= 0) {
      rc[i] = __ldg(cv + (size_t)y * rs);
      rbase[i] = ib[(size_t)y * W];
    }
  }
  for (int s0 = 0; s0 < H; s0 += PF) {
#pragma unroll
    for (int i = 0; i < PF; ++i) {
      const int s = s0 + i;
      if (s < H) {
        const int y = H - 1 - s;
        const uint32_t c = rc[i];
        const int base = rbase[i];
        if (s + PF < H) {
          rc[i] = __ldg(cv + (size_t)(y - PF) * rs);
          rbase[i] = ib[(size_t)(y - PF) * W];
        }
        if (s == 0) {
          L = c;
          m = __reduce_min_sync(kFull, c);
          btp[(size_t)y * bts] = (uint8_t)L;
        } else if (base == kInvalidShort) {
          m = kInvalidCost;
        } else {
          m = init_step(L, c, m, base, last_base, lane, P, p2tab);
          last_base = base;
          btp[(size_t)y * bts] = (uint8_t)L;
        }
      }
    }
  }
  __syncwarp();
  const bool col_ok = x >= 5 && x <= W - 5;
  last_base = ib[0];
  uint32_t ra[PF], rb[PF], re[PF];
#pragma unroll
  for (int i = 0; i < PF; ++i) {
    if (i < H) {
      rc[i] = __ldg(cv + (size_t)i * rs);
      ra[i] = __ldg(lrv + (size_t)i * rs);
      rb[i] = __ldg(rlv + (size_t)i * rs);
      re[i] = bt_smem ? 0u : (uint32_t)__ldcg(btp + (size_t)i * bts);
      rbase[i] = ib[(size_t)i * W];
    }
  }
  for (int y0 = 0; y0 < H; y0 += PF) {
#pragma unroll
    for (int i = 0; i < PF; ++i) {
      const int y = y0 + i;
      if (y < H) {
        const uint32_t c = rc[i], a = ra[i], b = rb[i];
        const uint32_t e = bt_smem ? (uint32_t)btp[(size_t)y * bts] : re[i];
        const int base = rbase[i];
        if (y + PF < H) {
          rc[i] = __ldg(cv + (size_t)(y + PF) * rs);
          ra[i] = __ldg(lrv + (size_t)(y + PF) * rs);
          rb[i] = __ldg(rlv + (size_t)(y + PF) * rs);
          if (!bt_smem) re[i] = __ldcg(btp + (size_t)(y + PF) * bts);
          rbase[i] = ib[(size_t)(y + PF) * W];
        }
        bool skipped = false;
        if (y == 0) {
          L = c;
          m = __reduce_min_sync(kFull, c);
        } else if (base == kInvalidShort) {
          m = kInvalidCost;
          skipped = true;
        } else {
          m = init_step(L, c, m, base, last_base, lane, P, p2tab);
          last_base = base;
        }
        float dv = kInvalidFloat;
        if (col_ok && y >= 5 && y <= H - 5 && y < Q.rows && base != kInvalidShort && !skipped) {
          uint32_t S[1];
          S[0] = (L & 0xFFu) + e + a + b;
          dv = Q.tie_rule == kTieRefB200 ? wta_pixel_init_ref(S[0], lane, base, Q)
                                         : wta_pixel<1>(S, lane, base, Q, 1, y);
        }
        if (lane == 0) dout[(size_t)y * W + x] = dv;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Left-right check (reference Kernel_LRCheck cusgm_ca.cu:3873-3898) and 3x3 median
// (cusgm_df.cu:16-75, launch :346-355), fused: a 32x8 output tile stages the LR-checked
// left map with a one-pixel halo in shared memory, then takes the median. The right map
// is read from a snapshot; failed pixels mark INVALID in dr_out (idempotent stores).
// Median rows 1..ylim (ylim = min(H-2, 2*ceil((W-2)/2))) and columns 1..W-2.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float lr_value(float dl, int x, const float* __restrict__ dr_row, float* dr_out_row, int W,
                                          float thr) {
  if (dl == kInvalidFloat) return dl;
  const float xrf = __fsub_rn((float)x, dl);
  const int xr = xrf > 0.0f ? (int)__dadd_rn((double)xrf, 0.5) : (int)__dsub_rn((double)xrf, 0.5);
  if (xr < 0 || xr >= W) return kInvalidFloat;
  const float dr = dr_row[xr];
  if (fabsf(__fsub_rn(dl, dr)) > thr) {
    if (dr_out_row) dr_out_row[xr] = kInvalidFloat;
    return kInvalidFloat;
  }
  return __fdiv_rn(__fadd_rn(dl, dr), 2.0f);
}

__device__ __forceinline__ void cswap(float& a, float& b) {
  const float lo = fminf(a, b), hi = fmaxf(a, b);
  a = lo;
  b = hi;
}

__device__ __forceinline__ float median9(float a0, float a1, float a2, float a3, float a4, float a5, float a6,
                                         float a7, float a8) {
  // 19 compare-exchanges selecting the middle of 9 (Paeth's median-of-9 network);
  // disparity values are never NaN, so min/max equal the reference's compare-and-swap.
  cswap(a1, a2); cswap(a4, a5); cswap(a7, a8);
  cswap(a0, a1); cswap(a3, a4); cswap(a6, a7);
  cswap(a1, a2); cswap(a4, a5); cswap(a7, a8);
  cswap(a0, a3); cswap(a5, a8); cswap(a4, a7);
  cswap(a3, a6); cswap(a1, a4); cswap(a2, a5);
  cswap(a4, a7); cswap(a4, a2); cswap(a6, a4);
  cswap(a4, a2);
  return a4;
}

// One 32x8 output tile at (bx, by) by a 32x8 block; every thread of the block calls it.
template <bool DoLR, bool DoMedian>
__device__ __forceinline__ void lr_median_tile(const float* __restrict__ dl, const float* __restrict__ dr,
                                               float* __restrict__ dr_out, float* __restrict__ out, int W, int H,
                                               float thr, int bx, int by, float (*tile)[34]) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int i = ty * 32 + tx; i < 10 * 34; i += 256) {
    const int ly = i / 34, lx = i - ly * 34;
    const int gx = bx + lx - 1, gy = by + ly - 1;
    float v = kInvalidFloat;
    if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
      v = dl[(size_t)gy * W + gx];
      if (DoLR) {
        const bool own = lx >= 1 && lx <= 32 && ly >= 1 && ly <= 8;  // marks only from the tile's own pixels
        v = lr_value(v, gx, dr + (size_t)gy * W, (own && dr_out) ? dr_out + (size_t)gy * W : nullptr, W, thr);
      }
    }
    tile[ly][lx] = v;
  }
  __syncthreads();
  const int x = bx + tx, y = by + ty;
  if (x >= W || y >= H) return;
  float v = tile[ty + 1][tx + 1];
  if (DoMedian) {
    int ylim = 2 * ((W - 1) / 2);
    ylim = ylim > H - 2 ? H - 2 : ylim;
    if (x >= 1 && x <= W - 2 && y >= 1 && y <= ylim) {
      v = median9(tile[ty][tx], tile[ty][tx + 1], tile[ty][tx + 2], tile[ty + 1][tx], tile[ty + 1][tx + 1],
                  tile[ty + 1][tx + 2], tile[ty + 2][tx], tile[ty + 2][tx + 1], tile[ty + 2][tx + 2]);
    }
  }
  out[(size_t)y * W + x] = v;
}

template <bool DoLR, bool DoMedian>
__global__ void __launch_bounds__(256) k_lr_median(const float* __restrict__ dl, const float* __restrict__ dr,
                                                   float* __restrict__ dr_out, float* __restrict__ out, int W, int H,
                                                   float thr) {
  __shared__ float tile[10][34];
  lr_median_tile<DoLR, DoMedian>(dl, dr, dr_out, out, W, H, thr, blockIdx.x * 32, blockIdx.y * 8, tile);
}

// Dilation of INVALID pixels (reference Kernel_Dilation, cusgm_df.cu:197-222).
template <typename T>
__device__ __forceinline__ void dilation_px(const T* __restrict__ in, T* __restrict__ out, int W, int H, int wth,
                                            int x, int y) {
  T v = in[(size_t)y * W + x];
  if ((float)v == kInvalidFloat || (float)v == (float)kInvalidShort) {
    if (x > wth && x < W - wth && y > wth && y < H - wth) {
      for (int dx = -wth; dx <= wth; ++dx)
        for (int dy = -wth; dy <= wth; ++dy) {
          const T u = in[(size_t)(y + dy) * W + x + dx];
          if (u > v) v = u;
        }
    }
  }
  out[(size_t)y * W + x] = v;
}

// Erosion (reference Kernel_Erosion, cusgm_df.cu:165-195): an interior pixel whose window
// holds an INVALID value becomes INVALID, every other pixel keeps its value.
__device__ __forceinline__ void erosion_px(const float* __restrict__ in, float* __restrict__ out, int W, int H,
                                           int wth, int x, int y) {
  const float v = in[(size_t)y * W + x];
  float mn = v;
  if (x > wth && x < W - wth && y > wth && y < H - wth) {
    for (int dx = -wth; dx <= wth; ++dx)
      for (int dy = -wth; dy <= wth; ++dy) {
        const float u = in[(size_t)(y + dy) * W + x + dx];
        if (u < mn) mn = u;
      }
  }
  out[(size_t)y * W + x] = mn == kInvalidFloat ? mn : v;
}

static __global__ void __launch_bounds__(256) k_erosion(const float* __restrict__ in, float* __restrict__ out, int W,
                                                        int H, int wth) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  erosion_px(in, out, W, H, wth, x, y);
}

// Range-limited Gaussian smoothing of the disparity (reference Kernel_GaussFilter,
// cusgm_df.cu:93-121, called with sigmaD 1.5 and sigmaR 2.0): weights exp(-(dx^2+dy^2)/(2 sD^2))
// over a (2*ceil(2 sD)+1)^2 window of valid neighbours within sR of the centre.
__device__ __forceinline__ void gauss_px(const float* __restrict__ in, float* __restrict__ out, int W, int H,
                                         float sigma_d, float sigma_r, int x, int y) {
  const int r = (int)ceil(2.0 * sigma_d);
  float result = kInvalidFloat;
  float sum = 0.0f, sum_w = 0.0f;
  const float c = in[(size_t)y * W + x];
  if (c != kInvalidFloat) {
    for (int m = x - r; m <= x + r; ++m)
      for (int n = y - r; n <= y + r; ++n)
        if (m >= 0 && n >= 0 && m < W && n < H) {
          const float v = in[(size_t)n * W + m];
          if (v != kInvalidFloat && fabsf(c - v) < sigma_r) {
            const int dx = m - x, dy = n - y;
            const float w = expf(-((dx * dx + dy * dy) / (2.0f * sigma_d * sigma_d)));
            sum_w += w;
            sum += w * v;
          }
        }
  }
  if (sum_w > 0.0f) result = sum / sum_w;
  out[(size_t)y * W + x] = result;
}

static __global__ void __launch_bounds__(256) k_gauss_filter(const float* __restrict__ in, float* __restrict__ out,
                                                             int W, int H, float sigma_d, float sigma_r) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  gauss_px(in, out, W, H, sigma_d, sigma_r, x, y);
}

// Bilateral smoothing guided by the left image (reference Kernel_BilateralFilter,
// cusgm_df.cu:123-162, called with sigmaD 2.5 and sigmaR 10.0): the spatial weight times
// exp(-g^2/(2 sR^2)) of the grey difference g (evaluated in double, as there), for valid
// neighbours with |g| < sR.
static __global__ void __launch_bounds__(256) k_bilateral_filter(const uint8_t* __restrict__ img,
                                                                 const float* __restrict__ in, float* __restrict__ out,
                                                                 int W, int H, float sigma_d, float sigma_r) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const int r = (int)ceil(2.0 * sigma_d);
  float result = kInvalidFloat;
  float sum = 0.0f, sum_w = 0.0f;
  const float c = in[(size_t)y * W + x];
  const uint8_t gc = img[(size_t)y * W + x];
  if (c != kInvalidFloat) {
    for (int m = x - r; m <= x + r; ++m)
      for (int n = y - r; n <= y + r; ++n)
        if (m >= 0 && n >= 0 && m < W && n < H) {
          const float v = in[(size_t)n * W + m];
          const uint8_t g = img[(size_t)n * W + m];
          if (v != kInvalidFloat && fabsf(float(g - gc)) < sigma_r) {
            const int dx = m - x, dy = n - y;
            const float dist = (float)(g - gc);
            const float wd = expf(-((dx * dx + dy * dy) / (2.0f * sigma_d * sigma_d)));
            const float wr = (float)exp(-(dist * dist) / (2.0 * sigma_r * sigma_r));
            const float w = wd * wr;
            sum_w += w;
            sum += w * v;
          }
        }
    if (sum_w > 0.0f) result = sum / sum_w;
  }
  out[(size_t)y * W + x] = result;
}

template <typename T>
__global__ void __launch_bounds__(256) k_dilation(const T* __restrict__ in, T* __restrict__ out, int W, int H,
                                                  int wth) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  dilation_px<T>(in, out, W, H, wth, x, y);
}

// ---------------------------------------------------------------------------------------------
// Small-region removal (reference StereoCudaImpl.cpp:32-125, 463-498) as connected-component
// labelling: union-find over 4-neighbours within a strip, roots = smallest pixel index.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool peaks_adjacent(float a, float b, int abs_mode) {
  const float d = __fsub_rn(a, b);
  if (abs_mode == kPeaksAbsFloat) return fabsf(d) <= 1.0f;
  const int t = (int)d;  // truncation toward zero, as int abs((int)x) in the g++ build
  return (t < 0 ? -t : t) <= 1;
}

// Root of p. Reads go to L2 (ld.global.cg): parents are rewritten by atomics from other SMs.
__device__ __forceinline__ int cc_find(const int* label, int p) {
  int q = __ldcg(label + p);
  while (q != p) {
    p = q;
    q = __ldcg(label + p);
  }
  return p;
}

// Row pass: label[i] = first pixel of i's horizontal run of connected pixels (its provisional
// root), -1 for INVALID pixels and rows >= `rows`; zeroes count. One warp per row, 32 pixels per
// step: run starts by ballot, the run of the previous step carried across.
__device__ __forceinline__ void cc_rows_warp(const float* __restrict__ disp, int* __restrict__ label,
                                             int* __restrict__ count, int W, int H, int rows, int abs_mode, int y) {
  const int lane = threadIdx.x & 31;
  const float* drow = disp + (size_t)y * W;
  int* lrow = label + (size_t)y * W;
  int* crow = count + (size_t)y * W;
  int carry = -1;
  float prev_v = kInvalidFloat;
  bool prev_valid = false;
  for (int x0 = 0; x0 < W; x0 += 32) {
    const int x = x0 + lane;
    const bool in = x < W;
    const float v = in ? drow[x] : kInvalidFloat;
    const bool valid = in && y < rows && v != kInvalidFloat;
    float lv = __shfl_up_sync(kFull, v, 1);
    bool lvalid = __shfl_up_sync(kFull, (int)valid, 1) != 0;
    if (lane == 0) {
      lv = prev_v;
      lvalid = prev_valid;
    }
    const bool conn = valid && lvalid && peaks_adjacent(v, lv, abs_mode);
    const unsigned brk = __ballot_sync(kFull, !conn);
    const unsigned upto = brk & (0xFFFFFFFFu >> (31 - lane));
    const int start = upto ? x0 + (31 - __clz(upto)) : carry;
    if (in) {
      lrow[x] = valid ? y * W + start : -1;
      crow[x] = 0;
    }
    carry = __shfl_sync(kFull, start, 31);
    prev_v = __shfl_sync(kFull, v, 31);
    prev_valid = __shfl_sync(kFull, (int)valid, 31) != 0;
  }
}

static __global__ void k_cc_rows(const float* __restrict__ disp, int* __restrict__ label, int* __restrict__ count,
                                 int W, int H, int rows, int abs_mode) {
  const int y = blockIdx.x * blockDim.y + threadIdx.y;
  if (y >= H) return;
  cc_rows_warp(disp, label, count, W, H, rows, abs_mode, y);
}

// Vertical pass: unions pixel i with the pixel below it (same strip) when both are valid and
// adjacent; roots are the smallest pixel index (atomicMin hooks the larger root).
__device__ __forceinline__ void cc_vert_px(const float* __restrict__ disp, int* label, int W, int H, int tiles,
                                           int rows, int abs_mode, int i) {
  const int y = i / W;
  if (y + 1 >= rows || (y + 1) / tiles != y / tiles) return;
  const int q = i + W;
  const float v = disp[i], w = disp[q];
  if (v == kInvalidFloat || w == kInvalidFloat || !peaks_adjacent(w, v, abs_mode)) return;
  int a = i, b = q;
  while (true) {
    a = cc_find(label, a);
    b = cc_find(label, b);
    if (a == b) break;
    if (a > b) { const int t = a; a = b; b = t; }
    const int old = atomicMin(&label[b], a);
    if (old == b) break;
    b = old;
  }
}

static __global__ void k_cc_vert(const float* __restrict__ disp, int* label, int W, int H, int tiles, int rows,
                                 int abs_mode) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W * H) return;
  cc_vert_px(disp, label, W, H, tiles, rows, abs_mode, i);
}

__device__ __forceinline__ void cc_count_px(int* label, int* __restrict__ count, int i) {
  if (label[i] < 0) return;
  const int r = cc_find(label, i);
  label[i] = r;
  atomicAdd(&count[r], 1);
}

// every processed strip has exactly `tiles` rows, so the threshold is the same for all of them
__device__ __forceinline__ void cc_filter_px(float* __restrict__ disp, const int* __restrict__ label,
                                             const int* __restrict__ count, int W, int tiles, float ratio, int i) {
  if (label[i] < 0) return;
  const int threshold = (int)__fmul_rn((float)(W * tiles), ratio);
  if (count[label[i]] < threshold) disp[i] = kInvalidFloat;
}

static __global__ void k_cc_count(int* label, int* __restrict__ count, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  cc_count_px(label, count, i);
}
static __global__ void k_cc_filter(float* __restrict__ disp, const int* __restrict__ label, const int* __restrict__ count,
                                   int W, int H, int tiles, float ratio) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W * H) return;
  cc_filter_px(disp, label, count, W, tiles, ratio, i);
}

// ---------------------------------------------------------------------------------------------
// Pyramid helpers (reference FasterStereoCuda.cpp:114-166, cusgm_util.cu:47-59).
// ---------------------------------------------------------------------------------------------
// Level image = full-resolution image sampled at (x << shift, y << shift); both views.
__device__ __forceinline__ void decimate_px(const uint8_t* __restrict__ full_l, const uint8_t* __restrict__ full_r,
                                            uint8_t* __restrict__ lvl_l, uint8_t* __restrict__ lvl_r, int W0, int w,
                                            int shift, int x, int y) {
  const size_t src = ((size_t)y << shift) * W0 + ((size_t)x << shift);
  lvl_l[(size_t)y * w + x] = full_l[src];
  lvl_r[(size_t)y * w + x] = full_r[src];
}
static __global__ void k_decimate(const uint8_t* __restrict__ full_l, const uint8_t* __restrict__ full_r,
                                  uint8_t* __restrict__ lvl_l, uint8_t* __restrict__ lvl_r, int W0, int w, int h,
                                  int shift) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= w || y >= h) return;
  decimate_px(full_l, full_r, lvl_l, lvl_r, W0, w, shift, x, y);
}

// Initial disparity of the next finer level: even rows (except the last) from cur at the flat
// index (y/2)*(width/2) + x/2 (INVALID past the end of cur); odd rows and the last row copy the
// row above.
__device__ __forceinline__ void init_next_px(const float* __restrict__ cur, long ncur, int16_t* __restrict__ next,
                                             int width, int height, int x, int y) {
  int ys = y;
  if (y % 2 == 1 || y == height - 1) ys = y - 1;
  if (ys % 2 == 1) ys -= 1;  // last row with an even index copies an odd row, whose source is one more up
  if (ys < 0) {
    next[(size_t)y * width + x] = kInvalidShort;
    return;
  }
  const long idx = (long)(ys >> 1) * (width >> 1) + (x >> 1);
  const float d = idx < ncur ? cur[idx] : kInvalidFloat;
  next[(size_t)y * width + x] =
      d != kInvalidFloat ? (int16_t)(int)__fsub_rn(__fmul_rn(2.0f, d), (float)(kLevelRange >> 1)) : kInvalidShort;
}
static __global__ void k_init_next_level(const float* __restrict__ cur, long ncur, int16_t* __restrict__ next, int width,
                                         int height) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= width || y >= height) return;
  init_next_px(cur, ncur, next, width, height, x, y);
}

// Right-view initial disparities: cleared to INVALID, then a scatter in which the largest
// source x wins for every target (the reference's concurrent scatter made deterministic).
static __global__ void k_right_init_scatter(const int16_t* __restrict__ init_l, unsigned* __restrict__ key, int W, int H) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const int16_t xl = (int16_t)x;
  const int16_t il = (int16_t)(init_l[(size_t)y * W + x] + (kLevelRange >> 1));
  const int t = xl - il;
  if (t > 0 && t < W) {
    const int16_t val = (int16_t)(il - (kLevelRange >> 1));
    atomicMax(&key[(size_t)y * W + t], ((unsigned)(x + 1) << 16) | (uint16_t)val);
  }
}

static __global__ void k_right_init_decode(const unsigned* __restrict__ key, int16_t* __restrict__ out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned k = key[i];
  out[i] = k == 0 ? kInvalidShort : (int16_t)(uint16_t)(k & 0xFFFFu);
}

// Disparity -> depth (reference Kernel_ComputeDepth, cusgm_util.cu:7-34):
// depth = baseline*focus / (d + x0_right - x0_left) in double, INVALID kept.
static __global__ void k_depth(const float* __restrict__ disp, float* __restrict__ depth, int n, double f1, double f2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float d = disp[i];
  depth[i] = d == kInvalidFloat ? kInvalidFloat : (float)__ddiv_rn(f1, __dadd_rn((double)d, f2));
}

}  // namespace sgm
