// Differentiable float32 SGM: 4-path hard-min recurrence with per-pixel P1/P2 maps, summed over the
// paths, followed by a soft-argmin disparity; and its adjoint.
//
// No counterpart in the reference (it is the training/serving addition beside the bit-exact path).
// The recurrence is the reference's path recurrence (cusgm_ca.cu:1517-1564) in float with the
// penalties read at the current pixel and +inf beyond d = 0 and d = D-1:
//   L_p(d) = C_p(d) + min(L_q(d), L_q(d-1)+P1(p), L_q(d+1)+P1(p), m_q+P2(p)) - m_q,  m_q = min_k L_q(k)
//   S(p,d) = ((L_0 + L_1) + L_2) + L_3;  disp(p) = sum_d d * softmax_d(-S(p,d)/T)
// Ties of the hard minima are broken in the fixed order same d, d-1, d+1, jump (lowest k for m_q).
//
// Mapping, forward: one warp per scanline, lane l holding the K = D/32 consecutive disparities
// K l .. K l + K - 1; the per-pixel minimum is one REDUX on order-preserving 32-bit keys of the
// floats (exactly the minimum), the d +- 1 terms stay in the lane except at its edges (one shuffle
// up, one down). Inputs move in chunks of kFC steps: a row chunk is one contiguous bulk copy, a
// column chunk one box of a 3D tensor map (TMA), double-buffered on mbarriers with bounded waits;
// the penalties of a chunk's steps are loaded one chunk ahead, one step per lane. A row scan is a
// chain of W dependent steps, so everything that does not depend on the path costs is kept off it.
// Backward: a scanline is held by G lanes of a warp, K = D/G disparities per lane (8 lanes, K = 8
// at D = 64: the segment buffers fit more lines per SM), minima and sums by butterflies.
// All four directions run in ONE launch (their blocks side by side, the long row scans first),
// each writing its own path volume; the soft-argmin kernel adds the four in path order. The
// backward launch likewise runs the four adjoint scans at once, each writing its own gradient
// volume and penalty-map gradients, and a last kernel adds them in path order.
//
// Backward: per path, scanlines are walked backwards segment by segment; each segment of
// kSeg pixels is recomputed from the state stored when the forward pass entered it, so no
// D-deep path volume is kept for the backward (only one state per kSeg pixels). The adjoint
// routes the gradient of every L_p(d) to C_p(d), to P1(p) or P2(p) through the recorded minimum,
// and to L_q.
//
// Layouts: cost/sum/grad volumes float [B][H][W][D] (16-byte aligned); maps float [B][H][W];
// checkpoints float [4 paths][lines][segments][D]. Paths: 0 top->bottom, 1 left->right,
// 2 bottom->top, 3 right->left.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <type_traits>

#include "../../include/sgm_b200.h"
#include "sgm_async.cuh"
#include "sgm_tma.h"

void sgm_set_process_error(const char* msg);

namespace {

constexpr unsigned kFullMask = 0xFFFFFFFFu;
constexpr int kK = 8;       // disparities per lane of the soft-argmin kernels
constexpr int kSeg = 8;     // pixels per recomputed segment (checkpoint interval)
constexpr int kBwdPF = 2;   // depth of the backward register rings (two interleaved scans per step)
constexpr int kWarps = 4;   // warps per block of the scan kernels
constexpr int kFC = 16;     // steps per staged chunk of the forward scans (a multiple of kSeg)
// lanes per scanline of the backward scans at D = 64 and D = 32 (any choice gives the same path
// states: the per-disparity arithmetic and the exact minimum do not depend on it)
constexpr int kBwdLanes64 = 8, kBwdLanes32 = 4;
#define kInf __int_as_float(0x7f800000)

struct Geo {
  int B, H, W, D;
  int dir;
  int lines, len, nseg;
};

__host__ __device__ inline Geo make_geo(int B, int H, int W, int D, int dir) {
  Geo g;
  g.B = B; g.H = H; g.W = W; g.D = D; g.dir = dir;
  const bool horiz = dir == 1 || dir == 3;
  g.lines = horiz ? B * H : B * W;
  g.len = horiz ? W : H;
  g.nseg = (g.len + kSeg - 1) / kSeg;
  return g;
}

// pixel index (b*H + y)*W + x of scan position 0 of `line`, and the pixel stride of one step
__device__ __forceinline__ void line_origin(const Geo& g, int line, long long& base, long long& step) {
  if (g.dir == 1 || g.dir == 3) {  // line = b*H + y
    base = (long long)line * g.W + (g.dir == 3 ? g.W - 1 : 0);
    step = g.dir == 3 ? -1 : 1;
  } else {  // line = b*W + x
    const int b = line / g.W, x = line - b * g.W;
    base = ((long long)b * g.H + (g.dir == 2 ? g.H - 1 : 0)) * g.W + x;
    step = g.dir == 2 ? -(long long)g.W : (long long)g.W;
  }
}

template <int G>
__device__ __forceinline__ float group_min(float v) {
#pragma unroll
  for (int o = G / 2; o; o >>= 1) v = fminf(v, __shfl_xor_sync(kFullMask, v, o));
  return v;
}
template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
  for (int o = G / 2; o; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
  return v;
}

// minimum of K values as a balanced tree
template <int K>
__device__ __forceinline__ float minK(const float (&v)[K]) {
  float t[K];
#pragma unroll
  for (int i = 0; i < K; ++i) t[i] = v[i];
#pragma unroll
  for (int w = 1; w < K; w *= 2)
#pragma unroll
    for (int i = 0; i + w < K; i += 2 * w) t[i] = fminf(t[i], t[i + w]);
  return t[0];
}

template <int K>
__device__ __forceinline__ void loadK(const float* p, float (&v)[K]) {
#pragma unroll
  for (int h = 0; h < K / 4; ++h) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p) + h);
    v[4 * h] = a.x; v[4 * h + 1] = a.y; v[4 * h + 2] = a.z; v[4 * h + 3] = a.w;
  }
}
template <int K>
__device__ __forceinline__ void storeK(float* p, const float (&v)[K]) {
#pragma unroll
  for (int h = 0; h < K / 4; ++h)
    reinterpret_cast<float4*>(p)[h] = make_float4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
}

// Neighbours of the lane's disparities d = gl*K + j within the line's group of G lanes.
template <int G, int K>
__device__ __forceinline__ void neighbours(const float (&L)[K], int gl, float (&lm)[K], float (&lp)[K]) {
  const float left = __shfl_up_sync(kFullMask, L[K - 1], 1);
  const float right = __shfl_down_sync(kFullMask, L[0], 1);
#pragma unroll
  for (int j = 0; j < K; ++j) {
    lm[j] = j > 0 ? L[j - 1] : (gl > 0 ? left : kInf);
    lp[j] = j < K - 1 ? L[j + 1] : (gl < G - 1 ? right : kInf);
  }
}

// One forward step from the previous state Lq into L; returns the new minimum.
template <int G, int K>
__device__ __forceinline__ float fstep(const float (&Lq)[K], float (&L)[K], const float (&c)[K], float m, float p1,
                                       float p2, int gl) {
  float lm[K], lp[K];
  neighbours<G, K>(Lq, gl, lm, lp);
  const float jump = m + p2;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const float t = fminf(fminf(Lq[j], lm[j] + p1), fminf(lp[j] + p1, jump));
    L[j] = c[j] + t - m;
  }
  return group_min<G>(minK<K>(L));
}

// Blocks of the four directions side by side in one grid: slot i (direction order[i]) owns blocks
// [first_block[i], first_block[i + 1]).
struct Grid4 {
  Geo g[4];
  int order[4];
  int first_block[5];
};

struct Line {
  int dir, line;
  bool live;  // false for the padding lanes of a warp past the direction's last line
};

// The line of this thread; false if the whole warp is past the direction's lines.
template <int G>
__device__ __forceinline__ bool locate(const Grid4& q, Line& ln, Geo& g) {
  const int b = blockIdx.x;
  const int slot = (b >= q.first_block[1]) + (b >= q.first_block[2]) + (b >= q.first_block[3]);
  ln.dir = q.order[slot];
  g = q.g[ln.dir];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wline = ((b - q.first_block[slot]) * kWarps + warp) * (32 / G);
  if (wline >= g.lines) return false;
  const int mine = wline + lane / G;
  ln.live = mine < g.lines;
  ln.line = ln.live ? mine : g.lines - 1;
  return true;
}

struct FwdArgs {
  const float* cost;
  const float* p1;
  const float* p2;
  float* out[4];   // path volumes, one per direction
  float* ckpt[4];  // segment entry states, one slab per direction
  Grid4 q;         // one line per warp
};

// Order-preserving 32-bit key of a (non-NaN) float and back: the unsigned order of the keys is the
// order of the values, so a REDUX minimum of keys is exactly the minimum.
__device__ __forceinline__ uint32_t fkey(float f) {
  const uint32_t b = __float_as_uint(f);
  return b ^ ((uint32_t)((int32_t)b >> 31) | 0x80000000u);
}
__device__ __forceinline__ float funkey(uint32_t k) {
  return __uint_as_float(k ^ ((uint32_t)((int32_t)~k >> 31) | 0x80000000u));
}
__device__ __forceinline__ float warp_min(float v) { return funkey(__reduce_min_sync(kFullMask, fkey(v))); }

// One forward step of a warp-held scanline (lane l: d = K l + j), the arithmetic of fstep.
template <int K>
__device__ __forceinline__ void fstep_warp(float (&L)[K], const float (&c)[K], float& m, float p1, float p2) {
  const int lane = threadIdx.x & 31;
  const float left = __shfl_up_sync(kFullMask, L[K - 1], 1);
  const float right = __shfl_down_sync(kFullMask, L[0], 1);
  const float jump = m + p2;
  float n[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const float lm = j > 0 ? L[j - 1] : (lane > 0 ? left : kInf);
    const float lp = j < K - 1 ? L[j + 1] : (lane < 31 ? right : kInf);
    const float t = fminf(fminf(L[j], lm + p1), fminf(lp + p1, jump));
    n[j] = c[j] + t - m;
  }
#pragma unroll
  for (int j = 0; j < K; ++j) L[j] = n[j];
  m = warp_min(minK<K>(L));
}

template <int K>
__device__ __forceinline__ void ld_lane(const float* p, float (&v)[K]) {
  if constexpr (K == 2) {
    const float2 x = *reinterpret_cast<const float2*>(p);
    v[0] = x.x;
    v[1] = x.y;
  } else {
#pragma unroll
    for (int j = 0; j < K; ++j) v[j] = p[j];
  }
}
template <int K>
__device__ __forceinline__ void st_lane(float* p, const float (&v)[K]) {
  if constexpr (K == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  } else {
#pragma unroll
    for (int j = 0; j < K; ++j) p[j] = v[j];
  }
}

// Shared memory of the forward kernel: per warp two chunk buffers of kFC x D floats.
template <int K>
constexpr size_t fwd_smem_bytes() {
  return (size_t)kWarps * 2 * kFC * 32 * K * sizeof(float);
}

// tm_cost: the cost volume as a 3D tensor map (floats of a row, rows, images), boxes of D x kFC x 1.
template <int K>
__global__ void __launch_bounds__(kWarps * 32) k_float_fwd(const __grid_constant__ CUtensorMap tm_cost,
                                                           const FwdArgs a) {
  constexpr int D = 32 * K, C = kFC, NB = 2;
  extern __shared__ __align__(128) float fsm[];
  __shared__ __align__(8) uint64_t bars[kWarps][NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    for (int b = 0; b < NB; ++b) sgm::mbar_init(&bars[w][b], 1);
    sgm::mbar_fence_init();
  }
  __syncwarp();
  Line ln;
  Geo g;
  if (!locate<32>(a.q, ln, g)) return;  // the whole warp
  long long base, step;
  line_origin(g, ln.line, base, step);
  const bool horiz = g.dir == 1 || g.dir == 3;
  const bool rev = g.dir == 2 || g.dir == 3;  // step j of a chunk at buffer row C - 1 - j
  float* box0 = fsm + (size_t)w * NB * C * D;
  const int len = g.len, nch = (len + C - 1) / C;
  auto chunk_n = [&](int c) { return min(C, len - c * C); };
  auto issue = [&](int c) {  // lane 0
    const int b = c % NB, n = chunk_n(c);
    float* dst = box0 + b * C * D;
    if (horiz) {  // pixels base + (cC + j) step, contiguous; right-to-left: a short chunk at the buffer's end
      const long long lo = step > 0 ? base + (long long)c * C : base - ((long long)c * C + n - 1);
      const uint32_t bytes = (uint32_t)(n * D * sizeof(float));
      sgm::mbar_expect_tx(&bars[w][b], bytes);
      sgm::bulk_to_smem(dst + (step > 0 ? 0 : (C - n) * D), a.cost + lo * D, bytes, &bars[w][b]);
    } else {  // column x of image bi: top-to-bottom boxes start at row cC, bottom-to-top ones end at H - cC
      const int bi = ln.line / g.W, x = ln.line - bi * g.W;
      const int y0 = g.dir == 0 ? c * C : g.H - C * (c + 1);
      sgm::mbar_expect_tx(&bars[w][b], (uint32_t)(C * D * sizeof(float)));
      sgm::tma_load_3d(dst, &tm_cost, x * D, y0, bi, &bars[w][b]);
    }
  };
  // the penalties of step `lane` of chunk c
  auto pen = [&](int c, float& q1, float& q2) {
    q1 = q2 = 0.f;
    if (lane < chunk_n(c)) {
      const long long p = base + ((long long)c * C + lane) * step;
      q1 = __ldg(a.p1 + p);
      q2 = __ldg(a.p2 + p);
    }
  };
  if (lane == 0) {
    issue(0);
    if (nch > 1) issue(1);
  }
  float c1, c2, n1 = 0.f, n2 = 0.f;
  pen(0, c1, c2);
  uint32_t phase = 0u;  // bit b: parity of buffer b's next phase
  float L[K], m = 0.f;
  float* out = a.out[g.dir] + lane * K;
  float* ck = a.ckpt[g.dir] + (size_t)ln.line * g.nseg * D + lane * K;
  for (int c = 0; c < nch; ++c) {
    const int b = c % NB, n = chunk_n(c);
    pen(c + 1, n1, n2);  // a chunk ahead
    if (!sgm::mbar_wait_warp(&bars[w][b], (phase >> b) & 1u)) {
      sgm::scan_give_up_mask(bars[w], phase, (1u << b) | (c + 1 < nch ? 1u << ((c + 1) % NB) : 0u));
      return;
    }
    phase ^= 1u << b;
    __syncwarp();
    const float* bx = box0 + b * C * D + lane * K;
    float cv[C][K];
#pragma unroll
    for (int j = 0; j < C; ++j) ld_lane<K>(bx + (rev ? C - 1 - j : j) * D, cv[j]);
    sgm::fence_proxy_async();  // this lane's reads of the buffer before the copy that refills it
    __syncwarp();
    if (lane == 0 && c + 2 < nch) issue(c + 2);
    float* op = out + (base + (long long)c * C * step) * D;  // step 0 of the chunk
    const long long od = step * D;
    auto one = [&](int j) {
      const float P1 = __shfl_sync(kFullMask, c1, j), P2 = __shfl_sync(kFullMask, c2, j);
      const int s = c * C + j;
      if (j % kSeg == 0 && (j > 0 || c > 0)) st_lane<K>(ck + (size_t)(s / kSeg) * D, L);  // state entering
      if (j == 0 && c == 0) {
#pragma unroll
        for (int t = 0; t < K; ++t) L[t] = cv[0][t];
        m = warp_min(minK<K>(L));
      } else {
        fstep_warp<K>(L, cv[j], m, P1, P2);
      }
      st_lane<K>(op + j * od, L);
    };
    if (n == C) {
#pragma unroll
      for (int j = 0; j < C; ++j) one(j);
    } else {  // the last, short chunk
#pragma unroll
      for (int j = 0; j < C; ++j)
        if (j < n) one(j);
    }
    c1 = n1;
    c2 = n2;
  }
}

// S = ((L0 + L1) + L2) + L3 written over L0; disp = sum_d d softmax(-S/T)
template <int G>
__global__ void __launch_bounds__(256) k_soft_argmin_fwd(float* __restrict__ sum, const float* __restrict__ l1,
                                                         const float* __restrict__ l2, const float* __restrict__ l3,
                                                         float* __restrict__ disp, size_t npix, float inv_t) {
  constexpr int D = G * kK;
  const size_t first = ((size_t)blockIdx.x * 8 + (threadIdx.x >> 5)) * (32 / G);
  if (first >= npix) return;
  const size_t mine = first + (threadIdx.x & 31) / G;
  const bool live = mine < npix;
  const size_t p = live ? mine : npix - 1;
  const int gl = threadIdx.x % G;
  const size_t off = p * D + gl * kK;
  float S[kK], b[kK], c[kK], d[kK];
  loadK<kK>(sum + off, S);
  loadK<kK>(l1 + off, b);
  loadK<kK>(l2 + off, c);
  loadK<kK>(l3 + off, d);
#pragma unroll
  for (int j = 0; j < kK; ++j) S[j] = ((S[j] + b[j]) + c[j]) + d[j];
  if (live) storeK<kK>(sum + off, S);
  const float mn = group_min<G>(minK<kK>(S));
  float z = 0.f, num = 0.f;
#pragma unroll
  for (int j = 0; j < kK; ++j) {
    const float e = expf(-(S[j] - mn) * inv_t);
    z += e;
    num += e * (float)(gl * kK + j);
  }
  z = group_sum<G>(z);
  num = group_sum<G>(num);
  if (live && gl == 0) disp[p] = num / z;
}

// dS = -gdisp/T * w(d) * (d - disp), w = softmax(-S/T)
template <int G>
__global__ void __launch_bounds__(256) k_soft_argmin_bwd(const float* __restrict__ sum,
                                                         const float* __restrict__ gdisp, float* __restrict__ gsum,
                                                         size_t npix, float inv_t) {
  constexpr int D = G * kK;
  const size_t first = ((size_t)blockIdx.x * 8 + (threadIdx.x >> 5)) * (32 / G);
  if (first >= npix) return;
  const size_t mine = first + (threadIdx.x & 31) / G;
  const bool live = mine < npix;
  const size_t p = live ? mine : npix - 1;
  const int gl = threadIdx.x % G;
  const size_t off = p * D + gl * kK;
  float S[kK], e[kK];
  loadK<kK>(sum + off, S);
  const float mn = group_min<G>(minK<kK>(S));
  float z = 0.f, num = 0.f;
#pragma unroll
  for (int j = 0; j < kK; ++j) {
    e[j] = expf(-(S[j] - mn) * inv_t);
    z += e[j];
    num += e[j] * (float)(gl * kK + j);
  }
  z = group_sum<G>(z);
  num = group_sum<G>(num);
  const float dd = num / z;
  const float gd = __ldg(gdisp + p);
  const float scale = -gd * inv_t / z;
  float gs[kK];
#pragma unroll
  for (int j = 0; j < kK; ++j) gs[j] = scale * e[j] * ((float)(gl * kK + j) - dd);
  if (live) storeK<kK>(gsum + off, gs);
}

struct BwdArgs {
  const float* cost;
  const float* p1;
  const float* p2;
  const float* gsum;
  const float* ckpt[4];
  float* gout[4];  // gradient volumes, one per direction (written)
  float* gp1[4];   // penalty-map gradients, one per direction (written)
  float* gp2[4];
  Grid4 q;
};

// Shared memory of one line: two buffers of (kSeg + 1) states of D floats (slot 0 = state entering
// the segment), so the recompute of one segment fills one buffer while the adjoint of the segment
// after it reads the other. Each state is D/4 float4 in the order (quarter h, lane gl); a lane
// reads back only what it wrote.
template <int G, int K>
constexpr size_t bwd_smem_bytes() {
  return (size_t)kWarps * (32 / G) * 2 * (kSeg + 1) * G * K * sizeof(float);
}

template <int G, int K>
__global__ void __launch_bounds__(kWarps * 32, 3) k_float_bwd(const BwdArgs a) {
  constexpr int D = G * K, Q = D / 4, kSlots = kSeg + 1;
  extern __shared__ float4 seg_smem[];
  Line ln;
  Geo g;
  if (!locate<G>(a.q, ln, g)) return;
  const int lane = threadIdx.x & 31, gl = lane % G, grp = lane / G;
  long long base, step;
  line_origin(g, ln.line, base, step);
  float4* st = seg_smem + (size_t)((threadIdx.x >> 5) * (32 / G) + grp) * 2 * kSlots * Q;
  auto st_put = [&](int buf, int slot, const float (&v)[K]) {
#pragma unroll
    for (int h = 0; h < K / 4; ++h)
      st[(buf * kSlots + slot) * Q + h * G + gl] = make_float4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
  };
  auto st_get = [&](int buf, int slot, float (&v)[K]) {
#pragma unroll
    for (int h = 0; h < K / 4; ++h) {
      const float4 x = st[(buf * kSlots + slot) * Q + h * G + gl];
      v[4 * h] = x.x; v[4 * h + 1] = x.y; v[4 * h + 2] = x.z; v[4 * h + 3] = x.w;
    }
  };
  const float* ck = a.ckpt[ln.dir] + (size_t)ln.line * g.nseg * D + gl * K;
  float* gout = a.gout[ln.dir];
  float* gp1 = a.gp1[ln.dir];
  float* gp2 = a.gp2[ln.dir];
  float gnext[K];
#pragma unroll
  for (int j = 0; j < K; ++j) gnext[j] = 0.f;
  float LA[K], LB[K];  // recomputed states of even / odd scan positions (segment starts are even)
  float m = 0.f;
  float rc[kBwdPF][K], rp1[kBwdPF], rp2[kBwdPF];  // inputs of the recompute steps
  float rg[kBwdPF][K], rq1[kBwdPF], rq2[kBwdPF];  // inputs of the adjoint steps
  auto fetch_r = [&](int j, int s) {
    const long long p = base + s * step;
    loadK<K>(a.cost + p * D + gl * K, rc[j]);
    rp1[j] = __ldg(a.p1 + p);
    rp2[j] = __ldg(a.p2 + p);
  };
  auto fetch_a = [&](int j, int s) {
    const long long p = base + s * step;
    loadK<K>(a.gsum + p * D + gl * K, rg[j]);
    rq1[j] = __ldg(a.p1 + p);
    rq2[j] = __ldg(a.p2 + p);
  };
  // Phase ph recomputes segment kr = last - ph (while ph <= last) and, interleaved with it step
  // by step, runs the adjoint backwards through segment kr + 1 (from ph = 1 on) over the states
  // the previous phase recomputed: two independent dependency chains per step.
  const int last = g.nseg - 1;
  for (int ph = 0; ph <= last + 1; ++ph) {
    const int kr = last - ph, ka = kr + 1;
    const int r0 = kr * kSeg, nr = kr >= 0 ? min(g.len, r0 + kSeg) - r0 : 0;
    const int a0 = ka * kSeg, na = ph >= 1 ? min(g.len, a0 + kSeg) - a0 : 0;
    const int br = kr & 1, ba = ka & 1;
    if (kr > 0) {
      loadK<K>(ck + (size_t)kr * D, LB);
      st_put(br, 0, LB);
      m = group_min<G>(minK<K>(LB));
    }
#pragma unroll
    for (int j = 0; j < kBwdPF; ++j) {
      if (j < nr) fetch_r(j, r0 + j);
      if (j < na) fetch_a(j, a0 + na - 1 - j);
    }
    // one recompute step into slot 1 + i of buffer br (L(r0 + i)); one adjoint step at
    // s = a0 + na - 1 - i (last pixel first). `at_start`: the step may be the path's first pixel.
    auto r_step = [&](int jr, int i, int n, auto at_start) {
      const int s = r0 + i;
      float(&L)[K] = (jr & 1) ? LB : LA;
      float(&Lq)[K] = (jr & 1) ? LA : LB;
      float c[K];
#pragma unroll
      for (int t = 0; t < K; ++t) c[t] = rc[jr][t];
      const float P1 = rp1[jr], P2 = rp2[jr];
      if (i + kBwdPF < n) fetch_r(jr, s + kBwdPF);
      if (decltype(at_start)::value && s == 0) {
#pragma unroll
        for (int t = 0; t < K; ++t) L[t] = c[t];
        m = group_min<G>(minK<K>(L));
      } else {
        m = fstep<G, K>(Lq, L, c, m, P1, P2, gl);
      }
      st_put(br, 1 + i, L);
    };
    auto a_step = [&](int jr, int i, int n, auto at_start) {
      const int s = a0 + na - 1 - i;
      const long long p = base + s * step;
      float gv[K];
#pragma unroll
      for (int t = 0; t < K; ++t) gv[t] = rg[jr][t] + gnext[t];
      const float P1 = rq1[jr], P2 = rq2[jr];
      if (i + kBwdPF < n) fetch_a(jr, s - kBwdPF);
      if (ln.live) storeK<K>(gout + p * D + gl * K, gv);
      if (decltype(at_start)::value && s == 0) {  // the first pixel of a path adds nothing to the penalties
        if (ln.live && gl == 0) {
          gp1[p] = 0.f;
          gp2[p] = 0.f;
        }
      } else {
        // previous state L_q = L(s-1): slot (s - a0) (slot 0 = checkpoint when s == a0)
        float Lq[K];
        st_get(ba, s - a0, Lq);
        // m_q and its (lowest) index
        float mn = Lq[0];
        int mi = gl * K;
#pragma unroll
        for (int j = 1; j < K; ++j)
          if (Lq[j] < mn) { mn = Lq[j]; mi = gl * K + j; }
        const float mq = group_min<G>(mn);
        const unsigned hit = (__ballot_sync(kFullMask, mn == mq) >> (grp * G)) & ((1u << G) - 1u);
        const int kq = __shfl_sync(kFullMask, mi, grp * G + __ffs(hit) - 1);
        // choices at p
        float lm[K], lp[K];
        neighbours<G, K>(Lq, gl, lm, lp);
        const float jump = mq + P2;
        float g1 = 0.f, g2 = 0.f, gall = 0.f;
        float gsame[K], gm1[K], gp1v[K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
          float t = Lq[j];
          int c3 = 0;
          if (lm[j] + P1 < t) { t = lm[j] + P1; c3 = 1; }
          if (lp[j] + P1 < t) { t = lp[j] + P1; c3 = 2; }
          if (jump < t) { c3 = 3; }
          gsame[j] = c3 == 0 ? gv[j] : 0.f;
          gm1[j] = c3 == 1 ? gv[j] : 0.f;   // flows to L_q(d-1)
          gp1v[j] = c3 == 2 ? gv[j] : 0.f;  // flows to L_q(d+1)
          if (c3 == 1 || c3 == 2) g1 += gv[j];
          if (c3 == 3) g2 += gv[j];
          gall += gv[j];
        }
        g1 = group_sum<G>(g1);
        g2 = group_sum<G>(g2);
        gall = group_sum<G>(gall);
        if (ln.live && gl == 0) {
          gp1[p] = g1;
          gp2[p] = g2;
        }
        // gradient of L_q: same d, from d+1 choosing d-1 (i.e. d), from d-1 choosing d+1 (i.e. d)
        const float from_up = __shfl_down_sync(kFullMask, gm1[0], 1);      // gm1 of d+1, for d = gl*8+7
        const float from_down = __shfl_up_sync(kFullMask, gp1v[K - 1], 1); // gp1 of d-1, for d = gl*8
#pragma unroll
        for (int j = 0; j < K; ++j) {
          float v = gsame[j];
          v += j < K - 1 ? gm1[j + 1] : (gl < G - 1 ? from_up : 0.f);
          v += j > 0 ? gp1v[j - 1] : (gl > 0 ? from_down : 0.f);
          if (gl * K + j == kq) v += g2 - gall;
          gnext[j] = v;
        }
      }
    };
    if (kr > 0 && nr == kSeg && na == kSeg) {
      // both chains over a whole segment, away from the path's first pixel: fully unrolled, so
      // the two steps of one iteration are one block of independent instructions
#pragma unroll
      for (int i = 0; i < kSeg; ++i) {
        r_step(i % kBwdPF, i, kSeg, std::false_type{});
        a_step(i % kBwdPF, i, kSeg, std::false_type{});
      }
    } else {
      for (int i0 = 0; i0 < max(nr, na); i0 += kBwdPF) {
#pragma unroll
        for (int jr = 0; jr < kBwdPF; ++jr) {
          const int i = i0 + jr;
          if (i < nr) r_step(jr, i, nr, std::true_type{});
          if (i < na) a_step(jr, i, na, std::true_type{});
        }
      }
    }
    __syncwarp();
  }
}

// grad_cost = ((G0 + G1) + G2) + G3 in place over G0; grad_p = (((0 + a0) + a1) + a2) + a3
struct SumArgs {
  float4* g0;
  const float4* g1;
  const float4* g2;
  const float4* g3;
  size_t n4;
  float* gp1;
  float* gp2;
  const float* a1[4];
  const float* a2[4];
  size_t npix;
};

__global__ void __launch_bounds__(256) k_grad_sum(const SumArgs a) {
  const size_t n = a.n4 + a.npix;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (i < a.n4) {
      float4 x = a.g0[i];
      const float4 y = __ldg(a.g1 + i), z = __ldg(a.g2 + i), w = __ldg(a.g3 + i);
      x.x = ((x.x + y.x) + z.x) + w.x;
      x.y = ((x.y + y.y) + z.y) + w.y;
      x.z = ((x.z + y.z) + z.z) + w.z;
      x.w = ((x.w + y.w) + z.w) + w.w;
      a.g0[i] = x;
    } else {
      const size_t p = i - a.n4;
      a.gp1[p] = (((0.f + a.a1[0][p]) + a.a1[1][p]) + a.a1[2][p]) + a.a1[3][p];
      a.gp2[p] = (((0.f + a.a2[0][p]) + a.a2[1][p]) + a.a2[2][p]) + a.a2[3][p];
    }
  }
}

int check(const char* what) {
  const cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(st);
    sgm_set_process_error(m.c_str());
    return SGM_ERR_CUDA;
  }
  return SGM_OK;
}

int validate(int B, int H, int W, int D, float temperature) {
  if (B <= 0 || H <= 0 || W <= 0 || (D != 32 && D != 64)) {
    sgm_set_process_error("float SGM: B, H, W > 0 and D in {32, 64} required");
    return SGM_ERR_ARG;
  }
  if (!(temperature > 0.0f) || !std::isfinite(1.0f / temperature)) {
    sgm_set_process_error("float SGM: temperature must be > 0 with a finite reciprocal");
    return SGM_ERR_ARG;
  }
  // B*H*W*D voxels, bounded factor by factor so that no product can wrap
  const uint64_t kMaxVoxels = (uint64_t)1 << 40;
  uint64_t n = 1;
  for (const int32_t f : {B, H, W, D}) {
    if ((uint64_t)f > kMaxVoxels / n) {
      sgm_set_process_error("float SGM: volume too large");
      return SGM_ERR_ARG;
    }
    n *= (uint64_t)f;
  }
  return SGM_OK;
}

int check_present(std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs)
    if (!p) {
      sgm_set_process_error("float SGM: null device pointer");
      return SGM_ERR_ARG;
    }
  return SGM_OK;
}

int check_aligned(std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) & 15) {
      sgm_set_process_error("float SGM: cost, sum, gradient and workspace arrays must be 16-byte aligned");
      return SGM_ERR_ARG;
    }
  return SGM_OK;
}

size_t slab_elems(int B, int H, int W, int D) { return sgm_float_checkpoint_elems(B, H, W, D) / 4; }

// The four directions of one launch, row scans first (their scanlines are the longest).
template <int G>
Grid4 make_grid(int B, int H, int W, int D) {
  Grid4 q;
  const int order[4] = {1, 3, 0, 2};
  const int lines_per_block = kWarps * (32 / G);
  q.first_block[0] = 0;
  for (int i = 0; i < 4; ++i) {
    q.order[i] = order[i];
    q.g[i] = make_geo(B, H, W, D, i);  // indexed by direction
  }
  for (int i = 0; i < 4; ++i)
    q.first_block[i + 1] = q.first_block[i] + (q.g[order[i]].lines + lines_per_block - 1) / lines_per_block;
  return q;
}

// The cost volume [B][H][W][D] floats as a 3D tensor map (floats of a row, rows, images) with
// boxes of D x kFC x 1: the forward column scans' chunks.
int cost_map(const float* cost, int B, int H, int W, int D, CUtensorMap* map) {
  const sgm::EncodeTiledFn fn = sgm::encode_tiled();
  if (!fn) {
    sgm_set_process_error("float SGM: cuTensorMapEncodeTiled is not available from the driver");
    return SGM_ERR_CUDA;
  }
  const cuuint64_t dims[3] = {(cuuint64_t)W * D, (cuuint64_t)H, (cuuint64_t)B};
  const cuuint64_t strides[2] = {(cuuint64_t)W * D * sizeof(float), (cuuint64_t)H * W * D * sizeof(float)};
  const cuuint32_t box[3] = {(cuuint32_t)D, (cuuint32_t)kFC, 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(cost), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    sgm_set_process_error("float SGM: cuTensorMapEncodeTiled failed for the cost volume");
    return SGM_ERR_CUDA;
  }
  return SGM_OK;
}

template <int K>
int forward_impl(const float* cost, const float* p1, const float* p2, int B, int H, int W, float inv_t, float* sum,
                 float* ckpt, float* work, float* disp, cudaStream_t s) {
  constexpr int D = 32 * K;
  const size_t V = (size_t)B * H * W * D, npix = (size_t)B * H * W;
  FwdArgs a;
  a.cost = cost;
  a.p1 = p1;
  a.p2 = p2;
  a.out[0] = sum;
  for (int i = 1; i < 4; ++i) a.out[i] = work + (i - 1) * V;
  const size_t slab = slab_elems(B, H, W, D);
  for (int i = 0; i < 4; ++i) a.ckpt[i] = ckpt + slab * i;
  a.q = make_grid<32>(B, H, W, D);
  CUtensorMap tm;
  int st = cost_map(cost, B, H, W, D, &tm);
  if (st) return st;
  constexpr size_t smem = fwd_smem_bytes<K>();
  if (cudaFuncSetAttribute(k_float_fwd<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return check("float forward attribute");
  k_float_fwd<K><<<a.q.first_block[4], kWarps * 32, smem, s>>>(tm, a);
  st = check("float forward");
  if (st) return st;
  constexpr int GS = D / kK;  // lanes per pixel of the soft-argmin kernels
  const size_t px_per_block = 8 * (32 / GS);
  k_soft_argmin_fwd<GS><<<(unsigned)((npix + px_per_block - 1) / px_per_block), 256, 0, s>>>(
      sum, a.out[1], a.out[2], a.out[3], disp, npix, inv_t);
  return check("soft argmin");
}

template <int G, int K>
int backward_impl(const float* cost, const float* p1, const float* p2, int B, int H, int W, float inv_t,
                  const float* sum, const float* ckpt, const float* grad_disp, float* grad_sum, float* work,
                  float* grad_cost, float* grad_p1, float* grad_p2, cudaStream_t s) {
  constexpr int D = G * K;
  const size_t V = (size_t)B * H * W * D, npix = (size_t)B * H * W;
  constexpr int GS = D / kK;  // lanes per pixel of the soft-argmin kernels
  const size_t px_per_block = 8 * (32 / GS);
  k_soft_argmin_bwd<GS><<<(unsigned)((npix + px_per_block - 1) / px_per_block), 256, 0, s>>>(
      sum, grad_disp, grad_sum, npix, inv_t);
  int st = check("soft argmin backward");
  if (st) return st;
  BwdArgs a;
  a.cost = cost;
  a.p1 = p1;
  a.p2 = p2;
  a.gsum = grad_sum;
  const size_t slab = slab_elems(B, H, W, D);
  float* maps = work + 3 * V;
  for (int i = 0; i < 4; ++i) {
    a.ckpt[i] = ckpt + slab * i;
    a.gout[i] = i == 0 ? grad_cost : work + (i - 1) * V;
    a.gp1[i] = maps + i * npix;
    a.gp2[i] = maps + (4 + i) * npix;
  }
  a.q = make_grid<G>(B, H, W, D);
  constexpr size_t smem = bwd_smem_bytes<G, K>();
  if (cudaFuncSetAttribute(k_float_bwd<G, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return check("float backward attribute");
  k_float_bwd<G, K><<<a.q.first_block[4], kWarps * 32, smem, s>>>(a);
  if ((st = check("float backward"))) return st;
  SumArgs r;
  r.g0 = reinterpret_cast<float4*>(grad_cost);
  r.g1 = reinterpret_cast<const float4*>(a.gout[1]);
  r.g2 = reinterpret_cast<const float4*>(a.gout[2]);
  r.g3 = reinterpret_cast<const float4*>(a.gout[3]);
  r.n4 = V / 4;
  r.gp1 = grad_p1;
  r.gp2 = grad_p2;
  for (int i = 0; i < 4; ++i) {
    r.a1[i] = a.gp1[i];
    r.a2[i] = a.gp2[i];
  }
  r.npix = npix;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  k_grad_sum<<<nsm * 8, 256, 0, s>>>(r);
  return check("float backward sum");
}

}  // namespace

// Waits of the forward scans that ran out (sgm_debug_wait_timeouts adds them to the engine's).
int64_t sgm_float_wait_timeouts() {
  unsigned int n = 0;
  if (cudaMemcpyFromSymbol(&n, sgm::g_scan_wait_timeouts, sizeof(n)) != cudaSuccess) return -1;
  return n;
}

extern "C" {

size_t sgm_float_checkpoint_elems(int32_t B, int32_t H, int32_t W, int32_t D) {
  size_t n = 0;
  for (int dir = 0; dir < 4; ++dir) {
    const Geo g = make_geo(B, H, W, D, dir);
    n = n > (size_t)g.lines * g.nseg * D ? n : (size_t)g.lines * g.nseg * D;
  }
  return 4 * n;
}

size_t sgm_float_workspace_elems(int32_t B, int32_t H, int32_t W, int32_t D) {
  return 3 * (size_t)B * H * W * D + 8 * (size_t)B * H * W;
}

int sgm_float_forward(const float* cost, const float* p1, const float* p2, int32_t B, int32_t H, int32_t W,
                      int32_t D, float temperature, float* sum, float* ckpt, float* work, float* disp, void* stream) {
  int st = validate(B, H, W, D, temperature);
  if (st || (st = check_present({cost, p1, p2, sum, ckpt, work, disp})) ||
      (st = check_aligned({cost, sum, ckpt, work})))
    return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float inv_t = 1.0f / temperature;
  return D == 64 ? forward_impl<2>(cost, p1, p2, B, H, W, inv_t, sum, ckpt, work, disp, s)
                 : forward_impl<1>(cost, p1, p2, B, H, W, inv_t, sum, ckpt, work, disp, s);
}

int sgm_float_backward(const float* cost, const float* p1, const float* p2, int32_t B, int32_t H, int32_t W, int32_t D,
                       float temperature, const float* sum, const float* ckpt, const float* grad_disp,
                       float* grad_sum, float* work, float* grad_cost, float* grad_p1, float* grad_p2, void* stream) {
  int st = validate(B, H, W, D, temperature);
  if (st || (st = check_present({cost, p1, p2, sum, ckpt, grad_disp, grad_sum, work, grad_cost, grad_p1, grad_p2})) ||
      (st = check_aligned({cost, sum, ckpt, grad_sum, work, grad_cost})))
    return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float inv_t = 1.0f / temperature;
  return D == 64 ? backward_impl<kBwdLanes64, 64 / kBwdLanes64>(cost, p1, p2, B, H, W, inv_t, sum, ckpt, grad_disp,
                                                                grad_sum, work, grad_cost, grad_p1, grad_p2, s)
                 : backward_impl<kBwdLanes32, 32 / kBwdLanes32>(cost, p1, p2, B, H, W, inv_t, sum, ckpt, grad_disp,
                                                                grad_sum, work, grad_cost, grad_p1, grad_p2, s);
}

}  // extern "C"
