// Latency form of the 32-disparity scans (pyramid levels below the coarsest), variant 4.
//
// A pair alone on the GPU offers few scanlines (375 rows x 2 directions at 1242x375), so the time
// of a scan is its number of steps times the length of one step's dependency chain. Here one warp
// owns a scanline and lane d holds disparity d in 32 bits, the reference's own arithmetic
// (Kernel_Aggregate_{Horizontal,Vertical}_Warp, cusgm_ca.cu:1181-1338). A step's chain is then
//   m = prev_invalid ? 127 : min_d L(d)            one redux.sync, issued beside the shuffles
//   a, b = L(d + s - 1), L(d + s + 1)              two shuffles (s = base - last_base)
//   L'(d) = C(d) + min(L(d), a + P1, b + P1, m + P2') - m
// and everything that does not depend on L is taken off it:
//   * the chunk's 32 steps of costs (and, for the top-to-bottom pass, of the three stored paths)
//     are staged in shared memory by bulk async copies (cp.async.bulk with an mbarrier), one chunk
//     ahead, double-buffered; a row chunk is one contiguous 1 KB copy, a column chunk one 32-byte
//     copy per step;
//   * the per-step bookkeeping of the initial disparities -- the realignment shift, P2' =
//     max(P1, P2 / |last_base - base + 1|), which steps are skipped for an INVALID base -- is
//     computed for the whole chunk at once, one step per lane (ballot for the last valid base);
//   * path costs go to a shared-memory chunk and leave with 16-byte stores.
// Every wait on an mbarrier is bounded: after kMaxWaitTries polls the warp records the timeout in
// g_scan_wait_timeouts (read by sgm_debug_wait_timeouts) and stops.
#pragma once
#include <type_traits>

#include "sgm_kernels3.cuh"

namespace sgm {

constexpr int kScanChunk = 32;          // steps per staged chunk
constexpr int kMaxWaitTries = 1 << 22;  // polls of an mbarrier before a wait is given up

static __device__ unsigned int g_scan_wait_timeouts;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Generic-proxy accesses of shared memory before async-proxy writes into it.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// `bytes` (a multiple of 16) from global src to shared dst (both 16-byte aligned), completing on bar.
__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Waits for the phase of bar with the given parity; false after kMaxWaitTries polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < kMaxWaitTries; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// The same wait by every lane of the warp, with one verdict for all: the warp stays converged for
// its shuffles even when the limit runs out in some lanes only.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity) {
  return __all_sync(kFull, mbar_wait(bar, parity));
}
// A wait that ran out: record it, then wait (again bounded) for the copies still in flight into
// this warp's buffers before the warp leaves.
// phase: bit b = the parity of the phase buffer b waits for next.
__device__ __forceinline__ void scan_give_up(uint64_t* bars, uint32_t phase, int nbars) {
  if ((threadIdx.x & 31) == 0) atomicAdd(&g_scan_wait_timeouts, 1u);
  for (int b = 0; b < nbars; ++b) mbar_wait(bars + b, (phase >> b) & 1u);
}

// Per-step parameters of a chunk, one step per lane (lane j = step j): packed as
// shift (8 bits, clamped to +-64: any |shift| > 33 puts both neighbours out of range) |
// kStepValid | kPrevInvalid, and P2'.
constexpr uint32_t kStepValid = 1u << 8, kPrevInvalid = 1u << 9;

struct ChunkState {
  int carry_base;      // base of the last step that set last_base before the chunk
  bool carry_invalid;  // the last step before the chunk was skipped (INVALID base)
};

// b: this lane's step base (INVALID for lanes past the chunk); gs0: global index of the chunk's
// first step; n: steps in the chunk; first_sets_base: the scanline's first pixel sets last_base
// (horizontal scans) or keeps the one given (vertical scans, cusgm_ca.cu:1291).
__device__ __forceinline__ void chunk_params(int b, int gs0, int n, bool first_sets_base, const InitParams& P,
                                             ChunkState& st, uint32_t& flags, uint32_t& p2) {
  const int j = threadIdx.x & 31;
  const bool in = j < n;
  const bool first = gs0 + j == 0;
  const bool step_valid = in && !first && b != kInvalidShort;
  const bool sets_base = in && (step_valid || (first && first_sets_base));
  const unsigned vm = __ballot_sync(kFull, sets_base);
  const unsigned prev = vm & ((1u << j) - 1u);
  const int from_prev = __shfl_sync(kFull, b, prev ? 31 - __clz(prev) : 0);
  const int lb = prev ? from_prev : st.carry_base;
  const int s = b - lb;
  const int sc = s < -64 ? -64 : (s > 64 ? 64 : s);
  const int k = abs(lb - b + 1);
  const int32_t q = k ? P.p2s / k : P.p2_div0;
  p2 = (uint32_t)(P.p1s > q ? P.p1s : q);
  // the previous step was skipped: the chunk's carry for lane 0, the left neighbour's flag else
  const unsigned inv = __ballot_sync(kFull, in && !first && b == kInvalidShort);
  const bool prev_inv = j == 0 ? st.carry_invalid : ((inv >> (j - 1)) & 1u);
  flags = (uint32_t)(sc & 0xFF) | (step_valid ? kStepValid : 0u) | (prev_inv ? kPrevInvalid : 0u);
  const int last_set = __shfl_sync(kFull, b, vm ? 31 - __clz(vm) : 0);
  if (vm) st.carry_base = last_set;
  if (n > 0) st.carry_invalid = (inv >> (n - 1)) & 1u;
}

// One step of the scanline held by the warp (lane = disparity). L: this lane's state; c: its cost.
__device__ __forceinline__ void scan_step(uint32_t& L, uint32_t c, uint32_t flags, uint32_t p2, uint32_t p1) {
  const int lane = threadIdx.x & 31;
  const int s = (int)(int8_t)(flags & 0xFFu);
  const uint32_t mr = __reduce_min_sync(kFull, L);
  const int i1 = lane + s - 1, i2 = lane + s + 1;
  const uint32_t a = __shfl_sync(kFull, L, i1 & 31);
  const uint32_t b = __shfl_sync(kFull, L, i2 & 31);
  const uint32_t m = (flags & kPrevInvalid) ? kInvalidCost : mr;
  const uint32_t A = (unsigned)i1 < 32u ? a + p1 : kInvalidCost;
  const uint32_t B = (unsigned)i2 < 32u ? b + p1 : kInvalidCost;
  const uint32_t t = min(__vimin3_u32(L, A, B), m + p2);
  const uint32_t Ln = c + (t - m);
  if (flags & kStepValid) L = Ln;
}

// WTA of one pixel of an initial-disparity level from its four stored path rows (32 bytes each;
// S(d) = sum of the four), computed by one lane: Kernel_ComputeDisparityByWTA for initial
// disparities (cusgm_ca.cu:3425-3512). d* <= 1 or d* >= 31 -> INVALID; uniqueness and the
// +0.5-shifted parabola as in wta_pixel; tie rules: kTieRefB200 the lowest tied d whose candidate
// is valid (every tied lane stores its own result there, a valid one wins), 1 / 2 the highest tied
// d, 0 / 3 the lowest (one disparity per lane: lane order is disparity order).
__device__ __forceinline__ float init_wta_serial(const uint8_t* a, const uint8_t* b, const uint8_t* c,
                                                 const uint8_t* e, int base, const WtaParams& Q) {
  constexpr int D = kLevelRange;
  uint32_t S[D];
#pragma unroll
  for (int k = 0; k < D / 4; ++k) {
    const uint32_t wa = reinterpret_cast<const uint32_t*>(a)[k], wb = reinterpret_cast<const uint32_t*>(b)[k];
    const uint32_t wc = reinterpret_cast<const uint32_t*>(c)[k], we = reinterpret_cast<const uint32_t*>(e)[k];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      S[4 * k + q] = ((wa >> (8 * q)) & 0xFFu) + ((wb >> (8 * q)) & 0xFFu) + ((wc >> (8 * q)) & 0xFFu) +
                     ((we >> (8 * q)) & 0xFFu);
  }
  uint32_t m = S[0];
#pragma unroll
  for (int d = 1; d < D; ++d) m = min(m, S[d]);
  const float ut = __fsub_rn(1.0f, Q.uniqueness);
  // S at a runtime d, summed again from the rows (S[] stays in registers, indexed statically)
  auto sum_at = [&](int d) { return (uint32_t)a[d] + b[d] + c[d] + e[d]; };
  auto candidate = [&](int d) {
    if (d <= 1 || d >= Q.dmax_excl) return kInvalidFloat;
    const float c1 = (float)sum_at(d - 1), c2 = (float)m, c3 = (float)sum_at(d + 1);
    const float d12 = __fsub_rn(c1, c2), d32 = __fsub_rn(c3, c2);
    const float uq = d12 < d32 ? d12 : d32;
    if (uq <= __fmul_rn(c2, ut)) return kInvalidFloat;
    return __fadd_rn((float)(d + base), subpix_bias(c1, c2, c3));
  };
  uint32_t tied = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) tied |= (S[d] == m ? 1u : 0u) << d;
  if (Q.tie_rule == kTieRefB200) {
    while (tied) {
      const int d = __ffs(tied) - 1;
      const float v = candidate(d);
      if (v != kInvalidFloat) return v;
      tied &= tied - 1u;
    }
    return kInvalidFloat;
  }
  const bool high = Q.tie_rule == kTieHighest || Q.tie_rule == kTieLaneHigh;
  return candidate(high ? 31 - __clz(tied) : __ffs(tied) - 1);
}

// ---------------------------------------------------------------------------------------------
// Horizontal scans: warp w of the grid owns scanline i = (view, dir, y) as in hpaths3_lane.
// ---------------------------------------------------------------------------------------------
template <int WPB>
__global__ void __launch_bounds__(32 * WPB) k_hscan_init4(const uint8_t* __restrict__ cost,
                                                          const int16_t* __restrict__ init_l,
                                                          const int16_t* __restrict__ init_r,
                                                          uint8_t* __restrict__ lr, uint8_t* __restrict__ rl,
                                                          InitParams P, int nviews) {
  constexpr int D = kLevelRange, C = kScanChunk;
  __shared__ __align__(128) uint8_t cbuf[WPB][2][C * D];
  __shared__ __align__(16) uint8_t obuf[WPB][C * D];
  __shared__ __align__(8) uint64_t bars[WPB][2];
  __shared__ __align__(16) uint32_t par[WPB][2][C];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    mbar_init(&bars[w][0], 1);
    mbar_init(&bars[w][1], 1);
    mbar_fence_init();
  }
  __syncwarp();
  const int H = P.H, W = P.W;
  const int i = blockIdx.x * WPB + w;
  if (i >= nviews * 2 * H) return;  // the whole warp
  const int grp = i / H, y = i - grp * H;
  const int view = grp >> 1, dir = grp & 1;
  const int len = W - P.x0;
  if (len <= 0) return;
  const size_t ro = (size_t)view * P.vstride + (size_t)y * W * D;
  const uint8_t* crow = cost + ro;
  uint8_t* orow = (dir == 0 ? lr : rl) + ro;
  const int16_t* ib = (view == 0 ? init_l : init_r) + (size_t)y * W;
  const int nch = (len + C - 1) / C;
  // chunk c: steps [c*C, c*C + n), pixels [xa, xa + n) in memory order
  auto chunk_n = [&](int c) { return min(C, len - c * C); };
  auto chunk_x = [&](int c) { return dir == 0 ? P.x0 + c * C : W - (c * C + chunk_n(c)); };
  auto issue = [&](int c, int buf) {
    if (lane == 0) {
      const uint32_t bytes = (uint32_t)chunk_n(c) * D;
      mbar_expect_tx(&bars[w][buf], bytes);
      bulk_to_smem(cbuf[w][buf], crow + (size_t)chunk_x(c) * D, bytes, &bars[w][buf]);
    }
  };
  auto base_of = [&](int c) {  // this lane's step of chunk c
    const int n = chunk_n(c);
    if (lane >= n) return (int)kInvalidShort;
    const int x = dir == 0 ? P.x0 + c * C + lane : W - 1 - (c * C + lane);
    return (int)ib[x];
  };
  issue(0, 0);
  if (nch > 1) issue(1, 1);
  uint32_t phase = 0u;  // bit b: parity of buffer b's next phase
  ChunkState st{0, false};
  int bnext = base_of(0);
  uint32_t L = 0;
  for (int c = 0; c < nch; ++c) {
    const int buf = c & 1, n = chunk_n(c);
    const int bcur = bnext;
    if (c + 1 < nch) bnext = base_of(c + 1);  // a chunk ahead
    uint32_t flags, p2;
    chunk_params(bcur, c * C, n, true, P, st, flags, p2);
    par[w][0][lane] = flags;
    par[w][1][lane] = p2;
    if (!mbar_wait_warp(&bars[w][buf], (phase >> buf) & 1u)) {
      scan_give_up(bars[w], phase, 2);
      return;
    }
    phase ^= 1u << buf;
    __syncwarp();
    const uint8_t* cb = cbuf[w][buf];
    uint8_t* ob = obuf[w];
    // the chunk's step parameters and this lane's costs in registers: the chain below then
    // touches no memory but the stores of its results
    uint32_t fl[C], pp[C], cvr[C];
#pragma unroll
    for (int j = 0; j < C; ++j) {
      fl[j] = par[w][0][j];
      pp[j] = par[w][1][j];
      cvr[j] = cb[(j < n ? (dir == 0 ? j : n - 1 - j) : 0) * D + lane];
    }
    // all 32 steps run: past the end of a short last chunk the steps are marked skipped (their
    // flags have no kStepValid), so the state is kept and nothing is stored
#pragma unroll
    for (int j = 0; j < C; ++j) {
      if (c == 0 && j == 0) L = cvr[0];  // first pixel of the scanline
      else scan_step(L, cvr[j], fl[j], pp[j], P.p1);
      if (j < n) ob[(dir == 0 ? j : n - 1 - j) * D + lane] = (uint8_t)L;
    }
    __syncwarp();
    // the chunk's path costs: lane j writes pixel xa + j (32 bytes)
    if (lane < n) {
      const uint4* src = reinterpret_cast<const uint4*>(ob + lane * D);
      uint4* dst = reinterpret_cast<uint4*>(orow + (size_t)(chunk_x(c) + lane) * D);
      const uint4 v0 = src[0], v1 = src[1];
      dst[0] = v0;
      dst[1] = v1;
    }
    __syncwarp();
    if (c + 2 < nch) {
      fence_proxy_async();
      issue(c + 2, buf);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Vertical scans: warp (blockIdx.x * WPB + w) owns column x of view blockIdx.y. PASS 1: bottom to
// top, storing its path costs. PASS 2: top to bottom with the 4-path sum and the WTA of an
// initial-disparity level (as vpaths3_init_lane / k_vpaths_wta_init). Both start last_base from
// row 0's base (cusgm_ca.cu:1291); the first pixel of a vertical path does not set it.
// ---------------------------------------------------------------------------------------------
template <int WPB, int PASS>
__global__ void __launch_bounds__(32 * WPB) k_vscan_init4(const uint8_t* __restrict__ cost,
                                                          const uint8_t* __restrict__ lr,
                                                          const uint8_t* __restrict__ rl,
                                                          const int16_t* __restrict__ init_l,
                                                          const int16_t* __restrict__ init_r,
                                                          uint8_t* __restrict__ bt, float* __restrict__ disp,
                                                          InitParams P, WtaParams Q) {
  constexpr int D = kLevelRange, C = kScanChunk;
  constexpr int NV = PASS == 2 ? 4 : 1;  // staged volumes: cost (+ bottom->top, L->R, R->L)
  __shared__ __align__(128) uint8_t cbuf[WPB][2][NV][C * D];
  __shared__ __align__(16) uint8_t obuf[WPB][C * D];
  __shared__ __align__(8) uint64_t bars[WPB][2];
  __shared__ __align__(16) uint32_t par[WPB][2][C];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    mbar_init(&bars[w][0], 1);
    mbar_init(&bars[w][1], 1);
    mbar_fence_init();
  }
  __syncwarp();
  const int W = P.W, H = P.H;
  const int x = blockIdx.x * WPB + w;
  const int view = blockIdx.y;
  if (x >= W) return;  // the whole warp
  float* dout = disp + (size_t)view * Q.dstride + x;
  if (x < P.x0) {
    if (PASS == 2)
      for (int y = lane; y < H; y += 32) dout[(size_t)y * W] = kInvalidFloat;
    return;
  }
  const size_t vo = (size_t)view * P.vstride + (size_t)x * D;
  const size_t rs = (size_t)W * D;  // bytes between rows
  const uint8_t* vol[4] = {cost + vo, bt + vo, lr + vo, rl + vo};
  const int16_t* ib = (view == 0 ? init_l : init_r) + x;
  const int nch = (H + C - 1) / C;
  auto chunk_n = [&](int c) { return min(C, H - c * C); };
  auto row_of = [&](int s) { return PASS == 1 ? H - 1 - s : s; };
  auto issue = [&](int c, int buf) {
    const int n = chunk_n(c);
    if (lane == 0) mbar_expect_tx(&bars[w][buf], (uint32_t)(n * D * NV));
    __syncwarp();
    if (lane < n) {
      const size_t ro = (size_t)row_of(c * C + lane) * rs;
#pragma unroll
      for (int v = 0; v < NV; ++v) bulk_to_smem(cbuf[w][buf][v] + lane * D, vol[v] + ro, D, &bars[w][buf]);
    }
  };
  auto base_of = [&](int c) {
    const int n = chunk_n(c);
    return lane < n ? (int)ib[(size_t)row_of(c * C + lane) * W] : (int)kInvalidShort;
  };
  issue(0, 0);
  if (nch > 1) issue(1, 1);
  uint32_t phase = 0u;  // bit b: parity of buffer b's next phase
  ChunkState st{(int)ib[0], false};  // row 0's base
  int bnext = base_of(0);
  uint32_t L = 0;
  const bool col_ok = x >= Q.xlo && x <= Q.xhi;
  for (int c = 0; c < nch; ++c) {
    const int buf = c & 1, n = chunk_n(c);
    const int bcur = bnext;
    if (c + 1 < nch) bnext = base_of(c + 1);
    uint32_t flags, p2;
    chunk_params(bcur, c * C, n, false, P, st, flags, p2);
    // flags in the low 16 bits, the step's base in the high 16 (the WTA needs it, PASS 2)
    par[w][0][lane] = flags | ((uint32_t)(uint16_t)(int16_t)bcur << 16);
    par[w][1][lane] = p2;
    if (!mbar_wait_warp(&bars[w][buf], (phase >> buf) & 1u)) {
      scan_give_up(bars[w], phase, 2);
      return;
    }
    phase ^= 1u << buf;
    __syncwarp();
    // the chunk's step parameters and this lane's costs in registers: the chain below touches no
    // memory but the stores of its results
    uint32_t fl[C], pp[C], cvr[C];
#pragma unroll
    for (int j = 0; j < C; ++j) {
      fl[j] = par[w][0][j];
      pp[j] = par[w][1][j];
      cvr[j] = cbuf[w][buf][0][j * D + lane];
    }
    // all 32 steps run (steps past a short last chunk are marked skipped and store nothing)
#pragma unroll
    for (int j = 0; j < C; ++j) {
      if (c == 0 && j == 0) L = cvr[0];
      else scan_step(L, cvr[j], fl[j], pp[j], P.p1);
      if (j < n) obuf[w][j * D + lane] = (uint8_t)L;
    }
    __syncwarp();
    float dv_keep = kInvalidFloat;  // lane j: the disparity of step j (PASS 2)
    if constexpr (PASS == 2) {
      // the WTA of the chunk's pixels, lane j = pixel j (off the steps' dependency chain)
      const int y = c * C + lane;
      const int base = (int)(int16_t)(par[w][0][lane] >> 16);
      const bool skipped = y > 0 && base == kInvalidShort;
      if (lane < n && y >= Q.ylo && y <= Q.yhi && y < Q.rows && col_ok && !skipped && base != kInvalidShort)
        dv_keep = init_wta_serial(obuf[w] + lane * D, cbuf[w][buf][1] + lane * D, cbuf[w][buf][2] + lane * D,
                                  cbuf[w][buf][3] + lane * D, base, Q);
    }
    __syncwarp();
    if (lane < n) {
      const size_t ro = (size_t)row_of(c * C + lane) * rs;
      if constexpr (PASS == 1) {
        const uint4* src = reinterpret_cast<const uint4*>(obuf[w] + lane * D);
        uint4* dst = reinterpret_cast<uint4*>(bt + vo + ro);
        const uint4 v0 = src[0], v1 = src[1];
        dst[0] = v0;
        dst[1] = v1;
      } else {
        dout[(size_t)(c * C + lane) * W] = dv_keep;
      }
    }
    __syncwarp();
    if (c + 2 < nch) {
      fence_proxy_async();
      issue(c + 2, buf);
    }
  }
}

}  // namespace sgm

namespace sgm {

// =============================================================================================
// Plain levels (no initial disparities), latency form. One warp owns a scanline; lane l holds
// d = l + 32k, k < K, in 32 bits (the reference's Kernel_Aggregate_*_Warpfor{32,64,128},
// cusgm_ca.cu:1343-1888, computes the same recurrence). A step:
//   m = min_d L(d)                       one redux.sync of the lanes' K-wide minima
//   L(d - 1), L(d + 1)                   2K shuffles (lane - 1 / lane + 1, across the k words)
//   L'(d) = C(d) + min(L(d), L(d-1) + P1 | 127, L(d+1) + P1 | 127, m + P2) - m
// Chunks of 32 steps move between global and shared memory with bulk async copies; a step's path
// costs overwrite its costs in the chunk buffer, which then leaves with a bulk store (rows: one
// contiguous copy; columns: one per step), three buffers deep so a load never waits for the store
// of the chunk before. The WTA of the top-to-bottom pass runs per chunk with lane = pixel.
// =============================================================================================

// `bytes` (a multiple of 16) from shared src to global dst (both 16-byte aligned), in the calling
// thread's current bulk group.
__device__ __forceinline__ void bulk_to_global(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// All but the newest N of this thread's bulk groups have finished reading shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// All of this thread's bulk groups are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// As scan_give_up, for the buffers whose bit is set in `pending` only.
__device__ __forceinline__ void scan_give_up_mask(uint64_t* bars, uint32_t phase, uint32_t pending) {
  if ((threadIdx.x & 31) == 0) atomicAdd(&g_scan_wait_timeouts, 1u);
  for (int b = 0; b < 32; ++b)
    if ((pending >> b) & 1u) mbar_wait(bars + b, (phase >> b) & 1u);
}

// Shared-memory row of one step: D bytes padded to D + 16, so that 16-byte loads of 8 lanes at
// consecutive rows fall in distinct banks.
template <int D>
__host__ __device__ constexpr int plain_row_stride() { return D + 16; }

template <int K>
__device__ __forceinline__ void plain_step4(uint32_t (&L)[K], const uint32_t (&c)[K], uint32_t p1, uint32_t p2) {
  const int lane = threadIdx.x & 31;
  uint32_t lm = L[0];
#pragma unroll
  for (int k = 1; k < K; ++k) lm = min(lm, L[k]);
  const uint32_t m = __reduce_min_sync(kFull, lm);
  uint32_t r[K], q[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    r[k] = __shfl_sync(kFull, L[k], (lane + 31) & 31);  // L(d - 1), lanes 1..31
    q[k] = __shfl_sync(kFull, L[k], (lane + 1) & 31);   // L(d + 1), lanes 0..30
  }
  const uint32_t l4 = m + p2;
  uint32_t n[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    // lane 0: d - 1 is lane 31 of word k - 1 (its r[k - 1]); lane 31: d + 1 is lane 0 of word k + 1
    const uint32_t A = lane > 0 ? r[k] + p1 : (k > 0 ? r[k - 1] + p1 : kInvalidCost);
    const uint32_t B = lane < 31 ? q[k] + p1 : (k < K - 1 ? q[k + 1] + p1 : kInvalidCost);
    const uint32_t t = min(__vimin3_u32(L[k], A, B), l4);
    n[k] = c[k] + (t - m);
  }
#pragma unroll
  for (int k = 0; k < K; ++k) L[k] = n[k];
}

// The 32 steps of a chunk held in shared memory: step j reads its costs from row(j) (byte
// lane + 32k) and leaves its path costs there. first: step 0 starts the scanline (L = C).
// Costs are read R steps ahead.
template <int K, typename RowOf>
__device__ __forceinline__ void plain_chunk(uint8_t* buf, RowOf row, int n, bool first, uint32_t (&L)[K],
                                            uint32_t p1, uint32_t p2) {
  constexpr int C = kScanChunk, R = 32 / K;
  const int lane = threadIdx.x & 31;
  uint32_t ring[R][K];
#pragma unroll
  for (int j = 0; j < R; ++j)
#pragma unroll
    for (int k = 0; k < K; ++k) ring[j][k] = j < n ? buf[row(j) + lane + 32 * k] : 0u;
#pragma unroll
  for (int j = 0; j < C; ++j) {
    if (j < n) {  // uniform over the warp
      uint32_t c[K];
#pragma unroll
      for (int k = 0; k < K; ++k) c[k] = ring[j % R][k];
      if (j + R < C && j + R < n) {
#pragma unroll
        for (int k = 0; k < K; ++k) ring[j % R][k] = buf[row(j + R) + lane + 32 * k];
      }
      if (j == 0 && first) {
#pragma unroll
        for (int k = 0; k < K; ++k) L[k] = c[k];
      } else {
        plain_step4<K>(L, c, p1, p2);
      }
      uint8_t* o = buf + row(j) + lane;
#pragma unroll
      for (int k = 0; k < K; ++k) o[32 * k] = (uint8_t)L[k];
    }
  }
}

// Horizontal scans of a plain level; warp (blockIdx.x * WPB + w) owns scanline i = (view, dir, y)
// as in hpaths3_lane. A chunk is 32 consecutive pixels of the row: one contiguous bulk copy in,
// one out.
template <int K>
__host__ __device__ constexpr int hscan_plain4_warps() { return K == 4 ? 2 : 4; }

template <int K, int WPB = hscan_plain4_warps<K>()>
__global__ void __launch_bounds__(32 * WPB) k_hscan_plain4(const uint8_t* __restrict__ cost, uint8_t* __restrict__ lr,
                                                           uint8_t* __restrict__ rl, PlainParams P, int nviews) {
  constexpr int D = 32 * K, C = kScanChunk, NB = 3;
  __shared__ __align__(128) uint8_t cbuf[WPB][NB][C * D];
  __shared__ __align__(8) uint64_t bars[WPB][NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    for (int b = 0; b < NB; ++b) mbar_init(&bars[w][b], 1);
    mbar_fence_init();
  }
  __syncwarp();
  const int H = P.H, W = P.W;
  const int i = blockIdx.x * WPB + w;
  if (i >= nviews * 2 * H) return;  // the whole warp
  const int grp = i / H, y = i - grp * H;
  const int view = grp >> 1, dir = grp & 1;
  const int len = W - P.x0;
  if (len <= 0) return;
  const size_t ro = (size_t)view * P.vstride + (size_t)y * W * D;
  const uint8_t* crow = cost + ro;
  uint8_t* orow = (dir == 0 ? lr : rl) + ro;
  const int nch = (len + C - 1) / C;
  auto chunk_n = [&](int c) { return min(C, len - c * C); };
  auto chunk_x = [&](int c) { return dir == 0 ? P.x0 + c * C : W - (c * C + chunk_n(c)); };
  auto issue = [&](int c) {  // lane 0
    const int b = c % NB;
    const uint32_t bytes = (uint32_t)chunk_n(c) * D;
    mbar_expect_tx(&bars[w][b], bytes);
    bulk_to_smem(cbuf[w][b], crow + (size_t)chunk_x(c) * D, bytes, &bars[w][b]);
  };
  if (lane == 0) {
    issue(0);
    if (nch > 1) issue(1);
  }
  uint32_t phase = 0u;
  uint32_t L[K];
  for (int c = 0; c < nch; ++c) {
    const int b = c % NB, n = chunk_n(c);
    if (!mbar_wait_warp(&bars[w][b], (phase >> b) & 1u)) {
      scan_give_up_mask(bars[w], phase, (1u << b) | (c + 1 < nch ? 1u << ((c + 1) % NB) : 0u));
      if (lane == 0) bulk_wait_all();
      return;
    }
    phase ^= 1u << b;
    __syncwarp();
    if (dir == 0)
      plain_chunk<K>(cbuf[w][b], [](int j) { return j * D; }, n, c == 0, L, P.p1, P.p2);
    else
      plain_chunk<K>(cbuf[w][b], [n](int j) { return (n - 1 - j) * D; }, n, c == 0, L, P.p1, P.p2);
    fence_proxy_async();  // the chunk's path costs (and its cost reads) before the bulk copies
    __syncwarp();
    if (lane == 0) {
      bulk_to_global(orow + (size_t)chunk_x(c) * D, cbuf[w][b], (uint32_t)n * D);
      bulk_commit();
      if (c + 2 < nch) {
        bulk_wait_read<1>();  // the store of chunk c - 1 has left the buffer chunk c + 2 goes to
        issue(c + 2);
      }
    }
  }
  if (lane == 0) bulk_wait_all();
}

// WTA of one plain-level pixel from its four path rows (D bytes each), by one lane:
// Kernel_ComputeDisparityByWTA_Warpfor{32,64,128} (cusgm_ca.cu:3514-3809). S(d) is summed in
// 16-bit halves (at most 4 x 255). d* = 0 or d* >= Q.dmax_excl -> INVALID; c3 at d* = D - 1 is
// the index itself; uniqueness and the +0.5-shifted parabola as in wta_pixel. Tie rules: kTieRefB200
// at D = 64 (A = {t < 32 : S(t) = m}, B = {t < 32 : S(t + 32) = m, S(t) != m}; even rows of the
// launch take the lowest of B (+ 32) if any, else of A; odd rows the lowest of A if any, else of B
// (+ 32)); kTieHighest the highest tied d; the rest the lowest.
template <int D>
__device__ __forceinline__ float plain_wta_rows(const uint8_t* a, const uint8_t* b, const uint8_t* c,
                                                const uint8_t* e, int min_d, int y, const WtaParams& Q) {
  constexpr int NW = D / 4, NB = D / 32;
  constexpr uint32_t M8 = 0x00FF00FFu;
  uint32_t lo[NW], hi[NW];  // lo[k] = S(4k) | S(4k + 2) << 16, hi[k] = S(4k + 1) | S(4k + 3) << 16
#pragma unroll
  for (int q = 0; q < D / 16; ++q) {
    const uint4 va = reinterpret_cast<const uint4*>(a)[q], vb = reinterpret_cast<const uint4*>(b)[q];
    const uint4 vc = reinterpret_cast<const uint4*>(c)[q], ve = reinterpret_cast<const uint4*>(e)[q];
    const uint32_t wa[4] = {va.x, va.y, va.z, va.w}, wb[4] = {vb.x, vb.y, vb.z, vb.w};
    const uint32_t wc[4] = {vc.x, vc.y, vc.z, vc.w}, we[4] = {ve.x, ve.y, ve.z, ve.w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      lo[4 * q + t] = (wa[t] & M8) + (wb[t] & M8) + (wc[t] & M8) + (we[t] & M8);
      hi[4 * q + t] = ((wa[t] >> 8) & M8) + ((wb[t] >> 8) & M8) + ((wc[t] >> 8) & M8) + ((we[t] >> 8) & M8);
    }
  }
  uint32_t mm = __vminu2(lo[0], hi[0]);
#pragma unroll
  for (int k = 1; k < NW; ++k) mm = __vminu2(mm, __vminu2(lo[k], hi[k]));
  const uint32_t m = min(mm & 0xFFFFu, mm >> 16);
  const uint32_t m2 = m * 0x10001u;
  uint32_t word[NB];  // bit t of word[k]: S(32k + t) == m
#pragma unroll
  for (int k = 0; k < NB; ++k) word[k] = 0u;
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    const uint32_t el = __vcmpeq2(lo[k], m2), eh = __vcmpeq2(hi[k], m2);
    const uint32_t nib = (el & 1u) | ((eh & 1u) << 1) | ((el >> 14) & 4u) | ((eh >> 13) & 8u);
    word[k / 8] |= nib << (4 * (k % 8));
  }
  int ds;
  if (D == 64 && Q.tie_rule == kTieRefB200) {
    const uint32_t A = word[0], B = word[NB - 1] & ~word[0];
    if ((y & 1) == 0) ds = B ? (__ffs(B) - 1 + 32) : (__ffs(A) - 1);
    else ds = A ? (__ffs(A) - 1) : (__ffs(B) - 1 + 32);
  } else if (Q.tie_rule == kTieHighest) {
    ds = -1;
#pragma unroll
    for (int k = 0; k < NB; ++k)
      if (word[k]) ds = 32 * k + 31 - __clz(word[k]);
  } else {
    ds = -1;
#pragma unroll
    for (int k = NB - 1; k >= 0; --k)
      if (word[k]) ds = 32 * k + __ffs(word[k]) - 1;
  }
  if (ds <= 0 || ds >= Q.dmax_excl) return kInvalidFloat;
  auto sum_at = [&](int d) { return (uint32_t)a[d] + b[d] + c[d] + e[d]; };
  const float c1 = (float)sum_at(ds - 1);
  const float c2 = (float)m;
  const float c3 = (ds + 1 < D) ? (float)sum_at(ds + 1) : (float)ds;
  const float d12 = __fsub_rn(c1, c2), d32 = __fsub_rn(c3, c2);
  const float uq = d12 < d32 ? d12 : d32;
  if (uq <= __fmul_rn(c2, __fsub_rn(1.0f, Q.uniqueness))) return kInvalidFloat;
  return __fadd_rn((float)(ds + min_d), subpix_bias(c1, c2, c3));
}

// Warps per CTA of the column kernels (shared memory: PASS 1 three chunk buffers, PASS 2 two
// chunk buffers and the three stored paths of a chunk, each C x (D + 16) bytes per warp).
template <int K>
__host__ __device__ constexpr int vscan_plain4_warps() { return K == 1 ? 4 : 2; }

// Vertical scans of a plain level: warp (blockIdx.x * WPB + w) owns column x of view blockIdx.y.
// PASS 1: bottom to top, storing its path costs (bt). PASS 2: top to bottom, then per chunk the
// WTA of its 32 pixels with lane = pixel (rows >= Q.rows INVALID, as the reference's two-row WTA
// blocks leave them; border and columns left of x0 INVALID).
template <int K, int PASS>
__global__ void __launch_bounds__(32 * vscan_plain4_warps<K>())
    k_vscan_plain4(const uint8_t* __restrict__ cost, const uint8_t* __restrict__ lr, const uint8_t* __restrict__ rl,
                   uint8_t* __restrict__ bt, float* __restrict__ disp, PlainParams P, WtaParams Q) {
  constexpr int D = 32 * K, C = kScanChunk, RS = plain_row_stride<D>();
  constexpr int WPB = vscan_plain4_warps<K>();
  constexpr int NB = PASS == 1 ? 3 : 2;        // cost chunk buffers
  constexpr int NS = PASS == 1 ? 0 : 3;        // stored-path buffers (bt, lr, rl)
  __shared__ __align__(128) uint8_t cbuf[WPB][NB + NS][C * RS];
  __shared__ __align__(8) uint64_t bars[WPB][NB + 1];  // bars[NB]: the stored paths
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    for (int b = 0; b <= NB; ++b) mbar_init(&bars[w][b], 1);
    mbar_fence_init();
  }
  __syncwarp();
  const int W = P.W, H = P.H;
  const int x = blockIdx.x * WPB + w;
  const int view = blockIdx.y;
  if (x >= W) return;  // the whole warp
  float* dout = disp + (size_t)view * Q.dstride + x;
  if (x < P.x0) {
    if (PASS == 2)
      for (int y = lane; y < H; y += 32) dout[(size_t)y * W] = kInvalidFloat;
    return;
  }
  const size_t vo = (size_t)view * P.vstride + (size_t)x * D;
  const size_t rs = (size_t)W * D;
  const int nch = (H + C - 1) / C;
  auto chunk_n = [&](int c) { return min(C, H - c * C); };
  auto row_of = [&](int s) { return PASS == 1 ? H - 1 - s : s; };
  // chunk c's cost rows into buffer c % NB (lane j: step j)
  auto issue_cost = [&](int c) {
    const int b = c % NB, n = chunk_n(c);
    if (lane == 0) mbar_expect_tx(&bars[w][b], (uint32_t)(n * D));
    __syncwarp();
    if (lane < n) bulk_to_smem(cbuf[w][b] + lane * RS, cost + vo + (size_t)row_of(c * C + lane) * rs, D, &bars[w][b]);
  };
  // chunk c's stored paths (PASS 2)
  auto issue_paths = [&](int c) {
    const int n = chunk_n(c);
    if (lane == 0) mbar_expect_tx(&bars[w][NB], (uint32_t)(3 * n * D));
    __syncwarp();
    if (lane < n) {
      const size_t ro = vo + (size_t)row_of(c * C + lane) * rs;
      bulk_to_smem(cbuf[w][NB + 0] + lane * RS, bt + ro, D, &bars[w][NB]);
      bulk_to_smem(cbuf[w][NB + 1] + lane * RS, lr + ro, D, &bars[w][NB]);
      bulk_to_smem(cbuf[w][NB + 2] + lane * RS, rl + ro, D, &bars[w][NB]);
    }
  };
  issue_cost(0);
  if (nch > 1) issue_cost(1);
  if (PASS == 2) issue_paths(0);
  uint32_t phase = 0u;  // bit b: parity awaited on bars[w][b]
  uint32_t L[K];
  const bool col_ok = x >= Q.xlo && x <= Q.xhi;
  for (int c = 0; c < nch; ++c) {
    const int b = c % NB, n = chunk_n(c);
    const uint32_t pend_cost = (1u << b) | (c + 1 < nch ? 1u << ((c + 1) % NB) : 0u);
    if (!mbar_wait_warp(&bars[w][b], (phase >> b) & 1u)) {
      scan_give_up_mask(bars[w], phase, pend_cost | (PASS == 2 ? 1u << NB : 0u));
      bulk_wait_all();
      return;
    }
    phase ^= 1u << b;
    __syncwarp();
    plain_chunk<K>(cbuf[w][b], [](int j) { return j * RS; }, n, c == 0, L, P.p1, P.p2);
    if constexpr (PASS == 1) {
      fence_proxy_async();
      __syncwarp();
      if (lane < n) {
        bulk_to_global(bt + vo + (size_t)row_of(c * C + lane) * rs, cbuf[w][b] + lane * RS, D);
        bulk_commit();
      }
      if (c + 2 < nch) {
        bulk_wait_read<1>();  // this lane's store of chunk c - 1 has left buffer (c + 2) % 3
        issue_cost(c + 2);
      }
    } else {
      __syncwarp();  // the chunk's path costs, written by disparity, are read by pixel
      if (!mbar_wait_warp(&bars[w][NB], (phase >> NB) & 1u)) {
        scan_give_up_mask(bars[w], phase, (1u << NB) | (c + 1 < nch ? 1u << ((c + 1) % NB) : 0u));
        return;
      }
      phase ^= 1u << NB;
      if (lane < n) {
        const int y = c * C + lane;
        float dv = kInvalidFloat;
        if (col_ok && y >= Q.ylo && y <= Q.yhi && y < Q.rows)
          dv = plain_wta_rows<D>(cbuf[w][b] + lane * RS, cbuf[w][NB] + lane * RS, cbuf[w][NB + 1] + lane * RS,
                                 cbuf[w][NB + 2] + lane * RS, P.min_d, y, Q);
        dout[(size_t)y * W] = dv;
      }
      fence_proxy_async();  // the reads of both buffers before the copies that refill them
      __syncwarp();
      if (c + 1 < nch) issue_paths(c + 1);
      if (c + 2 < nch) issue_cost(c + 2);
    }
  }
  if (PASS == 1) bulk_wait_all();
}

}  // namespace sgm
