// Latency form of the scans, variant 4: the 32-disparity pyramid levels (first half of this file)
// and plain levels with D <= 128 (second half).
//
// A pair alone on the GPU offers few scanlines (375 rows x 2 directions at 1242x375), so the time
// of a scan is its number of steps times the length of one step's dependency chain. Here one warp
// owns a scanline and holds its path costs in 32 bits, the reference's own arithmetic
// (Kernel_Aggregate_{Horizontal,Vertical}_Warp*, cusgm_ca.cu:1181-1888). At a 32-disparity level
// lane d holds disparity d and a step's chain is
//   m = prev_invalid ? 127 : min_d L(d)            one redux.sync, issued beside the shuffles
//   a, b = L(d + s - 1), L(d + s + 1)              two shuffles (s = base - last_base)
//   L'(d) = C(d) + min(L(d), a + P1, b + P1, m + P2') - m
// and everything that does not depend on L is taken off it:
//   * costs (and, for the top-to-bottom pass, the three stored paths) arrive in chunks of 32 steps
//     staged in shared memory by asynchronous copies completing on mbarriers: a row chunk is one
//     contiguous cp.async.bulk copy, a column chunk one box of a 3D tensor map
//     (cp.async.bulk.tensor, swizzled so that lanes reading consecutive box rows hit distinct
//     banks), issued ahead of use;
//   * the per-step bookkeeping of the initial disparities -- the realignment shift, P2' =
//     max(P1, P2 / |last_base - base + 1|), which steps are skipped for an INVALID base -- is
//     computed for a whole chunk at once, one step per lane (ballot for the last valid base), the
//     next chunk's beside the current chunk's steps;
//   * path costs leave per step (row scans at the 32-disparity levels) or per chunk with one bulk
//     or tensor store, and the top-to-bottom pass takes the WTA per chunk with lane = pixel.
// Every wait on an mbarrier is bounded: after kMaxWaitTries polls the warp records the timeout in
// g_scan_wait_timeouts (read by sgm_debug_wait_timeouts), waits (bounded again) for its copies in
// flight and stops.
#pragma once
#include <cuda.h>  // CUtensorMap

#include <type_traits>

#include "sgm_async.cuh"
#include "sgm_kernels3.cuh"

namespace sgm {

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

// scan_step for a step that is valid and follows a valid one (no INVALID base at either): the
// same result with P1 added before the shuffles and the m + P2' bound taken off their path.
__device__ __forceinline__ void scan_step_fast(uint32_t& L, uint32_t c, int s, uint32_t p2, uint32_t p1) {
  const int lane = threadIdx.x & 31;
  const uint32_t m = __reduce_min_sync(kFull, L);
  const uint32_t Lp = L + p1;
  const int i1 = lane + s - 1, i2 = lane + s + 1;
  const uint32_t a = __shfl_sync(kFull, Lp, i1 & 31);
  const uint32_t b = __shfl_sync(kFull, Lp, i2 & 31);
  const uint32_t A = (unsigned)i1 < 32u ? a : kInvalidCost;
  const uint32_t B = (unsigned)i2 < 32u ? b : kInvalidCost;
  const uint32_t t = __vimin3_u32(min(L, m + p2), A, B);
  L = c + t - m;
}

// ---------------------------------------------------------------------------------------------
// Horizontal scans: warp w of the grid owns scanline i = (view, dir, y) as in hpaths3_lane. A
// chunk is 32 consecutive pixels of the row, one contiguous bulk copy (double-buffered); its
// costs go to registers at once, which frees the buffer for the chunk after next. Right-to-left
// scans place a short (last) chunk at the end of the buffer, so that step j of every chunk reads
// row 31 - j; every chunk runs all 32 steps (the steps past a short chunk are marked skipped and
// keep the state). Each step stores its 32 path costs straight to global memory (one 32-byte
// segment per warp). The step parameters of the next chunk are computed
// beside the steps of this one (they do not depend on the path costs), and a chunk whose steps
// all have valid bases (the usual case) runs scan_step_fast. Step parameters: kStepValid,
// kPrevInvalid and the shift in bits 0-9, P2' above them (P1, P2 < 2^22).
// ---------------------------------------------------------------------------------------------
template <int WPB>
__global__ void __launch_bounds__(32 * WPB) k_hscan_init4(const uint8_t* __restrict__ cost,
                                                          const int16_t* __restrict__ init_l,
                                                          const int16_t* __restrict__ init_r,
                                                          uint8_t* __restrict__ lr, uint8_t* __restrict__ rl,
                                                          InitParams P, int nviews) {
  constexpr int D = kLevelRange, C = kScanChunk, NB = 2;
  __shared__ __align__(128) uint8_t cbuf[WPB][NB][C * D];
  __shared__ __align__(8) uint64_t bars[WPB][NB];
  __shared__ uint32_t par[WPB][C];
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
  const int16_t* ib = (view == 0 ? init_l : init_r) + (size_t)y * W;
  const int nch = (len + C - 1) / C;
  // chunk c: steps [c*C, c*C + n), pixels [chunk_x, chunk_x + n) in memory order (n <= 0: none)
  auto chunk_n = [&](int c) { return min(C, len - c * C); };
  auto chunk_x = [&](int c) { return dir == 0 ? P.x0 + c * C : W - (c * C + chunk_n(c)); };
  auto chunk_off = [&](int c) { return dir == 0 ? 0 : (C - chunk_n(c)) * D; };  // bytes into the buffer
  auto issue = [&](int c) {  // lane 0
    const int b = c % NB;
    const uint32_t bytes = (uint32_t)chunk_n(c) * D;
    mbar_expect_tx(&bars[w][b], bytes);
    bulk_to_smem(cbuf[w][b] + chunk_off(c), crow + (size_t)chunk_x(c) * D, bytes, &bars[w][b]);
  };
  auto base_of = [&](int c) {  // this lane's step of chunk c
    const int n = chunk_n(c);
    if (lane >= n) return (int)kInvalidShort;
    const int x = dir == 0 ? P.x0 + c * C + lane : W - 1 - (c * C + lane);
    return (int)ib[x];
  };
  ChunkState st{0, false};
  // packed step parameters of chunk c (lane j: step j) and whether it takes the fast path
  auto params = [&](int c, int bse, uint32_t& pk, bool& fast) {
    uint32_t flags, p2;
    chunk_params(bse, c * C, chunk_n(c), true, P, st, flags, p2);
    pk = (p2 << 10) | flags;
    fast = __all_sync(kFull, (flags & (kStepValid | kPrevInvalid)) == kStepValid || (c == 0 && lane == 0));
  };
  if (lane == 0) {
    issue(0);
    if (nch > 1) issue(1);
  }
  uint32_t pk;
  bool fast;
  params(0, base_of(0), pk, fast);
  int bnext = base_of(1);
  uint32_t phase = 0u;  // bit b: parity of buffer b's next phase
  uint32_t L = 0;
  for (int c = 0; c < nch; ++c) {
    const int b = c % NB, n = chunk_n(c);
    if (!mbar_wait_warp(&bars[w][b], (phase >> b) & 1u)) {
      scan_give_up_mask(bars[w], phase, (1u << b) | (c + 1 < nch ? 1u << ((c + 1) % NB) : 0u));
      return;
    }
    phase ^= 1u << b;
    __syncwarp();
    const uint8_t* cb = cbuf[w][b] + lane;
    const int r0 = dir == 0 ? 0 : (C - 1) * D, dr = dir == 0 ? D : -D;  // row of step j: r0 + j * dr
    uint32_t cvr[C];
#pragma unroll
    for (int j = 0; j < C; ++j) cvr[j] = cb[r0 + j * dr];
    fence_proxy_async();  // this lane's reads of the buffer before the copy that refills it
    __syncwarp();
    if (lane == 0 && c + 2 < nch) issue(c + 2);
    uint8_t* op = orow + (size_t)chunk_x(c) * D + lane + (dir == 0 ? 0 : (n - 1) * D);  // step 0's byte
    const int od = dir == 0 ? D : -D;
    const int bn = bnext;
    bnext = base_of(c + 2);  // a chunk ahead (no load past the scanline)
    // this chunk's step parameters to every lane
    par[w][lane] = pk;
    __syncwarp();
    uint32_t q[C];
#pragma unroll
    for (int j = 0; j < C; ++j) q[j] = par[w][j];
    __syncwarp();
    if (fast) {  // a full chunk (a short one has skipped steps)
      params(c + 1, bn, pk, fast);
#pragma unroll
      for (int j = 0; j < C; ++j) {
        uint32_t Ls = L;
        scan_step_fast(Ls, cvr[j], (int)(int8_t)(q[j] & 0xFFu), q[j] >> 10, P.p1);
        L = (j == 0 && c == 0) ? cvr[0] : Ls;  // the first pixel of the scanline starts it
        op[j * od] = (uint8_t)L;
      }
    } else {
      params(c + 1, bn, pk, fast);
#pragma unroll
      for (int j = 0; j < C; ++j) {
        uint32_t Ls = L;
        scan_step(Ls, cvr[j], q[j] & 0x3FFu, q[j] >> 10, P.p1);
        L = (j == 0 && c == 0) ? cvr[0] : Ls;
        // a skipped step past a short chunk keeps L: it rewrites the chunk's last pixel
        op[min(j, n - 1) * od] = (uint8_t)L;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Vertical scans: warp (blockIdx.x * WPB + w) owns column x of view blockIdx.y and stores its path
// costs: PASS 1 bottom to top (bt), PASS 3 top to bottom (tb); the WTA follows in k_wta_init4, so
// both passes can run beside the row scans. Both start last_base from row 0's base
// (cusgm_ca.cu:1291); the first pixel of a vertical path does not set it. Chunks are swizzled
// tensor-map boxes of 32 rows x 32 bytes, as in k_vscan_plain4: PASS 1 boxes end at rows H - 32c
// (the last one starts above row 0 and reads zeros there; its steps past row 0 are marked
// skipped), PASS 3 boxes start at rows 32c. A step's path costs overwrite its costs in the box,
// which then leaves with one tensor store (a box that reaches past the column, row by row).
// ---------------------------------------------------------------------------------------------
// m_out / out: the volume the pass stores (bt or tb) as a tensor map and as a pointer.
template <int WPB, int PASS>
__global__ void __launch_bounds__(32 * WPB)
    k_vscan_init4(const __grid_constant__ CUtensorMap m_cost, const __grid_constant__ CUtensorMap m_out,
                  const int16_t* __restrict__ init_l, const int16_t* __restrict__ init_r, uint8_t* __restrict__ out,
                  InitParams P) {
  static_assert(PASS == 1 || PASS == 3, "bottom-to-top or top-to-bottom");
  constexpr int D = kLevelRange, C = kScanChunk, BOX = C * D;
  constexpr int NB = 3;  // chunks in flight
  constexpr bool kUp = PASS == 1;
  __shared__ __align__(1024) uint8_t cbuf[WPB][NB][BOX];
  __shared__ __align__(8) uint64_t bars[WPB][NB];
  __shared__ __align__(16) uint32_t par[WPB][2][C];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    for (int b = 0; b < NB; ++b) mbar_init(&bars[w][b], 1);
    mbar_fence_init();
  }
  __syncwarp();
  const int W = P.W, H = P.H;
  const int x = blockIdx.x * WPB + w;
  const int view = blockIdx.y;
  if (x >= W || x < P.x0) return;  // the whole warp
  // the swizzle pattern is a function of the shared address: the boxes must start on 1 KB
  if (smem_u32(&cbuf[0][0][0]) & 1023u) {
    if (lane == 0) atomicAdd(&g_scan_wait_timeouts, 1u);
    return;
  }
  const int16_t* ib = (view == 0 ? init_l : init_r) + x;
  const int nch = (H + C - 1) / C;
  auto chunk_n = [&](int c) { return min(C, H - c * C); };
  auto row_of = [&](int s) { return kUp ? H - 1 - s : s; };
  auto box_y = [&](int c) { return kUp ? H - C * (c + 1) : C * c; };  // first row of chunk c's box
  auto issue = [&](int c) {  // lane 0
    const int b = c % NB;
    mbar_expect_tx(&bars[w][b], BOX);
    tma_load_3d(cbuf[w][b], &m_cost, x * D, box_y(c), view, &bars[w][b]);
  };
  auto base_of = [&](int c) {
    const int n = chunk_n(c);
    return lane < n ? (int)ib[(size_t)row_of(c * C + lane) * W] : (int)kInvalidShort;
  };
  if (lane == 0) {
    issue(0);
    if (nch > 1) issue(1);
  }
  uint32_t phase = 0u;  // bit b: parity of buffer b's next phase
  ChunkState st{(int)ib[0], false};  // row 0's base
  int bnext = base_of(0);
  uint32_t L = 0;
  const int lo0 = lane, lo1 = lane ^ 16;  // this lane's byte of a box row under the two swizzles
  for (int c = 0; c < nch; ++c) {
    const int b = c % NB, n = chunk_n(c);
    const int bcur = bnext;
    if (c + 1 < nch) bnext = base_of(c + 1);
    uint32_t flags, p2;
    chunk_params(bcur, c * C, n, false, P, st, flags, p2);
    par[w][0][lane] = flags;
    par[w][1][lane] = p2;
    if (!mbar_wait_warp(&bars[w][b], (phase >> b) & 1u)) {
      scan_give_up_mask(bars[w], phase, (1u << b) | (c + 1 < nch ? 1u << ((c + 1) % NB) : 0u));
      if (lane == 0) bulk_wait_all();
      return;
    }
    phase ^= 1u << b;
    __syncwarp();
    uint8_t* box = cbuf[w][b];
    // step j: box row C - 1 - j (PASS 1) or j (PASS 3); this lane's byte of it
    auto at = [&](int j) {
      const int r = kUp ? C - 1 - j : j;
      return box + r * D + (box_sw<D>(r) ? lo1 : lo0);
    };
    // the chunk's step parameters and this lane's costs in registers: the chain below touches no
    // memory but the stores of its results
    uint32_t fl[C], pp[C], cvr[C];
#pragma unroll
    for (int j = 0; j < C; ++j) {
      fl[j] = par[w][0][j];
      pp[j] = par[w][1][j];
      cvr[j] = *at(j);
    }
    // all 32 steps run (steps past a short last chunk are marked skipped)
#pragma unroll
    for (int j = 0; j < C; ++j) {
      if (c == 0 && j == 0) L = cvr[0];
      else scan_step(L, cvr[j], fl[j], pp[j], P.p1);
      *at(j) = (uint8_t)L;
    }
    fence_proxy_async();
    __syncwarp();
    const int y0 = box_y(c);
    if (y0 >= 0 && y0 + C <= H) {
      if (lane == 0) {
        tma_store_3d(&m_out, x * D, y0, view, box);
        bulk_commit();
      }
    } else {  // a box reaching past row 0 or row H - 1: its rows inside the column, one per lane
      const int y = y0 + lane;
      if (y >= 0 && y < H) {
        const uint4* src = reinterpret_cast<const uint4*>(box + lane * D);
        uint4* dst = reinterpret_cast<uint4*>(out + (size_t)view * P.vstride + ((size_t)y * W + x) * D);
        const int sw = box_sw<D>(lane);
        const uint4 v0 = src[sw], v1 = src[sw ^ 1];
        dst[0] = v0;
        dst[1] = v1;
      }
    }
    if (lane == 0 && c + 2 < nch) {
      bulk_wait_read<1>();  // the store of chunk c - 1 has left the box chunk c + 2 goes to
      issue(c + 2);
    }
  }
  if (lane == 0) bulk_wait_all();
}

// WTA of one pixel of an initial-disparity level from its four stored path rows (32 bytes each,
// in global memory; S(d) = sum of the four): Kernel_ComputeDisparityByWTA for initial disparities
// (cusgm_ca.cu:3425-3512). d* <= 1 or d* >= 31 -> INVALID; uniqueness and the +0.5-shifted
// parabola as in wta_pixel; tie rules: kTieRefB200 the lowest tied d whose candidate is valid
// (every tied lane stores its own result there, a valid one wins), 1 / 2 the highest tied d, 0 / 3
// the lowest (one disparity per lane: lane order is disparity order). A row is read as two 16-byte
// words; S(d) is summed in 16-bit halves, its minimum taken by SIMD minima and the tied set kept as
// a bit mask; S at a candidate's neighbours comes from single bytes.
__device__ __forceinline__ float init_wta_rows(const uint8_t* a, const uint8_t* b, const uint8_t* c,
                                               const uint8_t* e, int base, const WtaParams& Q) {
  constexpr int D = kLevelRange;
  uint32_t lo[D / 4], hi[D / 4];  // lo[k] = S(4k) | S(4k + 2) << 16, hi[k] = S(4k + 1) | S(4k + 3) << 16
#pragma unroll
  for (int q = 0; q < D / 16; ++q) {
    const uint4 va = reinterpret_cast<const uint4*>(a)[q], vb = reinterpret_cast<const uint4*>(b)[q];
    const uint4 vc = reinterpret_cast<const uint4*>(c)[q], ve = reinterpret_cast<const uint4*>(e)[q];
    const uint32_t wa[4] = {va.x, va.y, va.z, va.w}, wb[4] = {vb.x, vb.y, vb.z, vb.w};
    const uint32_t wc[4] = {vc.x, vc.y, vc.z, vc.w}, we[4] = {ve.x, ve.y, ve.z, ve.w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      lo[4 * q + t] = __byte_perm(wa[t], 0u, 0x4240u) + __byte_perm(wb[t], 0u, 0x4240u) +
                      __byte_perm(wc[t], 0u, 0x4240u) + __byte_perm(we[t], 0u, 0x4240u);
      hi[4 * q + t] = __byte_perm(wa[t], 0u, 0x4341u) + __byte_perm(wb[t], 0u, 0x4341u) +
                      __byte_perm(wc[t], 0u, 0x4341u) + __byte_perm(we[t], 0u, 0x4341u);
    }
  }
  uint32_t mm = __vminu2(lo[0], hi[0]);
#pragma unroll
  for (int k = 1; k < D / 4; ++k) mm = __vminu2(mm, __vminu2(lo[k], hi[k]));
  const uint32_t m = min(mm & 0xFFFFu, mm >> 16), m2 = m * 0x10001u;
  uint32_t tied = 0;  // bit d: S(d) == m
#pragma unroll
  for (int k = 0; k < D / 4; ++k) {
    const uint32_t el = __vcmpeq2(lo[k], m2), eh = __vcmpeq2(hi[k], m2);
    tied |= ((el & 1u) | ((eh & 1u) << 1) | ((el >> 14) & 4u) | ((eh >> 13) & 8u)) << (4 * k);
  }
  const float ut = __fsub_rn(1.0f, Q.uniqueness);
  auto sum_at = [&](int d) { return (uint32_t)a[d] + b[d] + c[d] + e[d]; };
  auto candidate = [&](int d) {
    if (d <= 1 || d >= Q.dmax_excl) return kInvalidFloat;
    const float c1 = (float)sum_at(d - 1), c2 = (float)m, c3 = (float)sum_at(d + 1);
    const float d12 = __fsub_rn(c1, c2), d32 = __fsub_rn(c3, c2);
    const float uq = d12 < d32 ? d12 : d32;
    if (uq <= __fmul_rn(c2, ut)) return kInvalidFloat;
    return __fadd_rn((float)(d + base), subpix_bias(c1, c2, c3));
  };
  if (Q.tie_rule == kTieRefB200) {
    while (tied) {
      const float v = candidate(__ffs(tied) - 1);
      if (v != kInvalidFloat) return v;
      tied &= tied - 1u;
    }
    return kInvalidFloat;
  }
  const bool high = Q.tie_rule == kTieHighest || Q.tie_rule == kTieLaneHigh;
  return candidate(high ? 31 - __clz(tied) : __ffs(tied) - 1);
}

// WTA of an initial-disparity level, one thread per pixel, from the four stored path volumes:
// INVALID left of x0, on the image border, in rows >= Q.rows and where the pixel's base is
// INVALID.
__global__ void __launch_bounds__(128) k_wta_init4(const uint8_t* __restrict__ bt, const uint8_t* __restrict__ tb,
                                                   const uint8_t* __restrict__ lr, const uint8_t* __restrict__ rl,
                                                   const int16_t* __restrict__ init_l,
                                                   const int16_t* __restrict__ init_r, float* __restrict__ disp,
                                                   InitParams P, WtaParams Q) {
  constexpr int D = kLevelRange;
  const int x = blockIdx.x * 128 + threadIdx.x, y = blockIdx.y, view = blockIdx.z;
  const int W = P.W;
  if (x >= W) return;
  float dv = kInvalidFloat;
  if (x >= P.x0 && x >= Q.xlo && x <= Q.xhi && y >= Q.ylo && y <= Q.yhi && y < Q.rows) {
    const int base = (view == 0 ? init_l : init_r)[(size_t)y * W + x];
    if (base != kInvalidShort) {
      const size_t o = (size_t)view * P.vstride + ((size_t)y * W + x) * D;
      dv = init_wta_rows(tb + o, bt + o, lr + o, rl + o, base, Q);
    }
  }
  disp[(size_t)view * Q.dstride + (size_t)y * W + x] = dv;
}

}  // namespace sgm

namespace sgm {

// =============================================================================================
// Plain levels (no initial disparities), latency form. One warp owns a scanline; lane l holds the
// K consecutive disparities d = K l + k in 32 bits, the reference's lane mapping
// (Kernel_Aggregate_*_Warpfor{32,64,128}, cusgm_ca.cu:1343-1888). A step:
//   m = min_d L(d)                       one redux.sync of the lanes' K-wide minima
//   L(d - 1) + P1, L(d + 1) + P1         in the lane, or one shuffle up / down at its edges
//   L'(d) = C(d) + min(L(d), L(d-1) + P1 | 127, L(d+1) + P1 | 127, m + P2) - m
// and a lane moves its K bytes of costs and path costs as one 8/16/32-bit shared access.
// Chunks of 32 steps move between global and shared memory with bulk async copies; a step's path
// costs overwrite its costs in the chunk buffer, which then leaves with a bulk store (rows: one
// contiguous copy; columns: one tensor-map box of 32 rows), three buffers deep so a load never
// waits for the store of the chunk before. Every chunk runs all 32 steps: the steps past a scanline's end read and
// write rows of the buffer that hold nothing of this scanline and are neither stored nor used.
// The WTA of the top-to-bottom pass runs per chunk with lane = pixel.
// =============================================================================================

// A lane's K bytes of a step row, as one shared-memory word.
template <int K>
using LaneBytes = std::conditional_t<K == 1, uint8_t, std::conditional_t<K == 2, uint16_t, uint32_t>>;

template <int K>
__device__ __forceinline__ void unpack_bytes(uint32_t w, uint32_t (&c)[K]) {
#pragma unroll
  for (int k = 0; k < K; ++k) c[k] = k == 0 && K == 1 ? w : __byte_perm(w, 0u, 0x4440u + k);
}
template <int K>
__device__ __forceinline__ uint32_t pack_bytes(const uint32_t (&L)[K]) {
  if constexpr (K == 1) return L[0];
  if constexpr (K == 2) return __byte_perm(L[0], L[1], 0x0040u);
  if constexpr (K == 4) return __byte_perm(__byte_perm(L[0], L[1], 0x0040u), __byte_perm(L[2], L[3], 0x0040u), 0x5410u);
  return 0u;
}

template <int K>
__device__ __forceinline__ void plain_step4(uint32_t (&L)[K], const uint32_t (&c)[K], uint32_t p1, uint32_t p2) {
  const int lane = threadIdx.x & 31;
  uint32_t lm = L[0];
#pragma unroll
  for (int k = 1; k < K; ++k) lm = min(lm, L[k]);
  const uint32_t m = __reduce_min_sync(kFull, lm);
  uint32_t Lp[K];
#pragma unroll
  for (int k = 0; k < K; ++k) Lp[k] = L[k] + p1;
  const uint32_t up = __shfl_up_sync(kFull, Lp[K - 1], 1);  // L(K l - 1) + P1 from lane l - 1
  const uint32_t dn = __shfl_down_sync(kFull, Lp[0], 1);    // L(K l + K) + P1 from lane l + 1
  const uint32_t a0 = lane > 0 ? up : kInvalidCost;
  const uint32_t bK = lane < 31 ? dn : kInvalidCost;
  const uint32_t l4 = m + p2;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const uint32_t A = k == 0 ? a0 : Lp[k - 1];
    const uint32_t B = k == K - 1 ? bK : Lp[k + 1];
    const uint32_t t = min(__vimin3_u32(L[k], A, B), l4);
    L[k] = c[k] + t - m;
  }
}

// The 32 steps of a chunk held in shared memory: at step j this lane reads its K bytes of costs
// at at(j) (a LaneBytes<K> pointer) and leaves its path costs there. first: step 0 starts the
// scanline (L = C). Costs are read R steps ahead.
template <int K, typename At>
__device__ __forceinline__ void plain_chunk(At at, bool first, uint32_t (&L)[K], uint32_t p1, uint32_t p2) {
  constexpr int C = kScanChunk, R = 16;
  uint32_t ring[R];
#pragma unroll
  for (int j = 0; j < R; ++j) ring[j] = *at(j);
#pragma unroll
  for (int j = 0; j < C; ++j) {
    uint32_t c[K];
    unpack_bytes<K>(ring[j % R], c);
    if (j + R < C) ring[j % R] = *at(j + R);
    if (j == 0 && first) {
#pragma unroll
      for (int k = 0; k < K; ++k) L[k] = c[k];
    } else {
      plain_step4<K>(L, c, p1, p2);
    }
    *at(j) = (LaneBytes<K>)pack_bytes<K>(L);
  }
}

// Horizontal scans of a plain level; warp (blockIdx.x * WPB + w) owns scanline i = (view, dir, y)
// as in hpaths3_lane. A chunk is 32 consecutive pixels of the row: one contiguous bulk copy in,
// one out. Right-to-left scans place a short (last) chunk at the end of the buffer, so that step
// j of every chunk reads row 31 - j.
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
  auto chunk_off = [&](int c) { return dir == 0 ? 0 : (C - chunk_n(c)) * D; };  // bytes into the buffer
  auto issue = [&](int c) {  // lane 0
    const int b = c % NB;
    const uint32_t bytes = (uint32_t)chunk_n(c) * D;
    mbar_expect_tx(&bars[w][b], bytes + (c == 0 && g_short_copy ? 16u : 0u));
    bulk_to_smem(cbuf[w][b] + chunk_off(c), crow + (size_t)chunk_x(c) * D, bytes, &bars[w][b]);
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
    LaneBytes<K>* lb = reinterpret_cast<LaneBytes<K>*>(cbuf[w][b]) + lane;
    if (dir == 0)
      plain_chunk<K>([lb](int j) { return lb + j * 32; }, c == 0, L, P.p1, P.p2);
    else
      plain_chunk<K>([lb](int j) { return lb + (C - 1 - j) * 32; }, c == 0, L, P.p1, P.p2);
    fence_proxy_async();  // the chunk's path costs (and its cost reads) before the bulk copies
    __syncwarp();
    if (lane == 0) {
      bulk_to_global(orow + (size_t)chunk_x(c) * D, cbuf[w][b] + chunk_off(c), (uint32_t)n * D);
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
// Kernel_ComputeDisparityByWTA_Warpfor{32,64,128} (cusgm_ca.cu:3514-3809). S(d) (at most 4 x 255)
// is summed in 16-bit halves and searched as the 16-bit key S(d) * 64 + (d mod 64) -- the lowest
// key of a block of 64 disparities is its minimum at its lowest d (with 63 - (d mod 64): at its
// highest d). d* = 0 or d* >= Q.dmax_excl -> INVALID; c3 at d* = D - 1 is the index itself;
// uniqueness and the +0.5-shifted parabola as in wta_pixel. Tie rules: kTieRefB200 at D = 64
// (A = {t < 32 : S(t) = m}, B = {t < 32 : S(t + 32) = m, S(t) != m}; even rows of the launch take
// the lowest of B (+ 32) if any, else of A; odd rows the lowest of A if any, else of B (+ 32));
// kTieHighest the highest tied d; the rest the lowest.
// a, b, c, e: the pixel's rows in four swizzled boxes (16-byte unit u of the row at u ^ sw).
template <int D>
__device__ __forceinline__ float plain_wta_rows(const uint8_t* a, const uint8_t* b, const uint8_t* c,
                                                const uint8_t* e, int sw, int min_d, int y, const WtaParams& Q) {
  constexpr int SPLIT = D == 64 ? 32 : 64;  // first d of the second key block (D = 64: A / B halves)
  const bool high = Q.tie_rule == kTieHighest;
  const uint32_t flip = high ? 63u * 0x10001u : 0u;
  uint32_t acc0 = 0xFFFFFFFFu, acc1 = 0xFFFFFFFFu;
#pragma unroll
  for (int q = 0; q < D / 16; ++q) {
    const int u = q ^ sw;
    const uint4 va = reinterpret_cast<const uint4*>(a)[u], vb = reinterpret_cast<const uint4*>(b)[u];
    const uint4 vc = reinterpret_cast<const uint4*>(c)[u], ve = reinterpret_cast<const uint4*>(e)[u];
    const uint32_t wa[4] = {va.x, va.y, va.z, va.w}, wb[4] = {vb.x, vb.y, vb.z, vb.w};
    const uint32_t wc[4] = {vc.x, vc.y, vc.z, vc.w}, we[4] = {ve.x, ve.y, ve.z, ve.w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int d0 = 16 * q + 4 * t;  // the word's first disparity
      // lo = S(d0) | S(d0 + 2) << 16, hi = S(d0 + 1) | S(d0 + 3) << 16
      const uint32_t lo = __byte_perm(wa[t], 0u, 0x4240u) + __byte_perm(wb[t], 0u, 0x4240u) +
                          __byte_perm(wc[t], 0u, 0x4240u) + __byte_perm(we[t], 0u, 0x4240u);
      const uint32_t hi = __byte_perm(wa[t], 0u, 0x4341u) + __byte_perm(wb[t], 0u, 0x4341u) +
                          __byte_perm(wc[t], 0u, 0x4341u) + __byte_perm(we[t], 0u, 0x4341u);
      const uint32_t dlo = (uint32_t)(d0 & 63) | ((uint32_t)((d0 + 2) & 63) << 16);
      const uint32_t dhi = dlo + 0x10001u;
      const uint32_t klo = (lo << 6) | (dlo ^ flip), khi = (hi << 6) | (dhi ^ flip);
      if (d0 < SPLIT) acc0 = __vimin3_u16x2(acc0, klo, khi);
      else acc1 = __vimin3_u16x2(acc1, klo, khi);
    }
  }
  const uint32_t k0 = min(acc0 & 0xFFFFu, acc0 >> 16), k1 = min(acc1 & 0xFFFFu, acc1 >> 16);
  const uint32_t s0 = k0 >> 6, s1 = k1 >> 6;
  // the disparities of the two keys (block 1 of D = 128 starts at 64; D = 64's halves share d mod 64 = d)
  const int t0 = (int)((k0 & 63u) ^ (flip & 63u)), t1 = (D == 128 ? 64 : 0) + (int)((k1 & 63u) ^ (flip & 63u));
  uint32_t m;
  int ds;
  if constexpr (D == 32) {
    m = s0;
    ds = t0;
  } else {
    m = min(s0, s1);
    // the lowest (highest) tied d of the two blocks
    ds = s0 < s1 || (s0 == s1 && !high) ? t0 : t1;
    if (D == 64 && Q.tie_rule == kTieRefB200 && s0 == s1) {
      // both halves hold the minimum: odd rows take A's lowest (t0); even rows B's lowest if B is
      // not empty (a t with S(t + 32) = m and S(t) != m; rare, searched directly)
      ds = t0;
      if ((y & 1) == 0) {
        for (int t = 0; t < 32; ++t) {
          const int ob = (t + 32) ^ (sw << 4), oa = t ^ (sw << 4);
          const uint32_t sb = (uint32_t)a[ob] + b[ob] + c[ob] + e[ob];
          const uint32_t sa = (uint32_t)a[oa] + b[oa] + c[oa] + e[oa];
          if (sb == m && sa != m) {
            ds = t + 32;
            break;
          }
        }
      }
    }
  }
  if (ds <= 0 || ds >= Q.dmax_excl) return kInvalidFloat;
  auto sum_at = [&](int d) {
    const int o = d ^ (sw << 4);
    return (uint32_t)a[o] + b[o] + c[o] + e[o];
  };
  const float c1 = (float)sum_at(ds - 1);
  const float c2 = (float)m;
  const float c3 = (ds + 1 < D) ? (float)sum_at(ds + 1) : (float)ds;
  const float d12 = __fsub_rn(c1, c2), d32 = __fsub_rn(c3, c2);
  const float uq = d12 < d32 ? d12 : d32;
  if (uq <= __fmul_rn(c2, __fsub_rn(1.0f, Q.uniqueness))) return kInvalidFloat;
  return __fadd_rn((float)(ds + min_d), subpix_bias(c1, c2, c3));
}

// Warps per CTA of the column kernels (shared memory per warp: PASS 1 three boxes, PASS 2 two
// boxes of costs and three of stored paths, C x D bytes each).
template <int K>
__host__ __device__ constexpr int vscan_plain4_warps() { return K == 4 ? 2 : 4; }

// Vertical scans of a plain level: warp (blockIdx.x * WPB + w) owns column x of view blockIdx.y.
// PASS 1: bottom to top over boxes ending at rows H - 32c (the last one starts above row 0 and
// reads zeros there), storing its path costs (bt) box by box -- the last box row by row. PASS 2:
// top to bottom over boxes starting at rows 32c, then per box the WTA of its pixels with lane =
// pixel (rows >= Q.rows INVALID, as the reference's two-row WTA blocks leave them; border and
// columns left of x0 INVALID). Maps: the cost, bt, lr and rl volumes, [views][H][W * D] bytes.
template <int K, int PASS>
__global__ void __launch_bounds__(32 * vscan_plain4_warps<K>())
    k_vscan_plain4(const __grid_constant__ CUtensorMap m_cost, const __grid_constant__ CUtensorMap m_bt,
                   const __grid_constant__ CUtensorMap m_lr, const __grid_constant__ CUtensorMap m_rl,
                   uint8_t* __restrict__ bt, float* __restrict__ disp, PlainParams P, WtaParams Q) {
  constexpr int D = 32 * K, C = kScanChunk, BOX = C * D, NSW = D / 16;
  constexpr int WPB = vscan_plain4_warps<K>();
  constexpr int NB = PASS == 1 ? 3 : 2;  // cost boxes
  constexpr int NS = PASS == 1 ? 0 : 3;  // stored-path boxes (bt, lr, rl)
  __shared__ __align__(1024) uint8_t cbuf[WPB][NB + NS][BOX];
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
  // the swizzle pattern is a function of the shared address: the boxes must start on 1 KB
  if (smem_u32(&cbuf[0][0][0]) & 1023u) {
    if (lane == 0) atomicAdd(&g_scan_wait_timeouts, 1u);
    return;
  }
  const int nch = (H + C - 1) / C;
  auto box_y = [&](int c) { return PASS == 1 ? H - C * (c + 1) : C * c; };  // first row of chunk c's box
  auto issue_cost = [&](int c) {  // lane 0
    const int b = c % NB;
    mbar_expect_tx(&bars[w][b], BOX);
    tma_load_3d(cbuf[w][b], &m_cost, x * D, box_y(c), view, &bars[w][b]);
  };
  auto issue_paths = [&](int c) {  // lane 0
    mbar_expect_tx(&bars[w][NB], 3 * BOX);
    tma_load_3d(cbuf[w][NB + 0], &m_bt, x * D, box_y(c), view, &bars[w][NB]);
    tma_load_3d(cbuf[w][NB + 1], &m_lr, x * D, box_y(c), view, &bars[w][NB]);
    tma_load_3d(cbuf[w][NB + 2], &m_rl, x * D, box_y(c), view, &bars[w][NB]);
  };
  if (lane == 0) {
    issue_cost(0);
    if (nch > 1) issue_cost(1);
    if (PASS == 2) issue_paths(0);
  }
  // this lane's K bytes of a box row under each of the NSW swizzle patterns
  int lane_off[NSW];
#pragma unroll
  for (int v = 0; v < NSW; ++v) lane_off[v] = (K * lane) ^ (v << 4);
  uint32_t phase = 0u;  // bit b: parity awaited on bars[w][b]
  uint32_t L[K];
  const bool col_ok = x >= Q.xlo && x <= Q.xhi;
  for (int c = 0; c < nch; ++c) {
    const int b = c % NB;
    const uint32_t pend_cost = (1u << b) | (c + 1 < nch ? 1u << ((c + 1) % NB) : 0u);
    if (!mbar_wait_warp(&bars[w][b], (phase >> b) & 1u)) {
      scan_give_up_mask(bars[w], phase, pend_cost | (PASS == 2 ? 1u << NB : 0u));
      if (lane == 0) bulk_wait_all();
      return;
    }
    phase ^= 1u << b;
    __syncwarp();
    uint8_t* box = cbuf[w][b];
    // step j: box row C - 1 - j (PASS 1) or j (PASS 2)
    plain_chunk<K>(
        [&](int j) {
          const int r = PASS == 1 ? C - 1 - j : j;
          return reinterpret_cast<LaneBytes<K>*>(box + r * D + lane_off[box_sw<D>(r)]);
        },
        c == 0, L, P.p1, P.p2);
    if constexpr (PASS == 1) {
      fence_proxy_async();
      __syncwarp();
      const int y0 = box_y(c);
      if (y0 >= 0) {
        if (lane == 0) {
          tma_store_3d(&m_bt, x * D, y0, view, box);
          bulk_commit();
        }
      } else if (lane < C + y0) {  // the top box: rows 0 .. C + y0 - 1 of the column, one per lane
        const int r = lane - y0;     // box row of image row `lane`
        const uint4* src = reinterpret_cast<const uint4*>(box + r * D);
        uint4* dst = reinterpret_cast<uint4*>(bt + (size_t)view * P.vstride + ((size_t)lane * W + x) * D);
#pragma unroll
        for (int u = 0; u < NSW; ++u) dst[u] = src[u ^ box_sw<D>(r)];
      }
      if (lane == 0 && c + 2 < nch) {
        bulk_wait_read<1>();  // the store of chunk c - 1 has left the box chunk c + 2 goes to
        issue_cost(c + 2);
      }
    } else {
      __syncwarp();  // the chunk's path costs, written by disparity, are read by pixel
      if (!mbar_wait_warp(&bars[w][NB], (phase >> NB) & 1u)) {
        scan_give_up_mask(bars[w], phase, (1u << NB) | (c + 1 < nch ? 1u << ((c + 1) % NB) : 0u));
        return;
      }
      phase ^= 1u << NB;
      const int y = C * c + lane;
      if (y < H) {
        float dv = kInvalidFloat;
        if (col_ok && y >= Q.ylo && y <= Q.yhi && y < Q.rows)
          dv = plain_wta_rows<D>(box + lane * D, cbuf[w][NB] + lane * D, cbuf[w][NB + 1] + lane * D,
                                 cbuf[w][NB + 2] + lane * D, box_sw<D>(lane), P.min_d, y, Q);
        dout[(size_t)y * W] = dv;
      }
      fence_proxy_async();  // the reads of the boxes before the copies that refill them
      __syncwarp();
      if (lane == 0) {
        if (c + 1 < nch) issue_paths(c + 1);
        if (c + 2 < nch) issue_cost(c + 2);
      }
    }
  }
  if (PASS == 1 && lane == 0) bulk_wait_all();
}

}  // namespace sgm
