// Shared definitions for the SGM device code (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

namespace sgm {

constexpr float kInvalidFloat = -999999.0f;    // output invalid value (StereoCuda::get_invad_float)
constexpr int16_t kInvalidShort = -32768;      // initial-disparity invalid value (get_invad_short)
constexpr uint32_t kInvalidCost = 127;         // out-of-range neighbour candidate of the recurrence
constexpr int kLevelRange = 32;                // disparity range of every non-coarsest pyramid level
constexpr unsigned kFull = 0xFFFFFFFFu;

// kTieRefB200: what the reference build does on a B200 (measured from its dumps):
//   D=64 plain -- lanes t with S(t)==m store t, lanes with only S(t+32)==m store t+32; the lowest
//   lane wins within a store and the later store wins; the store order is t then t+32 on even rows
//   and t+32 then t on odd rows (the two rows of one WTA block compile differently).
//   other plain D -- lowest d. Initial-disparity levels -- every tied lane stores its own result:
//   a valid disparity wins over INVALID, the lowest lane among valid ones.
enum TieRule : int { kTieLowest = 0, kTieHighest = 1, kTieLaneHigh = 2, kTieLaneLow = 3, kTieRefB200 = 4 };
enum PeaksAbs : int { kPeaksAbsInt = 0, kPeaksAbsFloat = 1 };

__device__ __forceinline__ uint32_t popc_word(uint64_t v) { return __popcll(v); }
__device__ __forceinline__ uint32_t popc_word(uint32_t v) { return __popc(v); }

// CostAdjust of the initial-disparity cost: floor(e^k), k = 4*|d-16|/16 (integer division).
__device__ __forceinline__ uint32_t cost_adjust(int d) {
  int k = 4 * abs(d - kLevelRange / 2) / (kLevelRange / 2);
  k = k < 0 ? 0 : (k > 4 ? 4 : k);
  return k == 0 ? 1u : k == 1 ? 2u : k == 2 ? 7u : k == 3 ? 20u : 54u;
}

// Spreads the low 16 bits of v so that bit i moves to bit 2*i.
__device__ __forceinline__ uint32_t spread2(uint32_t v) {
  v &= 0xFFFFu;
  v = (v | (v << 8)) & 0x00FF00FFu;
  v = (v | (v << 4)) & 0x0F0F0F0Fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}
// Spreads the low 8 bits of v so that bit i moves to bit 4*i.
__device__ __forceinline__ uint32_t spread4(uint32_t v) {
  v &= 0xFFu;
  v = (v | (v << 12)) & 0x000F000Fu;
  v = (v | (v << 6)) & 0x03030303u;
  v = (v | (v << 3)) & 0x11111111u;
  return v;
}
// Spreads the low 4 bits of v so that bit i moves to bit 8*i.
__device__ __forceinline__ uint32_t spread8(uint32_t v) {
  v &= 0xFu;
  return (v & 1u) | ((v & 2u) << 7) | ((v & 4u) << 14) | ((v & 8u) << 21);
}

// Tie-break over a warp whose lane l holds disparities d = l*K + j (j < K).
// bal[j] has bit l set when S(l*K + j) equals the minimum. Returns the chosen d.
template <int K>
__device__ __forceinline__ int pick_tie(const uint32_t (&bal)[K], int rule, int y) {
  uint32_t any = 0;
#pragma unroll
  for (int j = 0; j < K; ++j) any |= bal[j];
  if (rule == kTieRefB200 && K != 2) rule = kTieLowest;
  if (rule == kTieLowest || rule == kTieHighest) {
    const int lane = rule == kTieLowest ? __ffs(any) - 1 : 31 - __clz(any);
    int best = -1;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const bool hit = (bal[j] >> lane) & 1u;
      if (rule == kTieLowest) { if (hit && best < 0) best = j; }
      else if (hit) best = j;
    }
    return lane * K + best;
  }
  // Rules defined on the d = t + 32*i mapping: word i holds bit t for d = 32*i + t.
  uint32_t word[K];
  if constexpr (K == 1) {
    word[0] = bal[0];
  } else if constexpr (K == 2) {
    // d = 2*l + j: word w covers lanes 16w..16w+15
#pragma unroll
    for (int w = 0; w < K; ++w)
      word[w] = spread2(bal[0] >> (16 * w)) | (spread2(bal[1] >> (16 * w)) << 1);
  } else if constexpr (K == 4) {
#pragma unroll
    for (int w = 0; w < K; ++w) {
      uint32_t acc = 0;
#pragma unroll
      for (int j = 0; j < K; ++j) acc |= spread4(bal[j] >> (8 * w)) << j;
      word[w] = acc;
    }
  } else {  // K == 8
#pragma unroll
    for (int w = 0; w < K; ++w) {
      uint32_t acc = 0;
#pragma unroll
      for (int j = 0; j < K; ++j) acc |= spread8(bal[j] >> (4 * w)) << j;
      word[w] = acc;
    }
  }
  if (rule == kTieRefB200) {  // K == 2 only (D = 64)
    const uint32_t A = word[0], B = word[K - 1] & ~word[0];
    if ((y & 1) == 0) return B ? (__ffs(B) - 1 + 32) : (__ffs(A) - 1);
    return A ? (__ffs(A) - 1) : (__ffs(B) - 1 + 32);
  }
  uint32_t ref_any = 0;
#pragma unroll
  for (int w = 0; w < K; ++w) ref_any |= word[w];
  const int t = rule == kTieLaneHigh ? 31 - __clz(ref_any) : __ffs(ref_any) - 1;
  int best = -1;
#pragma unroll
  for (int w = 0; w < K; ++w)
    if (best < 0 && ((word[w] >> t) & 1u)) best = w;
  return t + 32 * best;
}

// Asks for the largest shared-memory carveout for kernel `fn`. An SM changes its shared memory /
// L1 split only when it is idle, so kernels that run side by side (the row scans beside the column
// passes of one level) are placed best when none of them leaves an SM configured for less shared
// memory than another needs: measured on B200 with a 32-disparity level's row scan launched before
// its two column passes, the columns took 169 instead of 110 µs. Once per (function, device).
template <typename F>
inline cudaError_t prefer_max_shared(F* fn) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t st = cudaGetDevice(&dev);
  if (st != cudaSuccess) return st;
  const void* f = reinterpret_cast<const void*>(fn);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({f, dev})) return cudaSuccess;
  st = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  if (st == cudaSuccess) done.insert({f, dev});
  return st;
}

// Lets kernel `fn` launch with as much dynamic shared memory as the device allows. The limit is a
// per-function attribute shared by every launcher in the process (other matchers, other host
// threads), so it is always raised to the device maximum instead of being set to the size of one
// launch, which could undercut a concurrent launch that needs more.
// Done once per (function, device); later calls are a set lookup.
template <typename F>
inline cudaError_t allow_max_dynamic_smem(F* fn) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0, optin = 0;
  cudaError_t st = cudaGetDevice(&dev);
  if (st != cudaSuccess) return st;
  const void* f = reinterpret_cast<const void*>(fn);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({f, dev})) return cudaSuccess;
  st = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (st == cudaSuccess) st = cudaFuncGetAttributes(&fa, f);
  if (st == cudaSuccess)
    st = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  if (st == cudaSuccess) done.insert({f, dev});
  return st;
}

// Parabola through (d-1,c1), (d,c0), (d+1,c2); the reference's SubPixBias.
__device__ __forceinline__ float subpix_bias(float c1, float c0, float c2) {
  float den = __fsub_rn(__fadd_rn(c1, c2), __fmul_rn(2.0f, c0));
  den = den < 1.0f ? 1.0f : den;
  return __fdiv_rn(__fadd_rn(__fsub_rn(c1, c2), den), __fmul_rn(2.0f, den));
}

}  // namespace sgm
