// Asynchronous copies between global and shared memory for the scan kernels: bulk copies and
// tensor-map (TMA) box copies completing on mbarriers, bulk stores, and bounded waits.
//
// Every wait on an mbarrier is bounded: after kMaxWaitTries polls the caller records the timeout
// in g_scan_wait_timeouts (one counter per translation unit, read back by the host) and stops.
// No copy here uses cluster multicast; every source and destination is this GPU's own memory.
#pragma once
#include <cuda.h>  // CUtensorMap
#include <cstdint>

namespace sgm {

constexpr int kScanChunk = 32;          // steps per staged chunk
constexpr int kMaxWaitTries = 1 << 22;  // polls of an mbarrier before a wait is given up

static __device__ unsigned int g_scan_wait_timeouts;
// Tests of the give-up path (set by sgm_debug_scan_wait): the poll limit of every wait, and a
// switch that makes the plain row scans expect 16 bytes more than their first copy delivers, so
// that wait runs out.
static __device__ unsigned int g_wait_limit = kMaxWaitTries;
static __device__ unsigned int g_short_copy;

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
// Waits for the phase of bar with the given parity; false after g_wait_limit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const unsigned int limit = g_wait_limit;
  for (unsigned int it = 0; it < limit; ++it) {
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
  return __all_sync(0xFFFFFFFFu, mbar_wait(bar, parity));
}
// A wait that ran out: record it, then wait (again bounded) for the copies still in flight into
// this warp's buffers -- those whose bit is set in `pending` (bit b: bars[b]; phase bit b: the
// parity bars[b] waits for next) -- before the warp leaves.
__device__ __forceinline__ void scan_give_up_mask(uint64_t* bars, uint32_t phase, uint32_t pending) {
  if ((threadIdx.x & 31) == 0) atomicAdd(&g_scan_wait_timeouts, 1u);
  for (int b = 0; b < 32; ++b)
    if ((pending >> b) & 1u) mbar_wait(bars + b, (phase >> b) & 1u);
}

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


// Column chunks are boxes of 32 rows x D bytes of one view's volume, copied by the tensor-memory
// accelerator (a 3D tensor map: bytes of a row, rows, views) with the 32/64/128-byte swizzle: the
// 16-byte unit u of box row r lands at unit u ^ box_sw(r) (bits 4.. of the shared address XORed
// with bits 7..), so that 8 lanes reading 8 consecutive rows hit distinct banks.
template <int D>
__host__ __device__ constexpr int box_sw(int r) { return ((r * D) >> 7) & (D / 16 - 1); }

// One box from global memory (tensor coordinates x = byte of the row, y = row, z = view; rows
// outside the tensor read as 0), completing on bar.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// One box to global memory (y >= 0), in the calling thread's current bulk group.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(map),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}

}  // namespace sgm
