// sgm_match_noalloc: single-level matching that allocates no memory.
//
// Who needs this: callers that may not allocate device memory once they are running -- real-time
// loops that forbid allocation after start-up (an allocation can block for milliseconds and
// synchronise the device), and plugin hosts that own the GPU memory budget and give a plugin only
// the buffers it is handed. They cannot use sgm_init, which allocates the matcher's working
// buffers with cudaMalloc.
//
// This entry point keeps all of its working memory (census words, cost and path volumes,
// disparity maps) in one file-scope __device__ array of kNoAllocScratchBytes (64 MiB). Every
// GPU that loads this module holds that array until the process exits. Calls share it: a call
// leaves its intermediate results there, and two calls whose work overlaps on the GPU (for
// example on two streams) race on it. Nothing in the array needs to start at zero -- every
// stage writes its whole output before the next stage reads it.
//
// Set-up: the first call on each device (that device current) looks up the device address of the
// array with cudaGetSymbolAddress, loads every kernel the entry point launches and sets their
// shared-memory limits, checking each result, and caches the address; later calls on that device
// make no set-up call. Make that first call before any stream capture begins.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/sgm_b200.h"
#include "sgm_kernels.cuh"

// Records the message returned by sgm_last_error(NULL) (defined with the engine).
void sgm_set_process_error(const char* msg);

namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;
int fail(int code, const char* fmt, ...) {
  char buf[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  sgm_set_process_error(buf);
  return code;
}

// Loads a kernel on the current device (cudaFuncGetAttributes forces the module load).
template <typename F>
cudaError_t load_kernel(F* fn) {
  cudaFuncAttributes a;
  return cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(fn));
}

// Every kernel the entry point launches, loaded on the current device, with the row kernels'
// dynamic shared-memory limit raised; stops at the first failure.
cudaError_t prepare_kernels() {
  cudaError_t st = cudaSuccess;
  auto chk = [&](cudaError_t e) { if (st == cudaSuccess) st = e; };
  chk(load_kernel(sgm::k_census<uint64_t, 4, 3>));
  chk(load_kernel(sgm::k_census<uint32_t, 2, 2>));
  chk(sgm::allow_max_dynamic_smem(sgm::k_hpaths_plain<1, uint64_t>));
  chk(sgm::allow_max_dynamic_smem(sgm::k_hpaths_plain<2, uint64_t>));
  chk(sgm::allow_max_dynamic_smem(sgm::k_hpaths_plain<4, uint64_t>));
  chk(sgm::allow_max_dynamic_smem(sgm::k_hpaths_plain<1, uint32_t>));
  chk(sgm::allow_max_dynamic_smem(sgm::k_hpaths_plain<2, uint32_t>));
  chk(sgm::allow_max_dynamic_smem(sgm::k_hpaths_plain<4, uint32_t>));
  chk(load_kernel(sgm::k_vpaths_wta_plain<1>));
  chk(load_kernel(sgm::k_vpaths_wta_plain<2>));
  chk(load_kernel(sgm::k_vpaths_wta_plain<4>));
  chk(load_kernel(sgm::k_lr_median<true, true>));
  chk(load_kernel(sgm::k_lr_median<true, false>));
  chk(load_kernel(sgm::k_lr_median<false, true>));
  return st;
}

// Device address of the scratch array on the current device. The first call on a device looks
// it up and prepares the kernels (see the file comment); later calls only read the cache.
int scratch_address(unsigned char** out) {
  int dev = 0;
  cudaError_t st = cudaGetDevice(&dev);
  if (st != cudaSuccess) return fail(SGM_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(st));
  if (dev < 0 || dev >= kMaxDevices) return fail(SGM_ERR_UNSUPPORTED, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    st = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (st != cudaSuccess || !p)
      return fail(SGM_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(st));
    st = prepare_kernels();
    if (st != cudaSuccess) return fail(SGM_ERR_CUDA, "kernel set-up failed: %s", cudaGetErrorString(st));
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
  return SGM_OK;
}

// Status of the launch just issued (the entry point has checked that no earlier error was pending).
int launched(const char* what) {
  const cudaError_t st = cudaGetLastError();
  return st == cudaSuccess ? SGM_OK : fail(SGM_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(st));
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

template <int K, typename Word>
int run(const uint8_t* dl, const uint8_t* dr, float* dout, int W, int H, int M, const sgm_option_t* o,
        unsigned char* scratch, cudaStream_t s) {
  constexpr int D = 32 * K;
  const int nv = o->do_lr_check ? 2 : 1;
  const size_t N = (size_t)W * H, V = N * D;
  // carve the scratch array
  size_t off = 0;
  Word* cs[2];
  for (int i = 0; i < 2; ++i) { cs[i] = reinterpret_cast<Word*>(scratch + off); off += align256(N * sizeof(Word)); }
  uint8_t* cost = scratch + off; off += align256(nv * V);
  uint8_t* lr = scratch + off;   off += align256(nv * V);
  uint8_t* rl = scratch + off;   off += align256(nv * V);
  uint8_t* bt = scratch + off;   off += align256(nv * V);
  float* wta = reinterpret_cast<float*>(scratch + off); off += align256(2 * N * sizeof(float));
  (void)off;
  int st;
  {
    dim3 g((W + 127) / 128, H, 2), b(128);
    if (sizeof(Word) == 8)
      sgm::k_census<uint64_t, 4, 3><<<g, b, 0, s>>>(dl, dr, (uint64_t*)cs[0], (uint64_t*)cs[1], W, H);
    else
      sgm::k_census<uint32_t, 2, 2><<<g, b, 0, s>>>(dl, dr, (uint32_t*)cs[0], (uint32_t*)cs[1], W, H);
    if ((st = launched("census"))) return st;
  }
  sgm::PlainParams P;
  P.W = W; P.H = H; P.min_d = M; P.x0 = std::max(0, M);
  P.p1 = (uint32_t)o->p1; P.p2 = (uint32_t)o->p2_init;
  P.vstride = V;
  int R = 4;
  while (R > 1 && (size_t)W * 2 * sizeof(Word) * R > 160 * 1024) R >>= 1;
  const size_t hsmem = (size_t)R * 2 * W * sizeof(Word);
  if (hsmem > 227 * 1024) return fail(SGM_ERR_UNSUPPORTED, "image width %d too large", W);
  sgm::k_hpaths_plain<K, Word><<<dim3((H + R - 1) / R, nv), dim3(32, 2 * R), hsmem, s>>>(cs[0], cs[1], cost, lr, rl,
                                                                                         P);
  if ((st = launched("row scans"))) return st;
  sgm::WtaParams Q;
  Q.uniqueness = o->unique_threshold;
  Q.tie_rule = sgm::kTieRefB200;
  Q.rows = (H / 2) * 2;
  Q.dmax_excl = D;
  Q.dstride = N;
  Q.image_border(W, H);
  sgm::k_vpaths_wta_plain<K><<<dim3((W + 7) / 8, nv), dim3(32, 8), 0, s>>>(cost, lr, rl, bt, wta, P, Q);
  if ((st = launched("column scans"))) return st;
  const bool lrc = o->do_lr_check, med = o->do_median_filter;
  dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
  if (lrc && med)
    sgm::k_lr_median<true, true><<<g, b, 0, s>>>(wta, wta + N, nullptr, dout, W, H, o->lr_threshold);
  else if (lrc)
    sgm::k_lr_median<true, false><<<g, b, 0, s>>>(wta, wta + N, nullptr, dout, W, H, o->lr_threshold);
  else if (med)
    sgm::k_lr_median<false, true><<<g, b, 0, s>>>(wta, nullptr, nullptr, dout, W, H, 0.0f);
  if (lrc || med) return launched("left-right check / median");
  const cudaError_t ce = cudaMemcpyAsync(dout, wta, N * sizeof(float), cudaMemcpyDeviceToDevice, s);
  return ce == cudaSuccess ? SGM_OK : fail(SGM_ERR_CUDA, "disparity copy failed: %s", cudaGetErrorString(ce));
}

// Bytes of the scratch array one call uses (the carving in run()).
size_t required_bytes(int32_t width, int32_t height, int32_t disp_range, const sgm_option_t* option) {
  const size_t N = (size_t)width * height, V = N * disp_range;
  const size_t nv = option->do_lr_check ? 2 : 1;
  const size_t word = option->cs_type == 1 ? 8 : 4;
  return 2 * align256(N * word) + 4 * align256(nv * V) + align256(2 * N * sizeof(float));
}

}  // namespace

extern "C" {

int sgm_match_noalloc(const uint8_t* d_left, const uint8_t* d_right, float* d_disp_left, int32_t width,
                      int32_t height, int32_t min_disparity, int32_t disp_range, const sgm_option_t* option,
                      void* stream) {
  if (!d_left || !d_right || !d_disp_left || !option) return fail(SGM_ERR_ARG, "null pointer argument");
  if (width <= 0 || height <= 0) return fail(SGM_ERR_ARG, "image size error (w=%d h=%d)", width, height);
  if (disp_range != 32 && disp_range != 64 && disp_range != 128)
    return fail(SGM_ERR_UNSUPPORTED, "disparity range %d unsupported here (32, 64, 128)", disp_range);
  if (option->cs_type != 0 && option->cs_type != 1) return fail(SGM_ERR_ARG, "census type %d invalid", option->cs_type);
  if (option->p1 < 0 || option->p2_init < 0) return fail(SGM_ERR_ARG, "negative penalties");
  if ((size_t)width * height > (size_t)INT32_MAX / 2) return fail(SGM_ERR_ARG, "image too large");
  if (height > 65535) return fail(SGM_ERR_ARG, "image height %d above 65535", height);
  if (min_disparity >= width)
    return fail(SGM_ERR_ARG, "minimum disparity %d leaves no pixel of a %d-pixel row to match", min_disparity, width);
  if (option->do_remove_peaks || option->morphology_type != 0 || option->post_filter_type != 0)
    return fail(SGM_ERR_UNSUPPORTED, "small-region removal, morphology and post filters are not available without "
                                     "allocation; use sgm_init / sgm_match_device");
  const size_t need = required_bytes(width, height, disp_range, option);
  if (need > kNoAllocScratchBytes)
    return fail(SGM_ERR_ARG, "%dx%d with %d disparities needs %zu bytes of working memory; the no-allocation "
                             "entry point has %zu (use sgm_init / sgm_match_device)", width, height, disp_range,
                need, kNoAllocScratchBytes);
  unsigned char* scratch = nullptr;
  int st = scratch_address(&scratch);
  if (st) return st;
  // an error left by the caller's earlier work is reported as such, not taken for this call's
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return fail(SGM_ERR_CUDA, "a CUDA error from earlier work is pending: %s", cudaGetErrorString(pending));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool w64 = option->cs_type == 1;
  switch (disp_range) {
    case 32: return w64 ? run<1, uint64_t>(d_left, d_right, d_disp_left, width, height, min_disparity, option, scratch, s)
                        : run<1, uint32_t>(d_left, d_right, d_disp_left, width, height, min_disparity, option, scratch, s);
    case 64: return w64 ? run<2, uint64_t>(d_left, d_right, d_disp_left, width, height, min_disparity, option, scratch, s)
                        : run<2, uint32_t>(d_left, d_right, d_disp_left, width, height, min_disparity, option, scratch, s);
    default: return w64 ? run<4, uint64_t>(d_left, d_right, d_disp_left, width, height, min_disparity, option, scratch, s)
                        : run<4, uint32_t>(d_left, d_right, d_disp_left, width, height, min_disparity, option, scratch, s);
  }
}

}  // extern "C"
