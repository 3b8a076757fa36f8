// Host side of the SGM engine: device buffers, the launch sequence of one matching level,
// the on-device pyramid driver and the C ABI declared in include/sgm_b200.h.
//
// Reference orchestration being replaced: StereoCudaImpl::Init/Match/Release
// (SgmStereoCuda/StereoCudaImpl.cpp:128-546) and HierSgmCudaImpl (FasterStereoCuda/
// FasterStereoCuda.cpp:201-635). Differences by design: all allocation happens in init;
// a match is one stream of kernels with no host synchronisation inside it; small-region
// removal runs on the GPU; the pyramid keeps every level on the device.
#include <cuda.h>  // CUtensorMap, cuTensorMapEncodeTiled (looked up through the runtime)
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sgm_b200.h"
#include "sgm_alloc.h"
#include "sgm_kernels4.cuh"
#include "sgm_levels.h"
#include "sgm_tma.h"

namespace {

thread_local std::string g_last_error;

void set_error(std::string* dst, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  if (dst) *dst = buf;
}


sgm_ext_options_t default_ext() {
  sgm_ext_options_t e;
  e.tie_rule = sgm::kTieRefB200;
  e.init_tie_rule = sgm::kTieRefB200;
  e.peaks_strips = 0;
  e.peaks_abs_mode = sgm::kPeaksAbsInt;
  e.p2_div0 = -1;
  return e;
}

// Optional per-launch timing with CUDA events recorded on the launching stream
// (process-wide; enable from one thread while no match is in flight).
struct Profiler {
  bool on = false;
  struct Rec { const char* name; cudaEvent_t a, b; };
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;
  struct Stat { std::string name; int64_t launches = 0; double ms = 0.0; };
  std::vector<Stat> stats;
  cudaEvent_t take() {
    if (pool.empty()) {
      cudaEvent_t ev;
      cudaEventCreate(&ev);
      return ev;
    }
    cudaEvent_t ev = pool.back();
    pool.pop_back();
    return ev;
  }
  void collect() {
    for (auto& r : pending) {
      float ms = 0.f;
      cudaEventSynchronize(r.b);
      cudaEventElapsedTime(&ms, r.a, r.b);
      Stat* st = nullptr;
      for (auto& x : stats)
        if (x.name == r.name) st = &x;
      if (!st) {
        stats.push_back(Stat{r.name, 0, 0.0});
        st = &stats.back();
      }
      st->launches++;
      st->ms += ms;
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    pending.clear();
  }
};
Profiler g_prof;
std::mutex g_prof_mu;
thread_local cudaEvent_t t_prof_start = nullptr;
thread_local cudaStream_t t_prof_stream = nullptr;

void prof_start(cudaStream_t s) {
  if (!g_prof.on) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  t_prof_start = g_prof.take();
  t_prof_stream = s;
  cudaEventRecord(t_prof_start, s);
}

void prof_end(const char* name) {
  if (!g_prof.on || !t_prof_start) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  cudaEvent_t b = g_prof.take();
  cudaEventRecord(b, t_prof_stream);
  g_prof.pending.push_back(Profiler::Rec{name, t_prof_start, b});
  t_prof_start = nullptr;
  if (g_prof.pending.size() > 4096) g_prof.collect();
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return cudaSuccess;
  return sgm_dev_malloc(reinterpret_cast<void**>(p), count * sizeof(T));
}

template <typename T>
void dfree(T*& p) {
  if (p) sgm_dev_free(p);
  p = nullptr;
}

// Fault injection and live-allocation count of sgm_dev_malloc (process-wide).
std::mutex g_alloc_mu;
int64_t g_alloc_live = 0;
int64_t g_alloc_fail_after = -1;  // < 0: never fail; else allocations left before one fails

}  // namespace

// The per-launch profiler as the batched engines (sgm_batch.cu) use it: with it on, a batch run
// enqueues its kernels one after another on one stream, each between sgm_prof_start and
// sgm_prof_end.
bool sgm_prof_on() { return g_prof.on; }
void sgm_prof_start(cudaStream_t s) { prof_start(s); }
void sgm_prof_end(const char* name) { prof_end(name); }

cudaError_t sgm_dev_malloc(void** p, size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    if (g_alloc_fail_after == 0) {
      g_alloc_fail_after = -1;  // one failure per arming
      *p = nullptr;
      return cudaErrorMemoryAllocation;
    }
    if (g_alloc_fail_after > 0) --g_alloc_fail_after;
  }
  const cudaError_t st = cudaMalloc(p, bytes);
  if (st == cudaSuccess) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    ++g_alloc_live;
  }
  return st;
}

cudaError_t sgm_dev_free(void* p) {
  if (!p) return cudaSuccess;
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    --g_alloc_live;
  }
  return cudaFree(p);
}

void sgm_set_process_error(const char* msg) { set_error(nullptr, "%s", msg); }
int64_t sgm_float_wait_timeouts();  // float_sgm.cu

// One matching level (the state of one StereoCuda instance).
struct sgm_engine {
  bool ready = false;
  int dev = 0;
  int nsm = 148;  // SMs of the device (set in init)
  int W = 0, H = 0, M = 0, D = 0;
  sgm_option_t opt{};
  sgm_ext_options_t ext = default_ext();
  bool print_log = false;
  bool has_cam = false;
  sgm_camera_t cam{};
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;                       // the bottom-to-top column pass beside the row scans
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;  // around the side stream's work
  std::string err;
  int64_t launches = 0;
  // device buffers
  uint8_t* img[2] = {nullptr, nullptr};
  void* cs[2] = {nullptr, nullptr};
  uint8_t *cost = nullptr, *lr = nullptr, *rl = nullptr, *bt = nullptr;
  uint8_t* tb = nullptr;  // top-to-bottom path costs (warp-per-scanline column kernels; on first use)
  float* wta = nullptr;     // [2][H][W]
  float* post = nullptr;    // LR/median output
  float* post2 = nullptr;   // dilation output
  float* dr_out = nullptr;  // right map after the LR marks
  float* out = nullptr;     // final left map for the host path
  // map the depth of Match2 is taken from, set by every match (the final map, or the map before a
  // lone post filter / morphology step, see engine_enqueue)
  const float* depth_src = nullptr;
  int16_t* init[2] = {nullptr, nullptr};
  int16_t* init_tmp = nullptr;
  unsigned* key = nullptr;
  int* label = nullptr;
  int* count = nullptr;
  bool own_volumes = true;  // false: cost/lr/rl/bt belong to a batch arena
  int tune_rows = 0;        // rows per CTA of the row kernels (0: default)
  int tune_cols = 0;        // columns per CTA of the column kernels (0: default)
  int tune_bt_smem = 0;     // 1: keep bottom->top path costs in shared memory when they fit
  int tune_row_kernel = 0;  // 0: 3 when exact else 2; 1 whole-row census, 2 chunked, 3 u16x2 per scanline
  int tune_col_kernel = 0;  // 0: 3 when exact else 1; 1 plain loads, 2 prefetch ring, 3 u16x2 per column
  int tune_row_lanes = 0;   // variant 3: lanes per scanline (0: default)
  int tune_col_lanes = 0;
  bool bt_stored = true;    // the last match wrote the bottom->top volume to global memory
  // tensor maps of the cost, bt, lr, rl and tb volumes for the column kernels' box copies, and
  // what each was built for (base, W, H, D, views)
  CUtensorMap tmap[5];
  struct TmapKey {
    const void* base = nullptr;
    int W = 0, H = 0, D = 0, nv = 0;
  } tmap_key[5];
  // img[0], img[1] -> out captured as a CUDA graph after a first direct run (matches without
  // initial disparities or a right map); later matches copy in, launch it, copy out. One graph
  // per kernel mode (0: the matcher's tuning, 1: the latency kernels of KernelMode).
  cudaGraphExec_t gexec[2] = {};
  int direct_runs[2] = {};
  int64_t graph_launches[2] = {};
  cudaEvent_t done = nullptr;  // blocking-sync event of the synchronous host API (see wait_stream)
  // Stages of a match: an NVTX range each, and with print_log a CUDA event at every stage boundary
  // for the per-stage report of the synchronous host API.
  static constexpr int kMaxStages = 10;
  bool stage_timing = false;
  bool nvtx_open = false;
  int nstage = 0;
  cudaEvent_t stage_ev[kMaxStages] = {};
  const char* stage_name[kMaxStages] = {};
  void drop_graph() {
    for (int k = 0; k < 2; ++k) {
      if (gexec[k]) cudaGraphExecDestroy(gexec[k]);
      gexec[k] = nullptr;
      direct_runs[k] = 0;
    }
  }
  bool tuning_is_default() const {
    return !tune_rows && !tune_cols && !tune_bt_smem && !tune_row_kernel && !tune_col_kernel && !tune_row_lanes &&
           !tune_col_lanes;
  }

  int nviews() const { return opt.do_lr_check ? 2 : 1; }
  size_t npix() const { return (size_t)W * H; }
  size_t vol() const { return (size_t)W * H * D; }
  int census_bytes() const { return opt.cs_type == 1 ? 8 : 4; }

  void free_all() {
    drop_graph();
    if (done) cudaEventDestroy(done);
    done = nullptr;
    for (auto& ev : stage_ev) {
      if (ev) cudaEventDestroy(ev);
      ev = nullptr;
    }
    stage_timing = false;
    for (int i = 0; i < 2; ++i) {
      dfree(img[i]);
      dfree(init[i]);
      if (cs[i]) sgm_dev_free(cs[i]);
      cs[i] = nullptr;
    }
    if (own_volumes) {
      dfree(cost); dfree(lr); dfree(rl); dfree(bt);
    }
    cost = lr = rl = bt = nullptr;
    dfree(tb);
    dfree(wta); dfree(post); dfree(post2); dfree(dr_out); dfree(out);
    dfree(init_tmp); dfree(key); dfree(label); dfree(count);
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    if (side) cudaStreamDestroy(side);
    side = nullptr;
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    ev_fork = ev_join = nullptr;
    ready = false;
  }
};

namespace {

// Waits for everything enqueued on s so far, on a blocking-sync event: a thread that has to wait
// sleeps and leaves its core to the other threads (many matchers on many host threads). While
// keep_polling() (non-null) holds, the event is polled instead: that returns as soon as the work
// is done rather than when the sleeping thread is woken, about 0.2 ms sooner per call for one
// caller matching 1242x375 frames from page-locked buffers (whose copies do not block the thread).
// `ev` is the matcher's own event, created on first use on its device.
cudaError_t wait_stream(cudaStream_t s, cudaEvent_t* ev, bool (*keep_polling)() = nullptr) {
  if (!*ev) {
    const cudaError_t st = cudaEventCreateWithFlags(ev, cudaEventBlockingSync | cudaEventDisableTiming);
    if (st != cudaSuccess) return st;
  }
  cudaError_t st = cudaEventRecord(*ev, s);
  if (st != cudaSuccess) return st;
  while (keep_polling && keep_polling())
    if ((st = cudaEventQuery(*ev)) != cudaErrorNotReady) return st;
  return cudaEventSynchronize(*ev);
}

// Starts stage `name` of the match being enqueued (ends the previous one); name == nullptr ends
// the last stage. NVTX ranges cost next to nothing without a tool attached.
void stage_mark(sgm_engine* e, const char* name) {
  if (e->nvtx_open) nvtxRangePop();
  e->nvtx_open = name != nullptr;
  if (name) nvtxRangePushA(name);
  if (e->stage_timing && e->nstage < sgm_engine::kMaxStages) {
    cudaEventRecord(e->stage_ev[e->nstage], e->stream);
    e->stage_name[e->nstage++] = name;
  }
}

#define SGM_CUDA_TRY(e, expr)                                                          \
  do {                                                                                 \
    cudaError_t _st = (expr);                                                          \
    if (_st != cudaSuccess) {                                                          \
      set_error(&(e)->err, "%s failed: %s", #expr, cudaGetErrorString(_st));           \
      return _st == cudaErrorMemoryAllocation ? SGM_ERR_NOMEM : SGM_ERR_CUDA;          \
    }                                                                                  \
  } while (0)

int check_launch(sgm_engine* e, const char* what) {
  prof_end(what);
  e->launches++;
  const cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) {
    set_error(&e->err, "launch of %s failed: %s", what, cudaGetErrorString(st));
    return SGM_ERR_CUDA;
  }
  return SGM_OK;
}

// Launches `...` (a kernel launch expression) on stream s, timed when profiling is on.
#define SGM_LAUNCH(e, s, name, ...) (prof_start(s), __VA_ARGS__, check_launch(e, name))

bool supported_range(int D) { return D == 32 || D == 64 || D == 128 || D == 256; }

int validate(sgm_engine* e, int W, int H, int M, int D, const sgm_option_t* o) {
  if (W <= 0 || H <= 0 || D <= 0) {
    set_error(&e->err, "image size or disparity range error (w=%d h=%d d=%d)", W, H, D);
    return SGM_ERR_ARG;
  }
  // the reference's grids cover columns [max(0, min_disparity), W) (cusgm_ca.cu:3991-3999): an
  // empty range launches nothing sensible there, so it is refused here
  if (M >= W) {
    set_error(&e->err, "minimum disparity %d leaves no pixel of a %d-pixel row to match", M, W);
    return SGM_ERR_ARG;
  }
  if (!supported_range(D)) {
    set_error(&e->err, "disparity range %d unsupported (32, 64, 128, 256)", D);
    return SGM_ERR_UNSUPPORTED;
  }
  if (o->cs_type != 0 && o->cs_type != 1) {
    set_error(&e->err, "census type %d invalid", o->cs_type);
    return SGM_ERR_ARG;
  }
  if (o->p1 < 0 || o->p2_init < 0) {
    set_error(&e->err, "negative penalties (p1=%d p2=%d)", o->p1, o->p2_init);
    return SGM_ERR_ARG;
  }
  if (o->post_filter_type < 0 || o->post_filter_type > 2) {
    set_error(&e->err, "post filter type %d invalid (0 none, 1 Gauss, 2 bilateral)", o->post_filter_type);
    return SGM_ERR_ARG;
  }
  if (o->morphology_type < 0 || o->morphology_type > 4) {
    set_error(&e->err, "morphology type %d invalid (0 none, 1 erosion, 2 dilation, 3 open, 4 close)",
              o->morphology_type);
    return SGM_ERR_ARG;
  }
  if ((size_t)W * H > (size_t)INT32_MAX / 2) {
    set_error(&e->err, "image too large");
    return SGM_ERR_ARG;
  }
  return SGM_OK;
}

// volumes == false: the cost and path volumes are supplied later (batch arena).
int engine_init(sgm_engine* e, int W, int H, int M, int D, const sgm_option_t* o, bool log, bool volumes = true) {
  if (e->ready) e->free_all();
  e->own_volumes = volumes;
  const int v = validate(e, W, H, M, D, o);
  if (v != SGM_OK) return v;
  SGM_CUDA_TRY(e, cudaGetDevice(&e->dev));
  SGM_CUDA_TRY(e, cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, e->dev));
  e->W = W; e->H = H; e->M = M; e->D = D;
  e->opt = *o;
  e->print_log = log;
  SGM_CUDA_TRY(e, cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  SGM_CUDA_TRY(e, cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking));
  SGM_CUDA_TRY(e, cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
  SGM_CUDA_TRY(e, cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
  const size_t N = e->npix();
  const size_t V = e->vol() * e->nviews();  // the right view's volumes only with the LR check
  for (int i = 0; i < 2; ++i) {
    SGM_CUDA_TRY(e, dalloc(&e->img[i], N));
    SGM_CUDA_TRY(e, sgm_dev_malloc(&e->cs[i], N * 8));
    SGM_CUDA_TRY(e, dalloc(&e->init[i], N));
  }
  if (volumes) {
    SGM_CUDA_TRY(e, dalloc(&e->cost, V));
    SGM_CUDA_TRY(e, dalloc(&e->lr, V));
    SGM_CUDA_TRY(e, dalloc(&e->rl, V));
    SGM_CUDA_TRY(e, dalloc(&e->bt, V));
  }
  SGM_CUDA_TRY(e, dalloc(&e->wta, 2 * N));
  SGM_CUDA_TRY(e, dalloc(&e->post, N));
  SGM_CUDA_TRY(e, dalloc(&e->post2, N));
  SGM_CUDA_TRY(e, dalloc(&e->dr_out, N));
  SGM_CUDA_TRY(e, dalloc(&e->out, N));
  SGM_CUDA_TRY(e, dalloc(&e->init_tmp, N));
  SGM_CUDA_TRY(e, dalloc(&e->key, N));
  SGM_CUDA_TRY(e, dalloc(&e->label, N));
  SGM_CUDA_TRY(e, dalloc(&e->count, N));
  e->ready = true;
  if (log) printf("sgm-b200: init %dx%d, disparities %d..%d, census %s\n", W, H, M, M + D, o->cs_type ? "9x7" : "5x5");
  return SGM_OK;
}

// Columns per CTA of the vertical kernels and whether the bottom->top path costs of those
// columns fit in shared memory (H*C*D bytes, at most 100 KB so two CTAs share an SM).
void vertical_shape(int H, int D, int* C, int* bt_smem, size_t* smem, int max_cols = 0, int use_smem = 0) {
  const size_t per_col = (size_t)H * D;
  const size_t budget = 100 * 1024;
  int c = max_cols > 0 ? max_cols : 8;
  if (!use_smem) {
    *C = c;
    *bt_smem = 0;
    *smem = 0;
    return;
  }
  while (c > 2 && per_col * c > budget) c >>= 1;
  if (per_col * c <= budget) {
    *C = c;
    *bt_smem = 1;
    *smem = per_col * c;
  } else {
    *C = 8;
    *bt_smem = 0;
    *smem = 0;
  }
}

int rows_per_cta(int W, int word_bytes, bool with_init) {
  const size_t per_row = (size_t)W * (2 * word_bytes + (with_init ? 2 : 0));
  int R = 4;
  while (R > 1 && per_row * R > 160 * 1024) R >>= 1;
  return R;
}

// Thread-per-scanline kernels (variant 3): G lanes per scanline, prefetch depth by slice size.
template <int K, int G>
constexpr int pf3() {
  return 32 * K / G >= 64 ? 2 : (32 * K / G >= 32 ? 4 : 8);
}
// the column kernel keeps four volumes in its prefetch ring
template <int K, int G>
constexpr int pf3v() {
  return 32 * K / G >= 32 ? 1 : (32 * K / G >= 16 ? 2 : 4);
}
template <int K>
constexpr bool lanes_ok(int G) {
  return (G == 1 || G == 2 || G == 4 || G == 8) && !(K == 4 && (G == 1 || G == 8)) && K <= 4;
}
constexpr int kDefaultRowLanes = 8, kDefaultColLanes = 4;

template <int K>
int launch_rows3(sgm_engine* e, int G, const sgm::PlainParams& P, int nv, cudaStream_t s) {
  if (!lanes_ok<K>(G)) G = kDefaultRowLanes;
  const long threads = (long)nv * 2 * e->H * G;
  const int blocks = (int)((threads + 127) / 128);
  auto go = [&](auto kern) {
    return SGM_LAUNCH(e, s, "hpaths_plain", kern<<<blocks, 128, 0, s>>>(e->cost, e->lr, e->rl, P, nv));
  };
  if constexpr (K == 4) {
    return G == 2 ? go(sgm::k_hpaths3<K, 2, pf3<K, 2>()>) : go(sgm::k_hpaths3<K, 4, pf3<K, 4>()>);
  } else {
    switch (G) {
      case 1: return go(sgm::k_hpaths3<K, 1, pf3<K, 1>()>);
      case 4: return go(sgm::k_hpaths3<K, 4, pf3<K, 4>()>);
      case 8: return go(sgm::k_hpaths3<K, 8, pf3<K, 8>()>);
      default: return go(sgm::k_hpaths3<K, 2, pf3<K, 2>()>);
    }
  }
}

// pass: 0 both column passes, 1 bottom-to-top only, 2 top-to-bottom + sum + WTA only
template <int K, int PASS>
int launch_cols3_pass(sgm_engine* e, int G, const sgm::PlainParams& P, const sgm::WtaParams& Q, float* wta, int nv,
                      cudaStream_t s) {
  if (!lanes_ok<K>(G)) G = kDefaultColLanes;
  const long threads = (long)e->W * G;
  dim3 grid((unsigned)((threads + 127) / 128), nv);
  const size_t smem = (size_t)(128 / G) * sgm::vpaths3_col_smem<K>();
  const char* name = PASS == 1 ? "vpaths_bt_plain" : "vpaths_wta_plain";
  auto go = [&](auto kern) {
    return SGM_LAUNCH(e, s, name, kern<<<grid, 128, smem, s>>>(e->cost, e->lr, e->rl, e->bt, wta, P, Q));
  };
  if constexpr (K == 4) {
    return G == 2 ? go(sgm::k_vpaths3<K, 2, pf3v<K, 2>(), PASS>) : go(sgm::k_vpaths3<K, 4, pf3v<K, 4>(), PASS>);
  } else {
    switch (G) {
      case 1: return go(sgm::k_vpaths3<K, 1, pf3v<K, 1>(), PASS>);
      case 2: return go(sgm::k_vpaths3<K, 2, pf3v<K, 2>(), PASS>);
      case 8: return go(sgm::k_vpaths3<K, 8, pf3v<K, 8>(), PASS>);
      default: return go(sgm::k_vpaths3<K, 4, pf3v<K, 4>(), PASS>);
    }
  }
}

using sgm::EncodeTiledFn;
using sgm::encode_tiled;

// Tensor map i (0 cost, 1 bt, 2 lr, 3 rl, 4 tb) of the engine's volumes, [nv][H][W * D] bytes, in boxes
// of 32 rows x D bytes with the D-byte swizzle (k_vscan_plain4); rebuilt when the volume moved.
int volume_map(sgm_engine* e, int i, const uint8_t* base, int nv, const CUtensorMap** out) {
  sgm_engine::TmapKey& k = e->tmap_key[i];
  if (k.base != base || k.W != e->W || k.H != e->H || k.D != e->D || k.nv != nv) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn) {
      set_error(&e->err, "cuTensorMapEncodeTiled is not available from the driver");
      return SGM_ERR_CUDA;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)e->W * e->D, (cuuint64_t)e->H, (cuuint64_t)nv};
    const cuuint64_t strides[2] = {(cuuint64_t)e->W * e->D, (cuuint64_t)e->W * e->H * e->D};
    const cuuint32_t box[3] = {(cuuint32_t)e->D, (cuuint32_t)sgm::kScanChunk, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUtensorMapSwizzle sw = e->D == 32   ? CU_TENSOR_MAP_SWIZZLE_32B
                                  : e->D == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                               : CU_TENSOR_MAP_SWIZZLE_128B;
    const CUresult r = fn(&e->tmap[i], CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t*>(base), dims, strides,
                          box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      k = sgm_engine::TmapKey{};
      set_error(&e->err, "cuTensorMapEncodeTiled failed (%d) for a %dx%dx%d volume", (int)r, e->W, e->H, e->D);
      return SGM_ERR_CUDA;
    }
    k = sgm_engine::TmapKey{base, e->W, e->H, e->D, nv};
  }
  *out = &e->tmap[i];
  return SGM_OK;
}

// Warp-per-scanline kernels (variant 4, D <= 128): the row scans, and the column passes (pass 1
// bottom-to-top, pass 2 top-to-bottom + sum + WTA).
template <int K>
int launch_rows4(sgm_engine* e, const sgm::PlainParams& P, int nv, cudaStream_t s) {
  if constexpr (K <= 4) {
    constexpr int wpb = sgm::hscan_plain4_warps<K>();
    const int blocks = (nv * 2 * e->H + wpb - 1) / wpb;
    SGM_CUDA_TRY(e, sgm::prefer_max_shared(sgm::k_hscan_plain4<K>));
    return SGM_LAUNCH(e, s, "hpaths_plain",
                      sgm::k_hscan_plain4<K><<<blocks, 32 * wpb, 0, s>>>(e->cost, e->lr, e->rl, P, nv));
  } else {
    return SGM_ERR_UNSUPPORTED;
  }
}

// The top-to-bottom volume of the warp-per-scanline column kernels, allocated on first use (a
// direct run: never inside a graph capture of the matcher's own).
int ensure_tb(sgm_engine* e, int nv) {
  if (e->tb) return SGM_OK;
  const cudaError_t r = dalloc(&e->tb, e->vol() * nv);
  if (r != cudaSuccess) {
    e->tb = nullptr;
    set_error(&e->err, "device allocation of the top-to-bottom volume failed: %s", cudaGetErrorString(r));
    return r == cudaErrorMemoryAllocation ? SGM_ERR_NOMEM : SGM_ERR_CUDA;
  }
  return SGM_OK;
}

template <int K, int PASS>
int launch_cols4(sgm_engine* e, const sgm::PlainParams& P, const sgm::WtaParams& Q, float* wta, int nv,
                 cudaStream_t s) {
  if constexpr (K <= 4) {
    constexpr int wpb = sgm::vscan_plain4_warps<K>();
    const dim3 grid((e->W + wpb - 1) / wpb, nv);
    const CUtensorMap *mc, *mb, *ml, *mr;
    int st = volume_map(e, 0, e->cost, nv, &mc);
    if (!st) st = volume_map(e, 1, e->bt, nv, &mb);
    if (!st) st = volume_map(e, 2, e->lr, nv, &ml);
    if (!st) st = volume_map(e, 3, e->rl, nv, &mr);
    if (st) return st;
    SGM_CUDA_TRY(e, sgm::prefer_max_shared(sgm::k_vscan_plain4<K, PASS>));
    return SGM_LAUNCH(e, s, PASS == 1 ? "vpaths_bt_plain" : "vpaths_wta_plain",
                      sgm::k_vscan_plain4<K, PASS><<<grid, 32 * wpb, 0, s>>>(*mc, *mb, *ml, *mr, e->bt, wta, P, Q));
  } else {
    return SGM_ERR_UNSUPPORTED;
  }
}

// The bottom-to-top column pass depends only on the cost volume, so it runs on the matcher's side
// stream while the row scans run on s; the top-to-bottom pass (which sums all four paths) follows
// the join. In a captured graph the side stream joins the capture through ev_fork.
constexpr bool kSplitColumns = true;

// With per-kernel profiling on, both run on s one after the other, so that every launch is timed
// alone.
template <typename SideWork, typename MainWork>
int fork_join(sgm_engine* e, cudaStream_t s, SideWork side_work, MainWork main_work) {
  if (g_prof.on) {
    const int st = side_work(s);
    return st ? st : main_work(s);
  }
  SGM_CUDA_TRY(e, cudaEventRecord(e->ev_fork, s));
  SGM_CUDA_TRY(e, cudaStreamWaitEvent(e->side, e->ev_fork, 0));
  int st = side_work(e->side);
  if (!st) st = main_work(s);
  // join even after an error, so that a capture in progress is not left with a forked stream
  const cudaError_t r = cudaEventRecord(e->ev_join, e->side);
  const cudaError_t w = r == cudaSuccess ? cudaStreamWaitEvent(s, e->ev_join, 0) : r;
  if (st) return st;
  SGM_CUDA_TRY(e, w);
  return SGM_OK;
}

template <int K, typename Word>
int launch_plain(sgm_engine* e, const Word* csl, const Word* csr, float* wta) {
  sgm::PlainParams P;
  P.W = e->W; P.H = e->H; P.min_d = e->M; P.x0 = std::max(0, e->M);
  P.p1 = (uint32_t)e->opt.p1; P.p2 = (uint32_t)e->opt.p2_init;
  P.vstride = e->vol();
  const int nv = e->nviews();
  // thread-per-scanline kernels: exact for 16-bit path costs and the min(x + P1, L) form
  const bool v3_ok = K <= 4 && e->opt.p1 <= (int)sgm::kMaxPenalty16 && e->opt.p2_init <= (int)sgm::kMaxPenalty16 &&
                     e->opt.p2_init >= e->opt.p1 &&
                     (e->ext.tie_rule == sgm::kTieLowest || e->ext.tie_rule == sgm::kTieRefB200);
  int st;
  // warp-per-scanline kernels: D <= 128 and the tie rules of their serial WTA; otherwise the
  // default takes their place
  const bool v4_ok = K <= 4 && (e->ext.tie_rule == sgm::kTieLowest || e->ext.tie_rule == sgm::kTieHighest ||
                                e->ext.tie_rule == sgm::kTieRefB200);
  const int tune_row = e->tune_row_kernel == 4 && !v4_ok ? 0 : e->tune_row_kernel;
  const int tune_col = e->tune_col_kernel == 4 && !v4_ok ? 0 : e->tune_col_kernel;
  const bool cols_v3 = (tune_col == 3 || tune_col == 0) && v3_ok;
  const bool cols_v4 = tune_col == 4;
  sgm::WtaParams Q;
  Q.uniqueness = e->opt.unique_threshold;
  Q.tie_rule = e->ext.tie_rule;
  const bool warp_kernel = (K <= 4);
  Q.rows = warp_kernel ? (e->H / 2) * 2 : e->H;
  Q.dmax_excl = warp_kernel ? 32 * K : 32 * K - 1;
  Q.dstride = e->npix();
  Q.image_border(e->W, e->H);
  if (((tune_row == 3 || tune_row == 0) && v3_ok) || tune_row == 4) {
    dim3 cg((e->W + 127) / 128, e->H, nv);
    st = SGM_LAUNCH(e, e->stream, "cost", sgm::k_cost3<K, Word><<<cg, 128, 0, e->stream>>>(csl, csr, e->cost, P));
    if (st) return st;
    const auto rows = [&](cudaStream_t ms) {
      return tune_row == 4 ? launch_rows4<K>(e, P, nv, ms) : launch_rows3<K>(e, e->tune_row_lanes, P, nv, ms);
    };
    if (kSplitColumns && (cols_v3 || cols_v4)) {
      e->bt_stored = true;
      const int gc = e->tune_col_lanes;
      st = fork_join(
          e, e->stream,
          [&](cudaStream_t ss) {
            return cols_v4 ? launch_cols4<K, 1>(e, P, Q, wta, nv, ss) : launch_cols3_pass<K, 1>(e, gc, P, Q, wta, nv, ss);
          },
          rows);
      if (st) return st;
      return cols_v4 ? launch_cols4<K, 2>(e, P, Q, wta, nv, e->stream)
                     : launch_cols3_pass<K, 2>(e, gc, P, Q, wta, nv, e->stream);
    }
    st = rows(e->stream);
  } else if (tune_row == 1) {  // whole census rows of R scanlines in shared memory
    const int R = e->tune_rows > 0 ? e->tune_rows : rows_per_cta(e->W, sizeof(Word), false);
    const size_t smem = (size_t)R * 2 * e->W * sizeof(Word);
    if (smem > 227 * 1024) {
      set_error(&e->err, "image width %d too large for the whole-row kernel", e->W);
      return SGM_ERR_UNSUPPORTED;
    }
    auto hk = sgm::k_hpaths_plain<K, Word>;
    SGM_CUDA_TRY(e, sgm::allow_max_dynamic_smem(hk));
    dim3 hg((e->H + R - 1) / R, nv), hb(32, 2 * R);
    st = SGM_LAUNCH(e, e->stream, "hpaths_plain", hk<<<hg, hb, smem, e->stream>>>(csl, csr, e->cost, e->lr, e->rl, P));
  } else {
    const int R = e->tune_rows > 0 ? e->tune_rows : 4;
    const size_t smem = (size_t)2 * R * sgm::hpaths2_warp_smem<K, Word>();
    auto hk = sgm::k_hpaths_plain2<K, Word>;
    SGM_CUDA_TRY(e, sgm::allow_max_dynamic_smem(hk));
    dim3 hg((e->H + R - 1) / R, nv), hb(32, 2 * R);
    st = SGM_LAUNCH(e, e->stream, "hpaths_plain", hk<<<hg, hb, smem, e->stream>>>(csl, csr, e->cost, e->lr, e->rl, P));
  }
  if (st) return st;
  int C = 8, bt_smem = 0;
  size_t vsmem = 0;
  if (cols_v3) {
    e->bt_stored = true;
    return launch_cols3_pass<K, 0>(e, e->tune_col_lanes, P, Q, wta, nv, e->stream);
  }
  if (cols_v4) {
    e->bt_stored = true;
    st = launch_cols4<K, 1>(e, P, Q, wta, nv, e->stream);
    return st ? st : launch_cols4<K, 2>(e, P, Q, wta, nv, e->stream);
  }
  if (tune_col != 2) {
    C = e->tune_cols > 0 ? e->tune_cols : 8;
    e->bt_stored = true;
    dim3 vg((e->W + C - 1) / C, nv), vb(32, C);
    return SGM_LAUNCH(e, e->stream, "vpaths_wta_plain",
                      sgm::k_vpaths_wta_plain<K><<<vg, vb, 0, e->stream>>>(e->cost, e->lr, e->rl, e->bt, wta, P, Q));
  }
  vertical_shape(e->H, 32 * K, &C, &bt_smem, &vsmem, e->tune_cols, e->tune_bt_smem);
  e->bt_stored = !bt_smem;
  auto vk = sgm::k_vpaths_wta_plain2<K, 8>;
  if (vsmem) SGM_CUDA_TRY(e, sgm::allow_max_dynamic_smem(vk));
  dim3 vg((e->W + C - 1) / C, nv), vb(32, C);
  return SGM_LAUNCH(e, e->stream, "vpaths_wta_plain",
                    vk<<<vg, vb, vsmem, e->stream>>>(e->cost, e->lr, e->rl, e->bt, wta, P, Q, bt_smem));
}

// ------------------------------------------------------------------------------------------
// Regions of interest (StereoCuda::Match with StereoROI_T; reference: cost cusgm_cc.cu:478-488,
// scans cusgm_ca.cu:3991-3999 and :4179-4192, WTA grid :4139-4165, small-region strips
// StereoCudaImpl.cpp:463-498). A view's region is matched as a sub-image of its own: its cost
// (partners from the whole image) goes into a compact [h][w][D] sub-volume, the thread-per-scanline
// scans and WTA run on it with the image border shifted, and the region's map is scattered into the
// view's full map, INVALID outside.
// ------------------------------------------------------------------------------------------
struct RoiRegion {
  int x0, y0, w, h;  // columns [x0, x0 + w), rows [y0, y0 + h)
  int bx;            // first column of the cost kernel's D-pixel blocks (the ROI's own x)
};

// Regions of both views. Without an ROI a view covers columns [max(0, min_disp), W) and every
// row; with one, its rectangle (which must lie inside the image), columns clipped to start at
// max(0, min_disp): the reference computes the left view's cost without the ROI, from that column.
int roi_regions(sgm_engine* e, const sgm_roi_t* roi_l, const sgm_roi_t* roi_r, RoiRegion reg[2]) {
  const int x0 = std::max(0, e->M);
  for (int v = 0; v < 2; ++v) {
    const sgm_roi_t* r = v == 0 ? roi_l : roi_r;
    reg[v] = RoiRegion{x0, 0, e->W - x0, e->H, x0};
    if (!r) continue;
    if (r->x < 0 || r->y < 0 || r->w <= 0 || r->h <= 0 || r->x > e->W - r->w || r->y > e->H - r->h) {
      set_error(&e->err, "ROI (%d, %d, %d, %d) does not lie inside the %dx%d image", r->x, r->y, r->w, r->h, e->W,
                e->H);
      return SGM_ERR_ARG;
    }
    const int c0 = std::max(r->x, x0);
    if (c0 >= r->x + r->w) {
      set_error(&e->err, "ROI (%d, %d, %d, %d) has no column at or right of the minimum disparity %d", r->x, r->y,
                r->w, r->h, e->M);
      return SGM_ERR_ARG;
    }
    reg[v] = RoiRegion{c0, r->y, r->x + r->w - c0, r->h, r->x};
  }
  return SGM_OK;
}

template <int K>
int roi_rows(sgm_engine* e, int G, const uint8_t* cost, uint8_t* lr, uint8_t* rl, const sgm::PlainParams& P,
             cudaStream_t s) {
  if (!lanes_ok<K>(G)) G = kDefaultRowLanes;
  const int blocks = (int)((2L * P.H * G + 127) / 128);
  auto go = [&](auto kern) {
    return SGM_LAUNCH(e, s, "hpaths_roi", kern<<<blocks, 128, 0, s>>>(cost, lr, rl, P, 1));
  };
  if constexpr (K == 4) {
    return G == 2 ? go(sgm::k_hpaths3<K, 2, pf3<K, 2>()>) : go(sgm::k_hpaths3<K, 4, pf3<K, 4>()>);
  } else {
    switch (G) {
      case 1: return go(sgm::k_hpaths3<K, 1, pf3<K, 1>()>);
      case 4: return go(sgm::k_hpaths3<K, 4, pf3<K, 4>()>);
      case 8: return go(sgm::k_hpaths3<K, 8, pf3<K, 8>()>);
      default: return go(sgm::k_hpaths3<K, 2, pf3<K, 2>()>);
    }
  }
}

template <int K>
int roi_cols(sgm_engine* e, int G, const uint8_t* cost, const uint8_t* lr, const uint8_t* rl, uint8_t* bt,
             float* wta, const sgm::PlainParams& P, const sgm::WtaParams& Q, cudaStream_t s) {
  if (!lanes_ok<K>(G)) G = kDefaultColLanes;
  const dim3 grid((unsigned)(((long)P.W * G + 127) / 128), 1);
  const size_t smem = (size_t)(128 / G) * sgm::vpaths3_col_smem<K>();
  auto go = [&](auto kern) {
    return SGM_LAUNCH(e, s, "vpaths_wta_roi", kern<<<grid, 128, smem, s>>>(cost, lr, rl, bt, wta, P, Q));
  };
  if constexpr (K == 4) {
    return G == 2 ? go(sgm::k_vpaths3<K, 2, pf3v<K, 2>(), 0>) : go(sgm::k_vpaths3<K, 4, pf3v<K, 4>(), 0>);
  } else {
    switch (G) {
      case 1: return go(sgm::k_vpaths3<K, 1, pf3v<K, 1>(), 0>);
      case 2: return go(sgm::k_vpaths3<K, 2, pf3v<K, 2>(), 0>);
      case 8: return go(sgm::k_vpaths3<K, 8, pf3v<K, 8>(), 0>);
      default: return go(sgm::k_vpaths3<K, 4, pf3v<K, 4>(), 0>);
    }
  }
}

// Cost, scans and WTA of each view's region, scattered into wta (view v at wta + v * W * H).
template <int K, typename Word>
int launch_roi(sgm_engine* e, const Word* csl, const Word* csr, const RoiRegion reg[2], float* wta) {
  constexpr int D = 32 * K;
  cudaStream_t s = e->stream;
  const size_t V = e->vol(), N = e->npix();
  sgm::PlainParams Pg;  // whole-image geometry for the cost kernel
  Pg.W = e->W; Pg.H = e->H; Pg.min_d = e->M; Pg.x0 = std::max(0, e->M);
  Pg.p1 = (uint32_t)e->opt.p1; Pg.p2 = (uint32_t)e->opt.p2_init;
  Pg.vstride = V;
  for (int v = 0; v < e->nviews(); ++v) {
    const RoiRegion& r = reg[v];
    uint8_t* cost = e->cost + v * V;
    uint8_t* lr = e->lr + v * V;
    uint8_t* rl = e->rl + v * V;
    uint8_t* bt = e->bt + v * V;
    float* region_map = v == 0 ? e->post : e->post2;
    int st = SGM_LAUNCH(e, s, "cost_roi", sgm::k_cost_roi<K, Word><<<dim3((r.w + 127) / 128, r.h), 128, 0, s>>>(
                                              csl, csr, cost, Pg, v, r.x0, r.y0, r.w, r.bx));
    if (st) return st;
    sgm::PlainParams P = Pg;  // the region as a sub-image
    P.W = r.w; P.H = r.h; P.x0 = 0;
    P.vstride = (size_t)r.w * r.h * D;
    if ((st = roi_rows<K>(e, e->tune_row_lanes, cost, lr, rl, P, s))) return st;
    sgm::WtaParams Q;
    Q.uniqueness = e->opt.unique_threshold;
    Q.tie_rule = e->ext.tie_rule;
    Q.rows = (r.h / 2) * 2;  // the reference's WTA launch: floor(h/2) blocks of two rows from the ROI's y
    Q.dmax_excl = D;
    Q.dstride = (size_t)r.w * r.h;
    Q.image_border(e->W, e->H, r.x0, r.y0);
    if ((st = roi_cols<K>(e, e->tune_col_lanes, cost, lr, rl, bt, region_map, P, Q, s))) return st;
    st = SGM_LAUNCH(e, s, "roi_scatter", sgm::k_roi_scatter<<<dim3((e->W + 127) / 128, e->H), 128, 0, s>>>(
                                             region_map, wta + v * N, e->W, e->H, r.x0, r.y0, r.w, r.h));
    if (st) return st;
  }
  e->bt_stored = true;
  return SGM_OK;
}

// Initial-disparity levels, thread-per-scanline kernels (uint32 per disparity): G = 2, 4 or 8.
constexpr int kDefaultInitRowLanes = 8, kDefaultInitColLanes = 8;

template <typename Word>
int init3_cost(sgm_engine* e, const Word* csl, const Word* csr, const int16_t* il, const int16_t* ir,
               const sgm::InitParams& P, cudaStream_t s) {
  const size_t csmem = (size_t)e->W * sizeof(Word);
  auto ck = sgm::k_cost3_init<Word>;
  SGM_CUDA_TRY(e, sgm::allow_max_dynamic_smem(ck));
  return SGM_LAUNCH(e, s, "cost", ck<<<dim3(e->H, e->nviews()), 256, csmem, s>>>(csl, csr, il, ir, e->cost, P));
}

inline int init3_rows(sgm_engine* e, const int16_t* il, const int16_t* ir, const sgm::InitParams& P,
                      cudaStream_t s) {
  const int nv = e->nviews();
  int G = e->tune_row_lanes;
  if (G != 2 && G != 4 && G != 8) G = kDefaultInitRowLanes;
  const long threads = (long)nv * 2 * e->H * G;
  const int blocks = (int)((threads + 127) / 128);
  auto go = [&](auto kern) {
    return SGM_LAUNCH(e, s, "hpaths_init", kern<<<blocks, 128, 0, s>>>(e->cost, il, ir, e->lr, e->rl, P, nv));
  };
  return G == 2   ? go(sgm::k_hpaths3_init<2, 8>)
         : G == 8 ? go(sgm::k_hpaths3_init<8, 8>)
                  : go(sgm::k_hpaths3_init<4, 8>);
}

// PASS as in launch_cols3_pass
template <int PASS>
int init3_cols(sgm_engine* e, const int16_t* il, const int16_t* ir, float* wta, const sgm::InitParams& P,
               const sgm::WtaParams& Q, cudaStream_t s) {
  const int nv = e->nviews();
  int G = e->tune_col_lanes;
  if (G != 2 && G != 4 && G != 8) G = kDefaultInitColLanes;
  e->bt_stored = true;
  dim3 grid((unsigned)(((long)e->W * G + 127) / 128), nv);
  const char* name = PASS == 1 ? "vpaths_bt_init" : "vpaths_wta_init";
  auto go = [&](auto kern) {
    return SGM_LAUNCH(e, s, name, kern<<<grid, 128, 0, s>>>(e->cost, e->lr, e->rl, il, ir, e->bt, wta, P, Q));
  };
  return G == 2   ? go(sgm::k_vpaths3_init<2, 1, PASS>)
         : G == 8 ? go(sgm::k_vpaths3_init<8, 4, PASS>)
                  : go(sgm::k_vpaths3_init<4, 4, PASS>);
}

// Initial-disparity levels, latency form (variant 4): one warp per scanline, chunks staged by
// bulk async copies (sgm_kernels4.cuh). Exact for any penalties and tie rule.
constexpr int kScan4RowWarps = 2, kScan4ColWarps = 4;

inline int init4_rows(sgm_engine* e, const int16_t* il, const int16_t* ir, const sgm::InitParams& P,
                      cudaStream_t s) {
  const int nv = e->nviews();
  const int blocks = (nv * 2 * e->H + kScan4RowWarps - 1) / kScan4RowWarps;
  SGM_CUDA_TRY(e, sgm::prefer_max_shared(sgm::k_hscan_init4<kScan4RowWarps>));
  return SGM_LAUNCH(e, s, "hpaths_init", sgm::k_hscan_init4<kScan4RowWarps><<<blocks, 32 * kScan4RowWarps, 0, s>>>(
                                             e->cost, il, ir, e->lr, e->rl, P, nv));
}

// PASS 1: bottom-to-top into bt; PASS 3: top-to-bottom into tb.
template <int PASS>
int init4_cols(sgm_engine* e, const int16_t* il, const int16_t* ir, const sgm::InitParams& P, cudaStream_t s) {
  e->bt_stored = true;
  const int nv = e->nviews();
  const dim3 grid((unsigned)((e->W + kScan4ColWarps - 1) / kScan4ColWarps), nv);
  int st = PASS == 3 ? ensure_tb(e, nv) : SGM_OK;
  uint8_t* out = PASS == 1 ? e->bt : e->tb;
  const CUtensorMap *mc, *mo;
  if (!st) st = volume_map(e, 0, e->cost, nv, &mc);
  if (!st) st = volume_map(e, PASS == 1 ? 1 : 4, out, nv, &mo);
  if (st) return st;
  SGM_CUDA_TRY(e, sgm::prefer_max_shared(sgm::k_vscan_init4<kScan4ColWarps, PASS>));
  return SGM_LAUNCH(e, s, PASS == 1 ? "vpaths_bt_init" : "vpaths_tb_init",
                    sgm::k_vscan_init4<kScan4ColWarps, PASS><<<grid, 32 * kScan4ColWarps, 0, s>>>(
                        *mc, *mo, il, ir, out, P));
}

inline int init4_cols_both(sgm_engine* e, const int16_t* il, const int16_t* ir, const sgm::InitParams& P,
                           cudaStream_t s) {
  const int st = init4_cols<1>(e, il, ir, P, s);
  return st ? st : init4_cols<3>(e, il, ir, P, s);
}

inline int init4_wta(sgm_engine* e, const int16_t* il, const int16_t* ir, float* wta, const sgm::InitParams& P,
                     const sgm::WtaParams& Q, cudaStream_t s) {
  const dim3 grid((e->W + 127) / 128, e->H, e->nviews());
  return SGM_LAUNCH(e, s, "wta_init",
                    sgm::k_wta_init4<<<grid, 128, 0, s>>>(e->bt, e->tb, e->lr, e->rl, il, ir, wta, P, Q));
}

template <typename Word>
int launch_init(sgm_engine* e, const Word* csl, const Word* csr, const int16_t* il, const int16_t* ir, float* wta) {
  sgm::InitParams P;
  P.W = e->W; P.H = e->H; P.x0 = std::max(0, e->M);
  P.p1 = (uint32_t)e->opt.p1; P.p1s = e->opt.p1; P.p2s = e->opt.p2_init; P.p2_div0 = e->ext.p2_div0;
  P.invalid_cost = e->opt.cs_type == 1 ? 0xFFu : sgm::kInvalidCost;
  P.vstride = e->vol();
  const int nv = e->nviews();
  sgm::WtaParams Q3;
  Q3.uniqueness = e->opt.unique_threshold;
  Q3.tie_rule = e->ext.init_tie_rule;
  Q3.rows = (e->H / 4) * 4;
  Q3.dmax_excl = sgm::kLevelRange - 1;
  Q3.dstride = e->npix();
  Q3.image_border(e->W, e->H);
  // thread-per-scanline kernels: uint32 arithmetic (exact for any penalties); WTA rules 0 and 4
  const bool v3_ok = e->ext.init_tie_rule == sgm::kTieLowest || e->ext.init_tie_rule == sgm::kTieRefB200;
  // the warp-per-scanline row kernel packs P2' into 22 bits; larger penalties take the default
  const bool pack_ok = e->opt.p1 >= 0 && e->opt.p1 < (1 << 22) && e->opt.p2_init < (1 << 22) && e->ext.p2_div0 < (1 << 22);
  const int tune_row = e->tune_row_kernel == 4 && !pack_ok ? 0 : e->tune_row_kernel;
  const bool rows3 = v3_ok && (tune_row == 0 || tune_row == 3);
  const bool cols3 = v3_ok && (e->tune_col_kernel == 0 || e->tune_col_kernel == 3);
  const bool rows4 = tune_row == 4, cols4 = e->tune_col_kernel == 4;
  // rows reading the cost volume (variants 3 and 4) and columns split into two passes
  auto rows_cv = [&](cudaStream_t ms) { return rows4 ? init4_rows(e, il, ir, P, ms) : init3_rows(e, il, ir, P, ms); };
  auto cols_bt = [&](cudaStream_t ss) {
    return cols4 ? init4_cols_both(e, il, ir, P, ss) : init3_cols<1>(e, il, ir, wta, P, Q3, ss);
  };
  int st;
  if ((rows3 || rows4) && (cols3 || cols4) && kSplitColumns) {  // bottom-to-top pass beside the row scans
    st = init3_cost<Word>(e, csl, csr, il, ir, P, e->stream);
    if (!st) st = fork_join(e, e->stream, cols_bt, rows_cv);
    if (st) return st;
    return cols4 ? init4_wta(e, il, ir, wta, P, Q3, e->stream) : init3_cols<2>(e, il, ir, wta, P, Q3, e->stream);
  }
  if (rows3 || rows4) {
    st = init3_cost<Word>(e, csl, csr, il, ir, P, e->stream);
    if (!st) st = rows_cv(e->stream);
  } else if (tune_row == 1) {  // whole census rows of R scanlines in shared memory
    const int R = e->tune_rows > 0 ? e->tune_rows : rows_per_cta(e->W, sizeof(Word), true);
    const size_t smem = (size_t)R * e->W * (2 * sizeof(Word) + 2);
    if (smem > 227 * 1024) {
      set_error(&e->err, "image width %d too large for the whole-row kernel", e->W);
      return SGM_ERR_UNSUPPORTED;
    }
    auto hk = sgm::k_hpaths_init<Word>;
    SGM_CUDA_TRY(e, sgm::allow_max_dynamic_smem(hk));
    dim3 hg((e->H + R - 1) / R, nv), hb(32, 2 * R);
    st = SGM_LAUNCH(e, e->stream, "hpaths_init",
                    hk<<<hg, hb, smem, e->stream>>>(csl, csr, il, ir, e->cost, e->lr, e->rl, P));
  } else {
    int R = e->tune_rows > 0 ? e->tune_rows : 4;
    const size_t row_bytes = ((size_t)e->W * (2 * sizeof(Word) + 2) + 15) & ~size_t(15);  // as in the kernel
    while (R > 1 && R * row_bytes > 120 * 1024) R >>= 1;
    const size_t smem = R * row_bytes + (size_t)2 * R * sgm::hinit2_warp_smem();
    if (smem > 220 * 1024) {
      set_error(&e->err, "image width %d too large for the row kernel", e->W);
      return SGM_ERR_UNSUPPORTED;
    }
    auto hk = sgm::k_hpaths_init2<Word>;
    SGM_CUDA_TRY(e, sgm::allow_max_dynamic_smem(hk));
    dim3 hg((e->H + R - 1) / R, nv), hb(32, 2 * R);
    st = SGM_LAUNCH(e, e->stream, "hpaths_init",
                    hk<<<hg, hb, smem, e->stream>>>(csl, csr, il, ir, e->cost, e->lr, e->rl, P));
  }
  if (st) return st;
  sgm::WtaParams Q;
  Q.uniqueness = e->opt.unique_threshold;
  Q.tie_rule = e->ext.init_tie_rule;
  Q.rows = (e->H / 4) * 4;
  Q.dmax_excl = sgm::kLevelRange - 1;
  Q.dstride = e->npix();
  Q.image_border(e->W, e->H);
  int C = 8, bt_smem = 0;
  size_t vsmem = 0;
  if (cols3) return init3_cols<0>(e, il, ir, wta, P, Q3, e->stream);
  if (cols4) {
    st = init4_cols_both(e, il, ir, P, e->stream);
    return st ? st : init4_wta(e, il, ir, wta, P, Q3, e->stream);
  }
  if (e->tune_col_kernel != 2) {
    C = e->tune_cols > 0 ? e->tune_cols : 8;
    e->bt_stored = true;
    dim3 vg((e->W + C - 1) / C, nv), vb(32, C);
    return SGM_LAUNCH(e, e->stream, "vpaths_wta_init",
                      sgm::k_vpaths_wta_init<<<vg, vb, 0, e->stream>>>(e->cost, e->lr, e->rl, il, ir, e->bt, wta, P, Q));
  }
  vertical_shape(e->H, sgm::kLevelRange, &C, &bt_smem, &vsmem, e->tune_cols, e->tune_bt_smem);
  e->bt_stored = !bt_smem;
  auto vk = sgm::k_vpaths_wta_init2<8>;
  if (vsmem) SGM_CUDA_TRY(e, sgm::allow_max_dynamic_smem(vk));
  dim3 vg((e->W + C - 1) / C, nv), vb(32, C);
  return SGM_LAUNCH(e, e->stream, "vpaths_wta_init",
                    vk<<<vg, vb, vsmem, e->stream>>>(e->cost, e->lr, e->rl, il, ir, e->bt, wta, P, Q, bt_smem));
}

// Enqueues one full match of this level on s. Inputs/outputs are dense device arrays.
// roi_l / roi_r: regions of interest of the views (NULL: the whole view), plain levels only.
int engine_enqueue(sgm_engine* e, const uint8_t* dl_img, const uint8_t* dr_img, const int16_t* dinit, float* dout,
                   float* dout_r, cudaStream_t s, const sgm_roi_t* roi_l = nullptr,
                   const sgm_roi_t* roi_r = nullptr) {
  if (!e->ready) {
    set_error(&e->err, "matcher not initialised");
    return SGM_ERR_STATE;
  }
  if (!e->opt.do_lr_check) roi_r = nullptr;  // no right view is matched (the reference ignores it too)
  const bool roi = roi_l || roi_r;
  RoiRegion reg[2];
  if (roi) {
    if (dinit) {
      set_error(&e->err, "ROI matching at initial-disparity levels is not supported (the reference's pyramid "
                         "never passes an ROI: is_using_roi is false, FasterStereoCuda.cpp:575)");
      return SGM_ERR_UNSUPPORTED;
    }
    const bool v3_ok = e->D <= 128 && e->opt.p1 <= (int)sgm::kMaxPenalty16 &&
                       e->opt.p2_init <= (int)sgm::kMaxPenalty16 && e->opt.p2_init >= e->opt.p1 &&
                       (e->ext.tie_rule == sgm::kTieLowest || e->ext.tie_rule == sgm::kTieRefB200);
    if (!v3_ok) {
      set_error(&e->err, "ROI matching needs D <= 128, P1 <= P2 <= %u and tie rule 0 or 4", sgm::kMaxPenalty16);
      return SGM_ERR_UNSUPPORTED;
    }
    const int rs = roi_regions(e, roi_l, roi_r, reg);
    if (rs) return rs;
  }
  if (dinit && e->D != sgm::kLevelRange) {
    set_error(&e->err, "initial disparities need a disparity range of %d (got %d)", sgm::kLevelRange, e->D);
    return SGM_ERR_UNSUPPORTED;
  }
  if (dinit && !e->opt.using_constant_p2) {
    set_error(&e->err, "initial disparities need using_constant_p2 (the reference launches no aggregation otherwise)");
    return SGM_ERR_UNSUPPORTED;
  }
  cudaStream_t saved = e->stream;
  e->stream = s ? s : e->stream;
  const int W = e->W, H = e->H;
  const size_t N = e->npix();
  int st = SGM_OK;
  // census of both images
  stage_mark(e, "census");
  {
    // 8 rows per block, or 2 when that leaves fewer blocks than SMs (small pyramid levels)
    constexpr int RY = sgm::kCensusRows;
    const bool tall = (long)((W + 511) / 512) * ((H + RY - 1) / RY) * 2 >= e->nsm;
    auto go = [&](auto kern, int ry, auto* csl, auto* csr) {
      dim3 g((W + 511) / 512, (H + ry - 1) / ry, 2), b(128);
      return SGM_LAUNCH(e, e->stream, "census", kern<<<g, b, 0, e->stream>>>(dl_img, dr_img, csl, csr, W, H));
    };
    if (e->opt.cs_type == 1) {
      auto* l = (uint64_t*)e->cs[0];
      auto* r = (uint64_t*)e->cs[1];
      st = tall ? go(sgm::k_census4<uint64_t, 4, 3, RY>, RY, l, r) : go(sgm::k_census4<uint64_t, 4, 3, 2>, 2, l, r);
    } else {
      auto* l = (uint32_t*)e->cs[0];
      auto* r = (uint32_t*)e->cs[1];
      st = tall ? go(sgm::k_census4<uint32_t, 2, 2, RY>, RY, l, r) : go(sgm::k_census4<uint32_t, 2, 2, 2>, 2, l, r);
    }
  }
  // right-view initial disparities when checking consistency at an init level
  const int16_t* dinit_r = nullptr;
  if (!st && dinit && e->opt.do_lr_check) {
    cudaMemsetAsync(e->key, 0, N * sizeof(unsigned), e->stream);
    dim3 g((W + 127) / 128, H);
    st = SGM_LAUNCH(e, e->stream, "right_init_scatter",
                    sgm::k_right_init_scatter<<<g, 128, 0, e->stream>>>(dinit, e->key, W, H));
    if (!st)
      st = SGM_LAUNCH(e, e->stream, "right_init_decode",
                      sgm::k_right_init_decode<<<(unsigned)((N + 255) / 256), 256, 0, e->stream>>>(e->key, e->init_tmp, (int)N));
    if (!st) {
      dim3 db(32, 8), dg((W + 31) / 32, (H + 7) / 8);
      st = SGM_LAUNCH(e, e->stream, "dilation_init",
                      sgm::k_dilation<int16_t><<<dg, db, 0, e->stream>>>(e->init_tmp, e->init[1], W, H, 2));
    }
    dinit_r = e->init[1];
  }
  // cost + four paths + WTA, both views
  stage_mark(e, "cost + aggregation + WTA");
  if (!st) {
    const bool w64 = e->opt.cs_type == 1;
    if (roi) {
      const auto* l64 = (const uint64_t*)e->cs[0];
      const auto* r64 = (const uint64_t*)e->cs[1];
      const auto* l32 = (const uint32_t*)e->cs[0];
      const auto* r32 = (const uint32_t*)e->cs[1];
      switch (e->D) {
        case 32: st = w64 ? launch_roi<1>(e, l64, r64, reg, e->wta) : launch_roi<1>(e, l32, r32, reg, e->wta); break;
        case 64: st = w64 ? launch_roi<2>(e, l64, r64, reg, e->wta) : launch_roi<2>(e, l32, r32, reg, e->wta); break;
        default: st = w64 ? launch_roi<4>(e, l64, r64, reg, e->wta) : launch_roi<4>(e, l32, r32, reg, e->wta); break;
      }
    } else if (dinit) {
      st = w64 ? launch_init<uint64_t>(e, (const uint64_t*)e->cs[0], (const uint64_t*)e->cs[1], dinit, dinit_r, e->wta)
               : launch_init<uint32_t>(e, (const uint32_t*)e->cs[0], (const uint32_t*)e->cs[1], dinit, dinit_r, e->wta);
    } else {
      switch (e->D) {
        case 32: st = w64 ? launch_plain<1, uint64_t>(e, (uint64_t*)e->cs[0], (uint64_t*)e->cs[1], e->wta)
                          : launch_plain<1, uint32_t>(e, (uint32_t*)e->cs[0], (uint32_t*)e->cs[1], e->wta); break;
        case 64: st = w64 ? launch_plain<2, uint64_t>(e, (uint64_t*)e->cs[0], (uint64_t*)e->cs[1], e->wta)
                          : launch_plain<2, uint32_t>(e, (uint32_t*)e->cs[0], (uint32_t*)e->cs[1], e->wta); break;
        case 128: st = w64 ? launch_plain<4, uint64_t>(e, (uint64_t*)e->cs[0], (uint64_t*)e->cs[1], e->wta)
                           : launch_plain<4, uint32_t>(e, (uint32_t*)e->cs[0], (uint32_t*)e->cs[1], e->wta); break;
        default: st = w64 ? launch_plain<8, uint64_t>(e, (uint64_t*)e->cs[0], (uint64_t*)e->cs[1], e->wta)
                          : launch_plain<8, uint32_t>(e, (uint32_t*)e->cs[0], (uint32_t*)e->cs[1], e->wta); break;
      }
    }
  }
  // left-right check + median, post filter, morphology (reference DisparityFilter::Filter,
  // cusgm_df.cu:275-339), then small-region removal. The reference's OPEN and CLOSE run both
  // of their steps from the same input into the same output, so OPEN leaves the dilation and
  // CLOSE the erosion (cusgm_df.cu:311-322); so do these.
  const bool lr = e->opt.do_lr_check, med = e->opt.do_median_filter;
  const int pf = e->opt.post_filter_type;
  const int mp = e->opt.morphology_type;
  const int morph = mp == 3 ? 2 : (mp == 4 ? 1 : mp);  // 1 erosion, 2 dilation
  const bool peaks = e->opt.do_remove_peaks;
  const int nstages = (lr || med ? 1 : 0) + (pf ? 1 : 0) + (morph ? 1 : 0);
  int stage = 0;
  float* spare[2] = {e->post, e->post2};
  // the last stage writes dout; the others alternate between the two spare maps
  auto next_out = [&]() { return ++stage == nstages ? dout : spare[stage & 1]; };
  float* cur = e->wta;  // view 0
  if (!st && lr && dout_r) {
    cudaMemcpyAsync(dout_r, e->wta + N, N * sizeof(float), cudaMemcpyDeviceToDevice, e->stream);
  }
  const dim3 fb(32, 8), fg((W + 31) / 32, (H + 7) / 8);
  if (!st && (lr || med)) {
    stage_mark(e, "left-right check + median");
    float* dst = next_out();
    float* marks = lr ? dout_r : nullptr;
    if (lr && med)
      st = SGM_LAUNCH(e, e->stream, "lr_median", sgm::k_lr_median<true, true><<<fg, fb, 0, e->stream>>>(
                                                     e->wta, e->wta + N, marks, dst, W, H, e->opt.lr_threshold));
    else if (lr)
      st = SGM_LAUNCH(e, e->stream, "lr_median", sgm::k_lr_median<true, false><<<fg, fb, 0, e->stream>>>(
                                                     e->wta, e->wta + N, marks, dst, W, H, e->opt.lr_threshold));
    else
      st = SGM_LAUNCH(e, e->stream, "lr_median", sgm::k_lr_median<false, true><<<fg, fb, 0, e->stream>>>(
                                                     e->wta, nullptr, nullptr, dst, W, H, 0.0f));
    cur = dst;
  }
  // StereoCudaImpl::Match2 (StereoCudaImpl.cpp:548-583) takes the depth from the aggregator's
  // buffer unless small-region removal ran; DisparityFilter::Filter (cusgm_df.cu:275-339) leaves a
  // lone post filter or morphology step in its own buffer and writes a morphology step after a
  // post filter back into the aggregator's buffer. So the depth of a map with exactly one of the
  // two steps and no removal is the depth of the map before that step.
  const float* agg = cur;
  if (!st && (pf || morph)) stage_mark(e, "post filter + morphology");
  if (!st && pf) {
    float* dst = next_out();
    if (pf == 1)
      st = SGM_LAUNCH(e, e->stream, "gauss", sgm::k_gauss_filter<<<fg, fb, 0, e->stream>>>(cur, dst, W, H, 1.5f, 2.0f));
    else
      st = SGM_LAUNCH(e, e->stream, "bilateral", sgm::k_bilateral_filter<<<fg, fb, 0, e->stream>>>(
                                                     dl_img, cur, dst, W, H, 2.5f, 10.0f));
    cur = dst;
  }
  if (!st && morph) {
    float* dst = next_out();
    const int s2 = std::min(W, H);
    const int wnd = s2 < 360 ? 3 : (s2 < 720 ? 5 : 7);
    if (morph == 2)
      st = SGM_LAUNCH(e, e->stream, "dilation", sgm::k_dilation<float><<<fg, fb, 0, e->stream>>>(cur, dst, W, H, (wnd - 1) / 2));
    else
      st = SGM_LAUNCH(e, e->stream, "erosion", sgm::k_erosion<<<fg, fb, 0, e->stream>>>(cur, dst, W, H, (wnd - 1) / 2));
    cur = dst;
  }
  if (!st && cur != dout) {
    cudaMemcpyAsync(dout, cur, N * sizeof(float), cudaMemcpyDeviceToDevice, e->stream);
    cur = dout;
  }
  if (!st && peaks) {
    stage_mark(e, "small-region removal");
    const int strips = e->ext.peaks_strips > 0 ? e->ext.peaks_strips : default_peaks_strips();
    // strips of floor(h / strips) rows from the ROI's first row, or from row 0 (StereoCudaImpl.cpp:
    // 463-498); they are labelled as a sub-image of the rows they cover
    const int y_off = roi_l ? roi_l->y : 0, Hs = roi_l ? roi_l->h : H;
    float* dsub = dout + (size_t)y_off * W;
    const size_t Ns = (size_t)W * Hs;
    const int tiles = Hs / strips;
    if (tiles > 0) {
      const int rows = strips * tiles;
      const unsigned nb = (unsigned)((Ns + 255) / 256);
      st = SGM_LAUNCH(e, e->stream, "cc_rows", sgm::k_cc_rows<<<(Hs + 7) / 8, dim3(32, 8), 0, e->stream>>>(
                                                   dsub, e->label, e->count, W, Hs, rows, e->ext.peaks_abs_mode));
      if (!st && tiles > 1)
        st = SGM_LAUNCH(e, e->stream, "cc_vert", sgm::k_cc_vert<<<nb, 256, 0, e->stream>>>(
                                                     dsub, e->label, W, Hs, tiles, rows, e->ext.peaks_abs_mode));
      if (!st)
        st = SGM_LAUNCH(e, e->stream, "cc_count", sgm::k_cc_count<<<nb, 256, 0, e->stream>>>(e->label, e->count,
                                                                                               (int)Ns));
      if (!st)
        st = SGM_LAUNCH(e, e->stream, "cc_filter", sgm::k_cc_filter<<<nb, 256, 0, e->stream>>>(
                                                       dsub, e->label, e->count, W, Hs, tiles,
                                                       e->opt.peaks_ratio_threshold));
    }
  }
  stage_mark(e, nullptr);
  e->depth_src = (!peaks && ((pf != 0) != (morph != 0))) ? agg : dout;
  e->stream = saved;
  return st;
}

}  // namespace

namespace {
// A match without initial disparities or a right map on stream s (0: the matcher's own). Without
// profiling, the second and later calls replay a CUDA graph of the match on the matcher's own
// buffers, with device-to-device copies around it when the caller's buffers differ.
int engine_run(sgm_engine* e, const uint8_t* dl, const uint8_t* dr, float* dout, cudaStream_t s, int mode = 0) {
  if (!s) s = e->stream;
  if (g_prof.on) {
    e->drop_graph();
    return engine_enqueue(e, dl, dr, nullptr, dout, nullptr, s);
  }
  cudaGraphExec_t& gexec = e->gexec[mode];
  if (!gexec && e->direct_runs[mode] == 0) {
    e->direct_runs[mode]++;
    return engine_enqueue(e, dl, dr, nullptr, dout, nullptr, s);
  }
  const size_t N = e->npix();
  if (!gexec) {
    if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      set_error(&e->err, "graph capture could not start");
      return SGM_ERR_CUDA;
    }
    e->launches = 0;
    const int st = engine_enqueue(e, e->img[0], e->img[1], nullptr, e->out, nullptr, e->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (st || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      if (!st) set_error(&e->err, "graph capture failed: %s", cudaGetErrorString(ce));
      return st ? st : SGM_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&gexec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      gexec = nullptr;
      set_error(&e->err, "graph instantiation failed: %s", cudaGetErrorString(ie));
      return SGM_ERR_CUDA;
    }
    e->graph_launches[mode] = e->launches;
  }
  if (dl != e->img[0]) SGM_CUDA_TRY(e, cudaMemcpyAsync(e->img[0], dl, N, cudaMemcpyDeviceToDevice, s));
  if (dr != e->img[1]) SGM_CUDA_TRY(e, cudaMemcpyAsync(e->img[1], dr, N, cudaMemcpyDeviceToDevice, s));
  SGM_CUDA_TRY(e, cudaGraphLaunch(gexec, s));
  if (dout != e->out) SGM_CUDA_TRY(e, cudaMemcpyAsync(dout, e->out, N * sizeof(float), cudaMemcpyDeviceToDevice, s));
  e->launches = e->graph_launches[mode];
  return SGM_OK;
}

// The synchronous host API (the reference's Match) adapts to the number of such calls in flight in
// the process (measured with page-locked buffers at 1242x375x64 on one B200, 16 host cores). While
// at most kLatencyInFlight calls are in flight -- a few callers matching one frame at a time --
//  * a matcher left at the default tuning takes the warp-per-scanline kernels (variant 4, the
//    shortest step chains: a pyramid pair 0.33 instead of 1.46 ms alone); with more calls in flight
//    the default thread-per-scanline kernels, which give more pairs per second once many pairs
//    share the GPU (16 callers: 7.4 k plain pairs/s against 6.0 k). Both give the same bits;
//  * the call polls for its results (one caller: 3.3 k plain pairs/s against 2.0 k sleeping),
//    until more calls are in flight; then it sleeps, and the cores go to the callers that submit
//    work (96 callers: 10.9 k pyramid pairs/s, 10.2 k when up to 16 of them poll).
constexpr int kLatencyInFlight = 8;
std::atomic<int> g_host_in_flight{0};

bool few_host_calls() { return g_host_in_flight.load(std::memory_order_relaxed) <= kLatencyInFlight; }

struct HostCall {
  int n;
  HostCall() : n(++g_host_in_flight) {}
  ~HostCall() { --g_host_in_flight; }
  HostCall(const HostCall&) = delete;
  HostCall& operator=(const HostCall&) = delete;
  bool latency() const { return n <= kLatencyInFlight; }
  bool (*poll() const)() { return latency() ? few_host_calls : nullptr; }
};

// Row and column kernels set to variant 4 on the given engines for the scope of one match, when
// `latency` and every engine is at the default tuning; mode() is the graph slot to use.
struct KernelMode {
  sgm_engine* const* lv;
  int n;
  bool on = false;
  KernelMode(sgm_engine* const* levels, int count, bool latency) : lv(levels), n(count) {
    if (!latency) return;
    for (int i = 0; i < n; ++i)
      if (!lv[i]->tuning_is_default()) return;
    on = true;
    for (int i = 0; i < n; ++i) lv[i]->tune_row_kernel = lv[i]->tune_col_kernel = 4;
  }
  ~KernelMode() {
    if (on)
      for (int i = 0; i < n; ++i) lv[i]->tune_row_kernel = lv[i]->tune_col_kernel = 0;
  }
  KernelMode(const KernelMode&) = delete;
  KernelMode& operator=(const KernelMode&) = delete;
  int mode() const { return on ? 1 : 0; }
};

int enqueue_depth(sgm_engine* e, const float* disp, float* depth, const sgm_camera_t& c, cudaStream_t s) {
  const int n = (int)e->npix();
  return SGM_LAUNCH(e, s, "depth", sgm::k_depth<<<(n + 255) / 256, 256, 0, s>>>(
                                       disp, depth, n, c.baseline * c.focus, c.x0_right - c.x0_left));
}
}  // namespace

// ------------------------------------------------------------------------------------------
// Pyramid matcher
// ------------------------------------------------------------------------------------------
struct sgm_pyramid {
  bool ready = false;
  int W = 0, H = 0, layers = 0;
  std::vector<sgm_engine*> lv;
  std::vector<uint8_t*> imgs_l, imgs_r;  // decimated images per level (level 0 unused)
  std::vector<float*> disp;              // per-level output (level 0 unused)
  std::vector<int16_t*> init;            // initial disparity per level (coarsest unused)
  uint8_t* in_l = nullptr;
  uint8_t* in_r = nullptr;
  float* out = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;
  bool depth_mode = false;
  sgm_camera_t cam0{};
  float* disp0 = nullptr;  // finest-level disparity in depth mode
  // The whole pyramid (in_l, in_r -> out) captured once as a CUDA graph after a first direct run;
  // later matches copy in, launch it, copy out. One graph per kernel mode (see KernelMode).
  cudaGraphExec_t gexec[2] = {};
  int direct_runs[2] = {};
  int64_t graph_launches[2] = {};  // kernels inside the graph
  cudaEvent_t done = nullptr;  // blocking-sync event of the synchronous host API (see wait_stream)

  void drop_graph() {
    for (int k = 0; k < 2; ++k) {
      if (gexec[k]) cudaGraphExecDestroy(gexec[k]);
      gexec[k] = nullptr;
      direct_runs[k] = 0;
    }
  }

  void free_all() {
    drop_graph();
    if (done) cudaEventDestroy(done);
    done = nullptr;
    if (disp0) sgm_dev_free(disp0);
    disp0 = nullptr;
    depth_mode = false;
    for (auto* e : lv) {
      if (e) { e->free_all(); delete e; }
    }
    lv.clear();
    for (auto* p : imgs_l) if (p) sgm_dev_free(p);
    for (auto* p : imgs_r) if (p) sgm_dev_free(p);
    for (auto* p : disp) if (p) sgm_dev_free(p);
    for (auto* p : init) if (p) sgm_dev_free(p);
    imgs_l.clear(); imgs_r.clear(); disp.clear(); init.clear();
    if (in_l) sgm_dev_free(in_l);
    if (in_r) sgm_dev_free(in_r);
    if (out) sgm_dev_free(out);
    in_l = in_r = nullptr;
    out = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    ready = false;
  }
};

namespace {

// SetSgmParameters (FasterStereoCuda.cpp:169-199) with the optional census/penalty override,
// and the disparity-range rules of HierSgmCudaImpl::Init (:264-288).

int pyr_enqueue(sgm_pyramid* p, const uint8_t* dl, const uint8_t* dr, float* dout, cudaStream_t s) {
  const int L = p->layers;
  int st = SGM_OK;
  for (int n = 1; n < L && !st; ++n) {
    sgm_engine* e = p->lv[n];
    dim3 g((e->W + 127) / 128, e->H);
    prof_start(s);
    sgm::k_decimate<<<g, 128, 0, s>>>(dl, dr, p->imgs_l[n], p->imgs_r[n], p->W, e->W, e->H, n);
    prof_end("decimate");
    p->launches++;
    if (cudaGetLastError() != cudaSuccess) st = SGM_ERR_CUDA;
  }
  for (int n = L - 1; n >= 0 && !st; --n) {
    sgm_engine* e = p->lv[n];
    const uint8_t* il = n == 0 ? dl : p->imgs_l[n];
    const uint8_t* ir = n == 0 ? dr : p->imgs_r[n];
    float* o = n == 0 ? dout : p->disp[n];
    const int64_t before = e->launches;
    if (n == 0 && p->depth_mode) o = p->disp0;
    st = engine_enqueue(e, il, ir, n < L - 1 ? p->init[n] : nullptr, o, nullptr, s);
    if (!st && n == 0 && p->depth_mode) st = enqueue_depth(e, e->depth_src, dout, p->cam0, s);
    p->launches += e->launches - before;
    if (st) {
      p->err = e->err;
      break;
    }
    if (n > 0) {
      sgm_engine* f = p->lv[n - 1];
      dim3 g((f->W + 127) / 128, f->H);
      prof_start(s);
      sgm::k_init_next_level<<<g, 128, 0, s>>>(p->disp[n], (long)e->W * e->H, p->init[n - 1], f->W, f->H);
      prof_end("init_next_level");
      p->launches++;
      if (cudaGetLastError() != cudaSuccess) st = SGM_ERR_CUDA;
    }
  }
  return st;
}

// One pyramid match on stream s. Without profiling, the second and later calls replay a CUDA
// graph of the whole pyramid on the matcher's own buffers (one launch instead of one per
// kernel), with device-to-device copies around it when the caller's buffers differ.
int pyr_run(sgm_pyramid* p, const uint8_t* dl, const uint8_t* dr, float* dout, cudaStream_t s, int mode = 0) {
  if (g_prof.on) {
    p->drop_graph();
    return pyr_enqueue(p, dl, dr, dout, s);
  }
  cudaGraphExec_t& gexec = p->gexec[mode];
  if (!gexec && p->direct_runs[mode] == 0) {
    p->direct_runs[mode]++;
    return pyr_enqueue(p, dl, dr, dout, s);
  }
  const size_t N = (size_t)p->W * p->H;
  if (!gexec) {
    if (cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      p->err = "graph capture could not start";
      return SGM_ERR_CUDA;
    }
    p->launches = 0;
    const int st = pyr_enqueue(p, p->in_l, p->in_r, p->out, p->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(p->stream, &g);
    if (st || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      if (!st) p->err = std::string("graph capture failed: ") + cudaGetErrorString(ce);
      return st ? st : SGM_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&gexec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      gexec = nullptr;
      p->err = std::string("graph instantiation failed: ") + cudaGetErrorString(ie);
      return SGM_ERR_CUDA;
    }
    p->graph_launches[mode] = p->launches;
  }
  if (dl != p->in_l && cudaMemcpyAsync(p->in_l, dl, N, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return SGM_ERR_CUDA;
  if (dr != p->in_r && cudaMemcpyAsync(p->in_r, dr, N, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return SGM_ERR_CUDA;
  if (cudaGraphLaunch(gexec, s) != cudaSuccess) {
    p->err = "graph launch failed";
    return SGM_ERR_CUDA;
  }
  if (dout != p->out && cudaMemcpyAsync(dout, p->out, N * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return SGM_ERR_CUDA;
  p->launches = p->graph_launches[mode];
  return SGM_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
extern "C" {

int sgm_create(sgm_handle_t* out) {
  if (!out) return SGM_ERR_ARG;
  *out = new (std::nothrow) sgm_engine();
  return *out ? SGM_OK : SGM_ERR_NOMEM;
}

int sgm_destroy(sgm_handle_t h) {
  if (!h) return SGM_ERR_ARG;
  h->free_all();
  delete h;
  return SGM_OK;
}

int sgm_init(sgm_handle_t h, int32_t width, int32_t height, int32_t min_disparity, int32_t disp_range,
             const sgm_option_t* option, int32_t print_log) {
  if (!h || !option) return SGM_ERR_ARG;
  const int st = engine_init(h, width, height, min_disparity, disp_range, option, print_log != 0);
  if (st) h->free_all();
  return st;
}

int sgm_set_ext_options(sgm_handle_t h, const sgm_ext_options_t* ext) {
  if (!h || !ext) return SGM_ERR_ARG;
  if (ext->tie_rule < 0 || ext->tie_rule > 4 || ext->init_tie_rule < 0 || ext->init_tie_rule > 4 ||
      ext->peaks_abs_mode < 0 || ext->peaks_abs_mode > 1) {
    set_error(&h->err, "extended option out of range");
    return SGM_ERR_ARG;
  }
  h->ext = *ext;
  h->drop_graph();
  return SGM_OK;
}

int sgm_get_ext_options(sgm_handle_t h, sgm_ext_options_t* ext) {
  if (!h || !ext) return SGM_ERR_ARG;
  *ext = h->ext;
  return SGM_OK;
}

namespace {
bool tuning_ok(const sgm_tuning_t* t) {
  const int r = t->rows_per_cta, c = t->cols_per_cta;
  return t->row_kernel >= 0 && t->row_kernel <= 4 && t->col_kernel >= 0 && t->col_kernel <= 4 &&
         (r == 0 || r == 1 || r == 2 || r == 4) && c >= 0 && c <= 8 && (t->bt_smem == 0 || t->bt_smem == 1) &&
         (t->row_lanes == 0 || t->row_lanes == 1 || t->row_lanes == 2 || t->row_lanes == 4 || t->row_lanes == 8) &&
         (t->col_lanes == 0 || t->col_lanes == 1 || t->col_lanes == 2 || t->col_lanes == 4 || t->col_lanes == 8);
}
void apply_tuning(sgm_engine* e, const sgm_tuning_t* t) {
  e->tune_row_kernel = t->row_kernel;
  e->tune_rows = t->rows_per_cta;
  e->tune_col_kernel = t->col_kernel;
  e->tune_cols = t->cols_per_cta;
  e->tune_bt_smem = t->bt_smem;
  e->tune_row_lanes = t->row_lanes;
  e->tune_col_lanes = t->col_lanes;
}
}  // namespace

int sgm_set_tuning(sgm_handle_t h, const sgm_tuning_t* t) {
  if (!h || !t) return SGM_ERR_ARG;
  if (!tuning_ok(t)) {
    set_error(&h->err, "tuning out of range (kernels 0-4, rows per CTA 0/1/2/4, columns per CTA 0-8, bt_smem 0/1)");
    return SGM_ERR_ARG;
  }
  apply_tuning(h, t);
  h->drop_graph();
  return SGM_OK;
}

int sgm_get_tuning(sgm_handle_t h, sgm_tuning_t* t) {
  if (!h || !t) return SGM_ERR_ARG;
  t->row_kernel = h->tune_row_kernel;
  t->rows_per_cta = h->tune_rows;
  t->col_kernel = h->tune_col_kernel;
  t->cols_per_cta = h->tune_cols;
  t->bt_smem = h->tune_bt_smem;
  t->row_lanes = h->tune_row_lanes;
  t->col_lanes = h->tune_col_lanes;
  return SGM_OK;
}

int sgm_match(sgm_handle_t h, const uint8_t* img_left, const uint8_t* img_right, float* disp_left,
              float* disp_right, const int16_t* init_disp_left, const sgm_roi_t* roi_left,
              const sgm_roi_t* roi_right) {
  if (!h) return SGM_ERR_ARG;
  if (!img_left || !img_right || !disp_left) {
    set_error(&h->err, "null image or output pointer");
    return SGM_ERR_ARG;
  }
  if (!h->ready) {
    set_error(&h->err, "matcher not initialised");
    return SGM_ERR_STATE;
  }
  const size_t N = h->npix();
  h->launches = 0;
  const HostCall call;
  const KernelMode km(&h, 1, call.latency());
  // with print_log: per-stage times, printed like the reference's timers (StereoCudaImpl.cpp:
  // 365-460, 530-543); the match then runs its kernels directly instead of as a graph
  h->stage_timing = h->print_log;
  h->nstage = 0;
  if (h->stage_timing)
    for (auto& ev : h->stage_ev)
      if (!ev) SGM_CUDA_TRY(h, cudaEventCreate(&ev));
  stage_mark(h, "input");
  SGM_CUDA_TRY(h, cudaMemcpyAsync(h->img[0], img_left, N, cudaMemcpyHostToDevice, h->stream));
  SGM_CUDA_TRY(h, cudaMemcpyAsync(h->img[1], img_right, N, cudaMemcpyHostToDevice, h->stream));
  if (init_disp_left)
    SGM_CUDA_TRY(h, cudaMemcpyAsync(h->init[0], init_disp_left, N * sizeof(int16_t), cudaMemcpyHostToDevice, h->stream));
  const bool right = disp_right && h->opt.do_lr_check;
  const bool roi = roi_left || (roi_right && h->opt.do_lr_check);
  int st = (!init_disp_left && !right && !roi && !h->stage_timing)
               ? engine_run(h, h->img[0], h->img[1], h->out, h->stream, km.mode())
               : engine_enqueue(h, h->img[0], h->img[1], init_disp_left ? h->init[0] : nullptr, h->out,
                                right ? h->dr_out : nullptr, h->stream, roi_left, roi_right);
  if (st) {
    h->stage_timing = false;
    return st;
  }
  if (h->stage_timing) stage_mark(h, "output");
  SGM_CUDA_TRY(h, cudaMemcpyAsync(disp_left, h->out, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (disp_right && h->opt.do_lr_check)
    SGM_CUDA_TRY(h, cudaMemcpyAsync(disp_right, h->dr_out, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  if (h->stage_timing) stage_mark(h, nullptr);
  SGM_CUDA_TRY(h, wait_stream(h->stream, &h->done, call.poll()));
  if (disp_right && !h->opt.do_lr_check)
    for (size_t i = 0; i < N; ++i) disp_right[i] = sgm::kInvalidFloat;
  if (h->stage_timing) {
    printf("Timing:\n");
    float total = 0.0f;
    for (int i = 0; i + 1 < h->nstage; ++i) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, h->stage_ev[i], h->stage_ev[i + 1]);
      if (h->stage_name[i]) printf("** %-28s %.3f ms\n", h->stage_name[i], ms);
      total += ms;
    }
    printf("** %-28s %.3f ms\n", "total", total);
    h->stage_timing = false;
  }
  return SGM_OK;
}

int sgm_match_device(sgm_handle_t h, const uint8_t* d_left, const uint8_t* d_right, float* d_disp_left,
                     float* d_disp_right, const int16_t* d_init_disp_left, void* stream) {
  if (!h) return SGM_ERR_ARG;
  if (!d_left || !d_right || !d_disp_left) {
    set_error(&h->err, "null device pointer");
    return SGM_ERR_ARG;
  }
  if (d_disp_right && !h->opt.do_lr_check) {
    set_error(&h->err, "a right disparity map needs the left-right check");
    return SGM_ERR_ARG;
  }
  h->launches = 0;
  if (!d_init_disp_left && !d_disp_right) return engine_run(h, d_left, d_right, d_disp_left, (cudaStream_t)stream);
  return engine_enqueue(h, d_left, d_right, d_init_disp_left, d_disp_left, d_disp_right, (cudaStream_t)stream);
}

int sgm_init2(sgm_handle_t h, int32_t width, int32_t height, int32_t min_disparity, int32_t disp_range,
              const sgm_option_t* option, const sgm_camera_t* camera, int32_t print_log) {
  if (!h || !option || !camera) return SGM_ERR_ARG;
  const int st = sgm_init(h, width, height, min_disparity, disp_range, option, print_log);
  if (st) return st;
  h->cam = *camera;
  h->has_cam = true;
  return SGM_OK;
}

int sgm_match2(sgm_handle_t h, const uint8_t* img_left, const uint8_t* img_right, float* depth_left,
               const int16_t* init_disp_left, const sgm_roi_t* roi_left, const sgm_roi_t* roi_right) {
  if (!h) return SGM_ERR_ARG;
  if (!h->has_cam) {
    set_error(&h->err, "Match2 needs Init2 (camera parameters)");
    return SGM_ERR_STATE;
  }
  if (!img_left || !img_right || !depth_left) return SGM_ERR_ARG;
  const size_t N = h->npix();
  h->launches = 0;
  const HostCall call;
  const KernelMode km(&h, 1, call.latency());
  SGM_CUDA_TRY(h, cudaMemcpyAsync(h->img[0], img_left, N, cudaMemcpyHostToDevice, h->stream));
  SGM_CUDA_TRY(h, cudaMemcpyAsync(h->img[1], img_right, N, cudaMemcpyHostToDevice, h->stream));
  if (init_disp_left)
    SGM_CUDA_TRY(h, cudaMemcpyAsync(h->init[0], init_disp_left, N * sizeof(int16_t), cudaMemcpyHostToDevice, h->stream));
  int st = engine_enqueue(h, h->img[0], h->img[1], init_disp_left ? h->init[0] : nullptr, h->out, nullptr, h->stream,
                          roi_left, roi_right);
  // the depth source is the final map, the LR / median output or the WTA map, never h->post
  if (!st) st = enqueue_depth(h, h->depth_src, h->post, h->cam, h->stream);
  if (st) return st;
  SGM_CUDA_TRY(h, cudaMemcpyAsync(depth_left, h->post, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  SGM_CUDA_TRY(h, wait_stream(h->stream, &h->done, call.poll()));
  return SGM_OK;
}

int sgm_release(sgm_handle_t h) {
  if (!h) return SGM_ERR_ARG;
  h->free_all();
  return SGM_OK;
}

int sgm_set_min_disparity(sgm_handle_t h, int32_t min_disparity) {
  if (!h) return SGM_ERR_ARG;
  if (h->ready && min_disparity >= h->W) {
    set_error(&h->err, "minimum disparity %d leaves no pixel of a %d-pixel row to match", min_disparity, h->W);
    return SGM_ERR_ARG;
  }
  h->M = min_disparity;
  h->drop_graph();  // kernel parameters are part of the graph
  return SGM_OK;
}

int32_t sgm_get_disparity_range(sgm_handle_t h) { return h ? h->D : 0; }

void sgm_roi_from_disp_map(const float* disp, int32_t width, int32_t height, sgm_roi_t* roi) {
  // StereoCudaImpl::GetRoiFromDispMap (StereoCudaImpl.cpp:585-628), same scan order
  if (!disp || !roi) return;
  const int size = width * height;
  int n = 0;
  for (n = 0; n < size; n++)
    if (disp[n] != sgm::kInvalidFloat) break;
  roi->y = n / width;
  const int size0 = roi->y * width;
  for (n = size - 1; n > size0; n--)
    if (disp[n] != sgm::kInvalidFloat) break;
  roi->h = n / width - roi->y + 1;
  bool done = false;
  for (int j = 0; j < width && !done; j++)
    for (int i = 0; i < height; i++)
      if (disp[i * width + j] != sgm::kInvalidFloat) { roi->x = j; done = true; break; }
  done = false;
  for (int j = width - 1; j > roi->x && !done; j--)
    for (int i = 0; i < height; i++)
      if (disp[i * width + j] != sgm::kInvalidFloat) { roi->w = j - roi->x + 1; done = true; break; }
}

float sgm_invalid_float(void) { return sgm::kInvalidFloat; }
int16_t sgm_invalid_short(void) { return sgm::kInvalidShort; }
int16_t sgm_level_range(void) { return (int16_t)sgm::kLevelRange; }

int sgm_malloc_page_locked(void** ptr, size_t size) {
  if (!ptr) return SGM_ERR_ARG;
  return cudaHostAlloc(ptr, size, cudaHostAllocDefault) == cudaSuccess ? SGM_OK : SGM_ERR_NOMEM;
}

int sgm_free_page_locked(void* ptr) {
  if (!ptr) return SGM_ERR_ARG;
  return cudaFreeHost(ptr) == cudaSuccess ? SGM_OK : SGM_ERR_CUDA;
}

const char* sgm_last_error(sgm_handle_t h) { return h ? h->err.c_str() : g_last_error.c_str(); }

int64_t sgm_kernel_launches(sgm_handle_t h) { return h ? h->launches : 0; }

int sgm_debug_read(sgm_handle_t h, int32_t which, int32_t view, void* dst, size_t bytes) {
  if (!h || !dst || view < 0 || view > 1) return SGM_ERR_ARG;
  if (!h->ready) return SGM_ERR_STATE;
  const size_t N = h->npix(), V = h->vol();
  if (cudaStreamSynchronize(h->stream) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return SGM_ERR_CUDA;
  if (which == 0 || which == 1) {
    if (bytes != N * 8) return SGM_ERR_ARG;
    const int wb = h->census_bytes();
    std::vector<uint8_t> tmp(N * wb);
    if (cudaMemcpy(tmp.data(), h->cs[which], N * wb, cudaMemcpyDeviceToHost) != cudaSuccess) return SGM_ERR_CUDA;
    uint64_t* out = static_cast<uint64_t*>(dst);
    for (size_t i = 0; i < N; ++i) {
      uint64_t v = 0;
      memcpy(&v, tmp.data() + i * wb, wb);
      out[i] = v;
    }
    return SGM_OK;
  }
  const uint8_t* src = nullptr;
  size_t n = V;
  if (which >= 2 && which <= 5 && view >= h->nviews()) {
    set_error(&h->err, "no right-view volumes without the left-right check");
    return SGM_ERR_ARG;
  }
  switch (which) {
    case 2: src = h->cost + view * V; break;
    case 3: src = h->lr + view * V; break;
    case 4: src = h->rl + view * V; break;
    case 5:
      if (!h->bt_stored) {
        set_error(&h->err, "the last match kept the bottom->top path costs in shared memory");
        return SGM_ERR_STATE;
      }
      src = h->bt + view * V;
      break;
    case 6: src = reinterpret_cast<const uint8_t*>(h->wta + view * N); n = N * sizeof(float); break;
    default: return SGM_ERR_ARG;
  }
  if (bytes != n) return SGM_ERR_ARG;
  return cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost) == cudaSuccess ? SGM_OK : SGM_ERR_CUDA;
}

int64_t sgm_debug_wait_timeouts(void) {
  unsigned int n = 0;
  if (cudaMemcpyFromSymbol(&n, sgm::g_scan_wait_timeouts, sizeof(n)) != cudaSuccess) return -1;
  const int64_t f = sgm_float_wait_timeouts();
  return f < 0 ? -1 : n + f;
}

int sgm_debug_scan_wait(int64_t max_polls, int32_t short_copy) {
  const unsigned int limit = max_polls > 0 && max_polls < sgm::kMaxWaitTries ? (unsigned int)max_polls
                                                                               : (unsigned int)sgm::kMaxWaitTries;
  const unsigned int sc = short_copy ? 1u : 0u;
  if (cudaMemcpyToSymbol(sgm::g_wait_limit, &limit, sizeof(limit)) != cudaSuccess ||
      cudaMemcpyToSymbol(sgm::g_short_copy, &sc, sizeof(sc)) != cudaSuccess)
    return SGM_ERR_CUDA;
  return SGM_OK;
}

int sgm_debug_reset_wait_timeouts(void) {
  const unsigned int z = 0;
  return cudaMemcpyToSymbol(sgm::g_scan_wait_timeouts, &z, sizeof(z)) == cudaSuccess ? SGM_OK : SGM_ERR_CUDA;
}

int sgm_debug_fail_device_alloc(int64_t after) {
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  g_alloc_fail_after = after < 0 ? -1 : after;
  return SGM_OK;
}

int64_t sgm_debug_live_device_allocations(void) {
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  return g_alloc_live;
}

int sgm_profile_enable(int32_t enable) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof.collect();
  g_prof.stats.clear();
  g_prof.on = enable != 0;
  return SGM_OK;
}

int sgm_profile_read(char* buf, size_t cap) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof.collect();
  std::string js = "{";
  for (size_t i = 0; i < g_prof.stats.size(); ++i) {
    char item[256];
    snprintf(item, sizeof(item), "%s\"%s\": {\"launches\": %lld, \"ms\": %.6f}", i ? ", " : "",
             g_prof.stats[i].name.c_str(), (long long)g_prof.stats[i].launches, g_prof.stats[i].ms);
    js += item;
  }
  js += "}";
  if (!buf || cap < js.size() + 1) return (int)(js.size() + 1);
  memcpy(buf, js.c_str(), js.size() + 1);
  return SGM_OK;
}

int sgm_pyr_create(sgm_pyr_handle_t* out) {
  if (!out) return SGM_ERR_ARG;
  *out = new (std::nothrow) sgm_pyramid();
  return *out ? SGM_OK : SGM_ERR_NOMEM;
}

int sgm_pyr_destroy(sgm_pyr_handle_t h) {
  if (!h) return SGM_ERR_ARG;
  h->free_all();
  delete h;
  return SGM_OK;
}

int sgm_pyr_init(sgm_pyr_handle_t h, const sgm_pyr_option1_t* o, const sgm_level_override_t* ov,
                 const sgm_ext_options_t* ext) {
  if (!h || !o) return SGM_ERR_ARG;
  h->free_all();
  if (o->width <= 0 || o->height <= 0) {
    set_error(&h->err, "image size error");
    return SGM_ERR_ARG;
  }
  const int L = std::max(1, o->num_layers);
  if ((o->width >> (L - 1)) < 8 || (o->height >> (L - 1)) < 8) {
    set_error(&h->err, "too many layers for a %dx%d image", o->width, o->height);
    return SGM_ERR_ARG;
  }
  h->W = o->width;
  h->H = o->height;
  h->layers = L;
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return SGM_ERR_CUDA;
  h->lv.assign(L, nullptr);
  h->imgs_l.assign(L, nullptr);
  h->imgs_r.assign(L, nullptr);
  h->disp.assign(L, nullptr);
  h->init.assign(L, nullptr);
  for (int i = 0; i < L; ++i) {
    sgm_option_t so;
    int dmin = 0, dr = 0;
    level_options(o, ov, i, L, &so, &dmin, &dr);
    h->lv[i] = new sgm_engine();
    if (ext) h->lv[i]->ext = *ext;
    const int w = o->width >> i, hh = o->height >> i;
    int st = engine_init(h->lv[i], w, hh, dmin, dr, &so, false);
    if (st) {
      h->err = h->lv[i]->err;
      h->free_all();
      return st;
    }
    const size_t n = (size_t)w * hh;
    if (i > 0) {
      if (sgm_dev_malloc(&h->imgs_l[i], n) || sgm_dev_malloc(&h->imgs_r[i], n) ||
          sgm_dev_malloc(&h->disp[i], n * sizeof(float))) {
        h->free_all();
        return SGM_ERR_NOMEM;
      }
    }
    if (i < L - 1 && sgm_dev_malloc(&h->init[i], n * sizeof(int16_t))) {
      h->free_all();
      return SGM_ERR_NOMEM;
    }
  }
  const size_t N = (size_t)o->width * o->height;
  if (sgm_dev_malloc(&h->in_l, N) || sgm_dev_malloc(&h->in_r, N) || sgm_dev_malloc(&h->out, N * sizeof(float))) {
    h->free_all();
    return SGM_ERR_NOMEM;
  }
  h->ready = true;
  return SGM_OK;
}

int sgm_pyr_match(sgm_pyr_handle_t h, const uint8_t* img_left, const uint8_t* img_right, float* disp) {
  if (!h) return SGM_ERR_ARG;
  if (!h->ready) return SGM_ERR_STATE;
  if (!img_left || !img_right || !disp) return SGM_ERR_ARG;
  const size_t N = (size_t)h->W * h->H;
  h->launches = 0;
  const HostCall call;
  const KernelMode km(h->lv.data(), (int)h->lv.size(), call.latency());
  if (cudaMemcpyAsync(h->in_l, img_left, N, cudaMemcpyHostToDevice, h->stream) ||
      cudaMemcpyAsync(h->in_r, img_right, N, cudaMemcpyHostToDevice, h->stream))
    return SGM_ERR_CUDA;
  int st = pyr_run(h, h->in_l, h->in_r, h->out, h->stream, km.mode());
  if (st) return st;
  if (cudaMemcpyAsync(disp, h->out, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream)) return SGM_ERR_CUDA;
  if (wait_stream(h->stream, &h->done, call.poll()) != cudaSuccess) {
    set_error(&h->err, "pyramid match failed: %s", cudaGetErrorString(cudaGetLastError()));
    return SGM_ERR_CUDA;
  }
  return SGM_OK;
}

int sgm_pyr_match_device(sgm_pyr_handle_t h, const uint8_t* d_left, const uint8_t* d_right, float* d_disp,
                         void* stream) {
  if (!h) return SGM_ERR_ARG;
  if (!h->ready) return SGM_ERR_STATE;
  if (!d_left || !d_right || !d_disp) return SGM_ERR_ARG;
  h->launches = 0;
  return pyr_run(h, d_left, d_right, d_disp, stream ? (cudaStream_t)stream : h->stream);
}

int sgm_pyr_init2(sgm_pyr_handle_t h, const sgm_pyr_option2_t* o, const sgm_level_override_t* ov,
                  const sgm_ext_options_t* ext) {
  if (!h || !o) return SGM_ERR_ARG;
  if (!(o->min_depth > 0.0f) || !(o->max_depth > o->min_depth)) {
    set_error(&h->err, "depth range must satisfy 0 < min_depth < max_depth");
    return SGM_ERR_ARG;
  }
  // HierSgmCudaImpl::Init2 (FasterStereoCuda.cpp:339-399): disparity range of the coarsest level from
  // the depth range seen by the camera scaled to that level; the finer levels search 32 disparities.
  const int L = std::max(1, o->num_layers);
  const int scale = 1 << (L - 1);
  const double x0l = o->epi.x0_left / scale, x0r = o->epi.x0_right / scale, f = o->epi.focus / scale;
  double dmin = o->epi.baseline * f / o->max_depth - x0r + x0l;
  const double dmax = o->epi.baseline * f / o->min_depth - x0r + x0l;
  double range = dmax - dmin;
  int k = 6;
  while (std::pow(2.0, k) < range && k < 30) ++k;
  range = std::pow(2.0, k);
  if (range > 2.0 * o->width) range /= 2;
  if (dmin >= o->width) {
    dmin = o->width - range;
    if (dmin < -o->width) dmin = -o->width;
  }
  // express the coarsest range as the min/max pair the disparity initialisation understands
  sgm_pyr_option1_t o1;
  o1.width = o->width;
  o1.height = o->height;
  o1.num_layers = L;
  o1.do_lr_check = o->do_lr_check;
  o1.do_rm_peaks = o->do_rm_peaks;
  o1.do_smooth = o->do_smooth;
  o1.min_disp = (int)std::floor(dmin) * scale;
  o1.max_disp = o1.min_disp + (int)range * scale;
  int st = sgm_pyr_init(h, &o1, ov, ext);
  if (st) return st;
  sgm_engine* c = h->lv[L - 1];
  if (c->M != (int)std::floor(dmin) || c->D != (int)range) {
    // fall back to setting the coarsest level directly when the integer round trip differs
    sgm_option_t so = c->opt;
    sgm_ext_options_t ex = c->ext;
    st = engine_init(c, c->W, c->H, (int)std::floor(dmin), (int)range, &so, false);
    c->ext = ex;
    if (st) {
      h->err = c->err;
      h->free_all();
      return st;
    }
  }
  h->cam0.x0_left = o->epi.x0_left;
  h->cam0.y0_left = o->epi.y0_left;
  h->cam0.x0_right = o->epi.x0_right;
  h->cam0.y0_right = o->epi.y0_right;
  h->cam0.focus = o->epi.focus;
  h->cam0.baseline = o->epi.baseline;
  if (sgm_dev_malloc(&h->disp0, (size_t)o->width * o->height * sizeof(float)) != cudaSuccess) {
    h->free_all();
    return SGM_ERR_NOMEM;
  }
  h->depth_mode = true;
  return SGM_OK;
}

int sgm_pyr_match2(sgm_pyr_handle_t h, const uint8_t* img_left, const uint8_t* img_right, float* depth) {
  if (!h) return SGM_ERR_ARG;
  if (!h->ready || !h->depth_mode) {
    set_error(&h->err, "Match2 needs Init2");
    return SGM_ERR_STATE;
  }
  return sgm_pyr_match(h, img_left, img_right, depth);
}

int sgm_pyr_release(sgm_pyr_handle_t h) {
  if (!h) return SGM_ERR_ARG;
  h->free_all();
  return SGM_OK;
}

int sgm_pyr_level_info(sgm_pyr_handle_t h, int32_t level, int32_t* width, int32_t* height, int32_t* min_disp,
                       int32_t* disp_range) {
  if (!h || !h->ready || level < 0 || level >= h->layers) return SGM_ERR_ARG;
  const sgm_engine* e = h->lv[level];
  if (width) *width = e->W;
  if (height) *height = e->H;
  if (min_disp) *min_disp = e->M;
  if (disp_range) *disp_range = e->D;
  return SGM_OK;
}

int64_t sgm_pyr_kernel_launches(sgm_pyr_handle_t h) { return h ? h->launches : 0; }

int sgm_pyr_set_tuning(sgm_pyr_handle_t h, int32_t level, const sgm_tuning_t* t) {
  if (!h || !t) return SGM_ERR_ARG;
  if (!h->ready || level < -1 || level >= h->layers) {
    h->err = "tuning: matcher not initialised or level out of range";
    return SGM_ERR_ARG;
  }
  if (!tuning_ok(t)) {
    h->err = "tuning out of range (kernels 0-4, rows per CTA 0/1/2/4, columns per CTA 0-8, bt_smem 0/1)";
    return SGM_ERR_ARG;
  }
  for (int i = 0; i < h->layers; ++i)
    if (level < 0 || level == i) apply_tuning(h->lv[i], t);
  h->drop_graph();
  return SGM_OK;
}

}  // extern "C"
