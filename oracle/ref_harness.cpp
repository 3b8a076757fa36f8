// Reference dump harness -- TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/build_ref.sh against the reference's own headers and linked with the
// reference built from its sources (oracle/_ref/libsgmref.so). It drives the reference's
// classes exactly as StereoCudaImpl::Match does and copies every stage buffer out, so the
// oracle can be checked against the reference itself. Access to the reference's private
// members comes from compiling this file with -Dprivate=public.
//
// Safety: the reference writes up to 3 floats past the end of each disparity row (WTA grid
// rounding) and reads one float past it (LR check, x == width); the initial-disparity WTA
// reads up to 3 int16 past each row. ref_match_dump() refuses a case unless the pitched
// allocations leave that much padding, and it refuses the kernels that index shared memory
// past their allocation (D = 32 without initial disparities, D = 128, D = 256).
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "StereoCudaImpl.h"
#include "cusgm_ca.cuh"
#include "cusgm_cc.cuh"
#include "cusgm_df.h"
#include "FasterStereoCuda.h"

// Reference host functions (StereoCudaImpl.cpp:32, FasterStereoCuda.cpp:114, :138 and :169).
void SetSgmParameters(const bool& do_lr_check, const bool& do_rm_peaks, const bool& do_smooth, CuSGMOption& sgm_param,
                      int layer_id, int num_layers);
sint32 RemovePeaks(float32* disp_map, sint32* segid, sint32 w, sint32 h, sint32 threshold);
void Zoom(const unsigned char* src, unsigned char* dst, int w_src, int h_src, int scale_x, int scale_y);
int ComputeInitDispInNextLevel(float* cur, short* next, int width, int height);

extern "C" {

struct ref_case_t {
  int32_t width, height, min_disp, disp_range;
  int32_t cs_type, p1, p2;
  float uniqueness;
  int32_t do_lr_check;
  float lr_threshold;
  int32_t do_median;
  int32_t morphology;  // 0 none, 1 erosion, 2 dilation, 3 open, 4 close
  int32_t do_remove_peaks;
  float peaks_ratio;
  int32_t post_filter;  // 0 none, 1 Gauss, 2 bilateral
};

int ref_remove_peaks(float* disp, int32_t* segid, int w, int h, int threshold) {
  memset(segid, 0, sizeof(int32_t) * (size_t)w * h);
  return RemovePeaks(disp, segid, w, h, threshold);
}

void ref_zoom_half(const uint8_t* src, uint8_t* dst, int w, int h) { Zoom(src, dst, w, h, 2, 2); }

int ref_init_next_level(float* cur, int16_t* next, int width, int height) {
  return ComputeInitDispInNextLevel(cur, next, width, height);
}

int ref_hardware_threads_peaks(void) {
  // the strip count StereoCudaImpl::Init derives (StereoCudaImpl.cpp:234)
  return (int)(std::thread::hardware_concurrency() * 3 / 4);
}

static const char* g_msg = "";
const char* ref_last_message(void) { return g_msg; }

static bool padding_ok(size_t pitch, size_t row_bytes, size_t extra) { return pitch >= row_bytes + extra; }

static void copy_pitched_volume(const cudaPitchedPtr& p, int W, int H, int D, uint8_t* out) {
  // cudaMalloc3D layout of the reference: (pitch, ceil(W/ppp), H), ppp = pitch / D pixels per pitch row
  const int ppp = (int)(p.pitch / D);
  const size_t slice = p.pitch * p.ysize;
  std::vector<uint8_t> host(slice * H);
  cudaMemcpy(host.data(), p.ptr, host.size(), cudaMemcpyDeviceToHost);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const uint8_t* src = host.data() + y * slice + (size_t)(x / ppp) * p.pitch + (size_t)(x % ppp) * D;
      memcpy(out + ((size_t)y * W + x) * D, src, D);
    }
}

static void clear_pitched_volume(const cudaPitchedPtr& p, int H) { cudaMemset(p.ptr, 0, p.pitch * p.ysize * H); }

static CuSGMOption make_option(const ref_case_t* c, bool lr, bool median, bool peaks, int morph, int pf) {
  CuSGMOption o;
  o.p1 = c->p1;
  o.p2_init = c->p2;
  o.p2_max = 64;
  o.cs_type = c->cs_type ? CuSGMOption::CS_9x7 : CuSGMOption::CS_5x5;
  o.num_paths = 4;
  o.do_median_filter = median;
  o.do_lr_check = lr;
  o.lr_threshold = c->lr_threshold;
  o.unique_threshold = c->uniqueness;
  o.using_constant_p2 = true;
  o.do_remove_peaks = peaks;
  o.peaks_ratio_threshold = c->peaks_ratio;
  o.post_filter_type = pf == 1 ? CuSGMOption::PF_GAUSS : (pf == 2 ? CuSGMOption::PF_BILATERAL : CuSGMOption::PF_NONE);
  o.morphology_type = morph == 1   ? CuSGMOption::MP_EROSION
                      : morph == 2 ? CuSGMOption::MP_DILATION
                      : morph == 3 ? CuSGMOption::MP_OPEN
                      : morph == 4 ? CuSGMOption::MP_CLOSE
                                   : CuSGMOption::MP_NONE;
  return o;
}

static int check_case(const ref_case_t* c, bool with_init) {
  if (c->width < 16 || c->height < 16) { g_msg = "size too small"; return -1; }
  if (!(c->disp_range == 64 || (c->disp_range == 32 && with_init))) {
    g_msg = "only D=64, or D=32 with initial disparities, are run (other widths index shared memory out of range)";
    return -1;
  }
  if (with_init && c->min_disp > 0) { g_msg = "initial disparities need min_disp <= 0"; return -1; }
  return 0;
}

// Stage dumps of one case. Any output pointer may be NULL.
//   run A (LR, median, peaks off): census_l/census_r, cost_lr, paths_lr, wta_l
//   run B (LR on, median off):     cost_rl, paths_rl, lr_l (left after LR), lr_r (right after marks)
//   run C (the case's options):    disp_l, disp_r
int ref_match_dump(const ref_case_t* c, const uint8_t* left, const uint8_t* right, const int16_t* init,
                   uint64_t* census_l, uint64_t* census_r, uint8_t* cost_lr, uint8_t* paths_lr, float* wta_l,
                   uint8_t* cost_rl, uint8_t* paths_rl, float* lr_l, float* lr_r, float* disp_l, float* disp_r) {
  if (check_case(c, init != nullptr)) return -1;
  const int W = c->width, H = c->height, D = c->disp_range;
  std::vector<uint8_t> L(left, left + (size_t)W * H), R(right, right + (size_t)W * H);
  std::vector<int16_t> I;
  if (init) I.assign(init, init + (size_t)W * H);
  std::vector<float> tmp_l((size_t)W * H), tmp_r((size_t)W * H);
  for (int run = 0; run < 3; ++run) {
    const bool lr = run == 0 ? false : (run == 1 ? true : c->do_lr_check != 0);
    const bool median = run == 2 ? c->do_median != 0 : false;
    const bool peaks = run == 2 ? c->do_remove_peaks != 0 : false;
    const int morph = run == 2 ? c->morphology : 0;
    const int pf = run == 2 ? c->post_filter : 0;
    StereoCudaImpl impl;
    if (!impl.Init(W, H, c->min_disp, D, make_option(c, lr, median, peaks, morph, pf), false)) {
      g_msg = "reference Init failed";
      return -2;
    }
    const size_t dp = impl.aggregator_->dp_psize_;
    const size_t wta_extra = 4 * sizeof(float);  // up to 3 floats written past a row, 1 read
    if (!padding_ok(dp, (size_t)W * sizeof(float), wta_extra) ||
        (init && !padding_ok(impl.idp_psize_, (size_t)W * sizeof(int16_t), 3 * sizeof(int16_t)))) {
      g_msg = "pitch padding too small for the reference's row overrun";
      impl.Release();
      return -3;
    }
    // known contents for everything the reference leaves unwritten
    clear_pitched_volume(*impl.computor_->cost_, H);
    for (int k = 0; k < 4; ++k) clear_pitched_volume(impl.aggregator_->cost_aggr_dir_[k], H);
    cudaMemset(impl.aggregator_->disp_map_, 0, dp * H);
    cudaMemset(impl.aggregator_->disp_map_r_, 0, dp * H);
    cudaDeviceSynchronize();
    const bool ok = impl.Match(L.data(), R.data(), tmp_l.data(), tmp_r.data(), init ? I.data() : nullptr);
    if (cudaDeviceSynchronize() != cudaSuccess || !ok) {
      g_msg = "reference Match failed";
      impl.Release();
      return -4;
    }
    if (run == 0) {
      const size_t cs = impl.computor_->cs_psize_;
      const int bytes = c->cs_type ? 8 : 4;
      std::vector<uint8_t> buf(cs * H);
      for (int view = 0; view < 2; ++view) {
        uint64_t* dst = view == 0 ? census_l : census_r;
        if (!dst) continue;
        cudaMemcpy(buf.data(), view == 0 ? impl.computor_->census_left_ : impl.computor_->census_right_, buf.size(),
                   cudaMemcpyDeviceToHost);
        for (int y = 0; y < H; ++y)
          for (int x = 0; x < W; ++x) {
            uint64_t v = 0;
            memcpy(&v, buf.data() + y * cs + (size_t)x * bytes, bytes);
            dst[(size_t)y * W + x] = v;
          }
      }
      if (cost_lr) copy_pitched_volume(*impl.computor_->cost_, W, H, D, cost_lr);
      if (paths_lr)
        for (int k = 0; k < 4; ++k)
          copy_pitched_volume(impl.aggregator_->cost_aggr_dir_[k], W, H, D, paths_lr + (size_t)k * W * H * D);
      if (wta_l) memcpy(wta_l, tmp_l.data(), sizeof(float) * W * H);
    } else if (run == 1) {
      if (cost_rl) copy_pitched_volume(*impl.computor_->cost_, W, H, D, cost_rl);
      if (paths_rl)
        for (int k = 0; k < 4; ++k)
          copy_pitched_volume(impl.aggregator_->cost_aggr_dir_[k], W, H, D, paths_rl + (size_t)k * W * H * D);
      if (lr_l) memcpy(lr_l, tmp_l.data(), sizeof(float) * W * H);
      if (lr_r) memcpy(lr_r, tmp_r.data(), sizeof(float) * W * H);
    } else {
      if (disp_l) memcpy(disp_l, tmp_l.data(), sizeof(float) * W * H);
      if (disp_r) memcpy(disp_r, tmp_r.data(), sizeof(float) * W * H);
    }
    impl.Release();
  }
  return 0;
}

// Stage dumps of a match with regions of interest (roi = {x, y, w, h}; roi_r may be NULL):
//   run A (LR, median, peaks off; left ROI):  cost_lr, paths_lr (4 volumes), wta_l
//   run B (LR on, median off; both ROIs):     cost_rl, paths_rl (the right view's cost and paths)
// Runs only rectangles inside the image whose width is a multiple of 4: the reference's WTA launch
// covers ceil(w/4)*4 columns and floor(h/2)*2 rows from (x, y) (cusgm_ca.cu:4139-4165) and writes
// without a column bound, and its scans start at x / y and run to x+w / y+h (:1478-1598); inside
// these limits every access of the plain D = 64 path stays in its allocation.
int ref_match_roi_dump(const ref_case_t* c, const uint8_t* left, const uint8_t* right, const int32_t* roi_l,
                       const int32_t* roi_r, uint8_t* cost_lr, uint8_t* paths_lr, float* wta_l, uint8_t* cost_rl,
                       uint8_t* paths_rl) {
  if (check_case(c, false)) return -1;
  const int W = c->width, H = c->height, D = c->disp_range;
  for (const int32_t* r : {roi_l, roi_r}) {
    if (!r) continue;
    if (r[0] < 0 || r[1] < 0 || r[2] <= 0 || r[3] <= 0 || r[0] + r[2] > W || r[1] + r[3] > H || r[2] % 4) {
      g_msg = "ROI outside the image or its width not a multiple of 4";
      return -1;
    }
  }
  if (!roi_l) { g_msg = "a left ROI is required"; return -1; }
  StereoROI_T rl{roi_l[0], roi_l[1], roi_l[2], roi_l[3]};
  StereoROI_T rr{};
  if (roi_r) rr = StereoROI_T{roi_r[0], roi_r[1], roi_r[2], roi_r[3]};
  std::vector<uint8_t> L(left, left + (size_t)W * H), R(right, right + (size_t)W * H);
  std::vector<float> tmp_l((size_t)W * H), tmp_r((size_t)W * H);
  for (int run = 0; run < 2; ++run) {
    StereoCudaImpl impl;
    if (!impl.Init(W, H, c->min_disp, D, make_option(c, run == 1, false, false, 0, 0), false)) {
      g_msg = "reference Init failed";
      return -2;
    }
    const size_t dp = impl.aggregator_->dp_psize_;
    if (!padding_ok(dp, (size_t)W * sizeof(float), 4 * sizeof(float))) {
      g_msg = "pitch padding too small for the reference's row overrun";
      impl.Release();
      return -3;
    }
    clear_pitched_volume(*impl.computor_->cost_, H);
    for (int k = 0; k < 4; ++k) clear_pitched_volume(impl.aggregator_->cost_aggr_dir_[k], H);
    cudaMemset(impl.aggregator_->disp_map_, 0, dp * H);
    cudaMemset(impl.aggregator_->disp_map_r_, 0, dp * H);
    cudaDeviceSynchronize();
    const bool ok = impl.Match(L.data(), R.data(), tmp_l.data(), tmp_r.data(), nullptr, &rl, roi_r ? &rr : nullptr);
    if (cudaDeviceSynchronize() != cudaSuccess || !ok) {
      g_msg = "reference Match failed";
      impl.Release();
      return -4;
    }
    uint8_t* cost = run == 0 ? cost_lr : cost_rl;
    uint8_t* paths = run == 0 ? paths_lr : paths_rl;
    if (cost) copy_pitched_volume(*impl.computor_->cost_, W, H, D, cost);
    if (paths)
      for (int k = 0; k < 4; ++k)
        copy_pitched_volume(impl.aggregator_->cost_aggr_dir_[k], W, H, D, paths + (size_t)k * W * H * D);
    if (run == 0 && wta_l) memcpy(wta_l, tmp_l.data(), sizeof(float) * W * H);
    impl.Release();
  }
  return 0;
}

// StereoCudaImpl::Init2 / Match2 (StereoCudaImpl.cpp:263-278, :548-583): depth of the left view
// with the case's options. cam = {x0_left, y0_left, x0_right, y0_right, focus, baseline}.
// Same case restrictions and row-padding check as ref_match_dump.
int ref_match2(const ref_case_t* c, const double* cam, const uint8_t* left, const uint8_t* right, float* depth) {
  if (check_case(c, false)) return -1;
  const int W = c->width, H = c->height;
  std::vector<uint8_t> L(left, left + (size_t)W * H), R(right, right + (size_t)W * H);
  CamParam_T p{};
  p.x0_left = cam[0];
  p.y0_left = cam[1];
  p.x0_right = cam[2];
  p.y0_right = cam[3];
  p.focus = cam[4];
  p.baseline = cam[5];
  StereoCudaImpl impl;
  const CuSGMOption o =
      make_option(c, c->do_lr_check != 0, c->do_median != 0, c->do_remove_peaks != 0, c->morphology, c->post_filter);
  if (!impl.Init2(W, H, c->min_disp, c->disp_range, o, p, false)) {
    g_msg = "reference Init2 failed";
    return -2;
  }
  if (!padding_ok(impl.aggregator_->dp_psize_, (size_t)W * sizeof(float), 4 * sizeof(float))) {
    g_msg = "pitch padding too small for the reference's row overrun";
    impl.Release();
    return -3;
  }
  const bool ok = impl.Match2(L.data(), R.data(), depth);
  if (cudaDeviceSynchronize() != cudaSuccess || !ok) {
    g_msg = "reference Match2 failed";
    impl.Release();
    return -4;
  }
  impl.Release();
  return 0;
}

// FasterStereoCuda::Init2 / Match2 through the reference's public API (FasterStereoCuda.cpp:297-406,
// :531-635): depth of the finest level for a depth range. epi = {x0_left, y0_left, x0_right,
// y0_right, baseline, focus}. Never released, like ref_pyr_match. Only ranges whose levels all
// run D = 32 or 64 are safe to run (the D = 128 / 256 kernels index shared memory out of range):
// the caller checks the coarsest range first.
int ref_pyr_match2(int width, int height, float min_depth, float max_depth, int layers, int lr, int peaks,
                   const double* epi, const uint8_t* left, const uint8_t* right, float* depth) {
  FasterStereoCuda& s = *new FasterStereoCuda;  // leaked on purpose, see ref_pyr_match
  FasterStereoCuda::StereoOption2 o;
  o.width = width;
  o.height = height;
  o.min_depth = min_depth;
  o.max_depth = max_depth;
  o.num_layers = layers;
  o.do_lr_check = lr != 0;
  o.do_rm_peaks = peaks != 0;
  o.do_smooth = false;
  o.epi.x0_left = epi[0];
  o.epi.y0_left = epi[1];
  o.epi.x0_right = epi[2];
  o.epi.y0_right = epi[3];
  o.epi.baseline = epi[4];
  o.epi.focus = epi[5];
  if (!s.Init2(o)) { g_msg = "FasterStereoCuda::Init2 failed"; return -2; }
  const bool ok = s.Match2(left, right, depth);
  if (!ok || cudaDeviceSynchronize() != cudaSuccess) { g_msg = "FasterStereoCuda::Match2 failed"; return -4; }
  return 0;
}

// FasterStereoCuda::Match through the reference's public API (per-level options as the
// reference hard-codes them). Returns 0 on success.
// The matcher is deliberately never released: HierSgmCudaImpl::Release (FasterStereoCuda.cpp:
// 641-679) frees each level's pinned disparity buffer before releasing that level's StereoCuda,
// whose teardown (ThreadBase::WaitForTerminate, common/thread.h) wakes the small-region worker
// threads once more on the freed buffer -- a host-side use-after-free that crashed the process.
int ref_pyr_match(int width, int height, int min_disp, int max_disp, int layers, int lr, int peaks,
                  const uint8_t* left, const uint8_t* right, float* disp) {
  FasterStereoCuda& s = *new FasterStereoCuda;  // leaked on purpose, see above
  FasterStereoCuda::StereoOption1 o;
  o.width = width;
  o.height = height;
  o.min_disp = min_disp;
  o.max_disp = max_disp;
  o.num_layers = layers;
  o.do_lr_check = lr != 0;
  o.do_rm_peaks = peaks != 0;
  o.do_smooth = false;
  if (!s.Init(o)) { g_msg = "FasterStereoCuda::Init failed"; return -2; }
  const bool ok = s.Match(left, right, disp);
  if (!ok || cudaDeviceSynchronize() != cudaSuccess) { g_msg = "FasterStereoCuda::Match failed"; return -4; }
  return 0;
}

// Wall time of n StereoCuda::Match calls on one pair (host buffers in and out), in ms per call.
double ref_time_match(const ref_case_t* c, const uint8_t* left, const uint8_t* right, int warmup, int n) {
  if (check_case(c, false)) return -1.0;
  StereoCudaImpl impl;
  if (!impl.Init(c->width, c->height, c->min_disp, c->disp_range,
                 make_option(c, c->do_lr_check != 0, c->do_median != 0, c->do_remove_peaks != 0, c->morphology,
                             c->post_filter),
                 false))
    return -2.0;
  std::vector<uint8_t> L(left, left + (size_t)c->width * c->height), R(right, right + (size_t)c->width * c->height);
  std::vector<float> d((size_t)c->width * c->height);
  for (int i = 0; i < warmup; ++i) impl.Match(L.data(), R.data(), d.data());
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < n; ++i) impl.Match(L.data(), R.data(), d.data());
  cudaDeviceSynchronize();
  const auto t1 = std::chrono::steady_clock::now();
  impl.Release();
  return std::chrono::duration<double, std::milli>(t1 - t0).count() / n;
}

// The pyramid of FasterStereoCuda::Match (HierSgmCudaImpl::Init :201-295 and Match :408-529)
// driven level by level with the reference's own pieces -- SetSgmParameters, StereoCudaImpl,
// Zoom, ComputeInitDispInNextLevel -- so that every level's output can be dumped.
// disp_levels receives the levels' disparity maps concatenated (coarsest first), init_levels the
// initial disparities handed to the finer levels (next-coarsest first).
int ref_pyr_levels(int width, int height, int min_disp, int max_disp, int layers, int lr, int peaks,
                   const uint8_t* left, const uint8_t* right, float* disp_levels, int16_t* init_levels) {
  const int L = layers < 1 ? 1 : layers;
  std::vector<int> w(L), h(L);
  std::vector<std::vector<uint8_t>> bl(L), br(L);
  std::vector<std::vector<float>> disp(L);
  std::vector<std::vector<int16_t>> init(L);
  std::vector<StereoCudaImpl*> st(L, nullptr);
  for (int i = 0; i < L; ++i) {
    const int scale = 1 << i;
    w[i] = width / scale;
    h[i] = height / scale;
    bl[i].resize((size_t)w[i] * h[i]);
    br[i].resize((size_t)w[i] * h[i]);
    disp[i].resize((size_t)w[i] * h[i]);
    init[i].resize((size_t)w[i] * h[i]);
    CuSGMOption param;
    SetSgmParameters(lr != 0, peaks != 0, false, param, i, L);
    if (!param.using_constant_p2) { param.p1 = 10; param.p2_init = 150; }
    int dmin = min_disp / scale, dmax = max_disp / scale, range = 32;
    if (i == L - 1) {
      range = dmax - dmin;
      int k = 6;
      while ((1 << k) < range) k++;
      range = 1 << k;
      if (range > 2 * width) range /= 2;
      if (dmin >= width) { dmin = width - range; if (dmin < -width) dmin = -width; }
    } else {
      dmin = 0;
    }
    st[i] = new StereoCudaImpl;  // released below only after its output buffer is copied
    if (!st[i]->Init(w[i], h[i], dmin, range, param, false)) { g_msg = "level Init failed"; return -2; }
  }
  memcpy(bl[0].data(), left, (size_t)w[0] * h[0]);
  memcpy(br[0].data(), right, (size_t)w[0] * h[0]);
  for (int i = 1; i < L; ++i) {
    Zoom(bl[i - 1].data(), bl[i].data(), w[i - 1], h[i - 1], 2, 2);
    Zoom(br[i - 1].data(), br[i].data(), w[i - 1], h[i - 1], 2, 2);
  }
  size_t doff = 0, ioff = 0;
  for (int n = L - 1; n >= 0; --n) {
    if (!st[n]->Match(bl[n].data(), br[n].data(), disp[n].data(), nullptr, n < L - 1 ? init[n].data() : nullptr)) {
      g_msg = "level Match failed";
      return -4;
    }
    memcpy(disp_levels + doff, disp[n].data(), sizeof(float) * w[n] * h[n]);
    doff += (size_t)w[n] * h[n];
    if (n > 0) {
      // one spare INVALID after the coarse map for the reference's read past its end (odd widths)
      std::vector<float> cur(disp[n]);
      cur.push_back(INVALID_VALUE);
      ComputeInitDispInNextLevel(cur.data(), init[n - 1].data(), w[n - 1], h[n - 1]);
      memcpy(init_levels + ioff, init[n - 1].data(), sizeof(int16_t) * w[n - 1] * h[n - 1]);
      ioff += (size_t)w[n - 1] * h[n - 1];
    }
  }
  cudaDeviceSynchronize();
  // the levels' small-region workers still point at disp[]: release them while it is alive
  for (int i = 0; i < L; ++i) { st[i]->Release(); delete st[i]; }
  return 0;
}

// Wall time of n FasterStereoCuda::Match calls (host buffers in and out), ms per call.
// The matcher is leaked for the reason given at ref_pyr_match.
double ref_time_pyr(int width, int height, int min_disp, int max_disp, int layers, int lr, int peaks,
                    const uint8_t* left, const uint8_t* right, int warmup, int n) {
  FasterStereoCuda& s = *new FasterStereoCuda;
  FasterStereoCuda::StereoOption1 o;
  o.width = width;
  o.height = height;
  o.min_disp = min_disp;
  o.max_disp = max_disp;
  o.num_layers = layers;
  o.do_lr_check = lr != 0;
  o.do_rm_peaks = peaks != 0;
  o.do_smooth = false;
  if (!s.Init(o)) return -2.0;
  std::vector<float> d((size_t)width * height);
  for (int i = 0; i < warmup; ++i) s.Match(left, right, d.data());
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < n; ++i) s.Match(left, right, d.data());
  cudaDeviceSynchronize();
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double, std::milli>(t1 - t0).count() / n;
}

}  // extern "C"

// Runs body(k) for k = 0 .. threads-1, one host thread each; every thread first runs its warm-up
// part, then all start the timed part together. Returns the wall time of the timed part in s.
template <typename Warm, typename Body>
static double timed_threads(int threads, Warm warm, Body body) {
  std::atomic<int> ready{0};
  std::atomic<bool> go{false};
  std::vector<std::thread> pool;
  for (int k = 0; k < threads; ++k)
    pool.emplace_back([&, k] {
      warm(k);
      ready.fetch_add(1);
      while (!go.load()) std::this_thread::yield();
      body(k);
    });
  while (ready.load() < threads) std::this_thread::yield();
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  go.store(true);
  for (auto& t : pool) t.join();
  cudaDeviceSynchronize();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

extern "C" {

// Pairs per second of `threads` host threads, each with its own StereoCudaImpl, matching the pair
// n times through StereoCuda::Match (host buffers in and out); < 0 on failure.
double ref_throughput_match(const ref_case_t* c, const uint8_t* left, const uint8_t* right, int warmup, int n,
                            int threads) {
  if (check_case(c, false) || threads < 1) return -1.0;
  const size_t N = (size_t)c->width * c->height;
  std::vector<StereoCudaImpl*> impl(threads, nullptr);
  const CuSGMOption o =
      make_option(c, c->do_lr_check != 0, c->do_median != 0, c->do_remove_peaks != 0, c->morphology, c->post_filter);
  for (int k = 0; k < threads; ++k) {
    impl[k] = new StereoCudaImpl;
    if (!impl[k]->Init(c->width, c->height, c->min_disp, c->disp_range, o, false)) {
      for (int j = 0; j <= k; ++j) { impl[j]->Release(); delete impl[j]; }
      return -2.0;
    }
  }
  std::vector<std::vector<uint8_t>> L(threads, std::vector<uint8_t>(left, left + N)),
      R(threads, std::vector<uint8_t>(right, right + N));
  std::vector<std::vector<float>> d(threads, std::vector<float>(N));
  const double s = timed_threads(
      threads, [&](int k) { for (int i = 0; i < warmup; ++i) impl[k]->Match(L[k].data(), R[k].data(), d[k].data()); },
      [&](int k) { for (int i = 0; i < n; ++i) impl[k]->Match(L[k].data(), R[k].data(), d[k].data()); });
  for (int k = 0; k < threads; ++k) { impl[k]->Release(); delete impl[k]; }
  return s > 0 ? (double)threads * n / s : -3.0;
}

// The same for FasterStereoCuda::Match (the reference's per-level parameters); the matchers are
// leaked for the reason given at ref_pyr_match.
double ref_throughput_pyr(int width, int height, int min_disp, int max_disp, int layers, int lr, int peaks,
                          const uint8_t* left, const uint8_t* right, int warmup, int n, int threads) {
  if (threads < 1) return -1.0;
  std::vector<FasterStereoCuda*> m(threads, nullptr);
  FasterStereoCuda::StereoOption1 o;
  o.width = width;
  o.height = height;
  o.min_disp = min_disp;
  o.max_disp = max_disp;
  o.num_layers = layers;
  o.do_lr_check = lr != 0;
  o.do_rm_peaks = peaks != 0;
  o.do_smooth = false;
  for (int k = 0; k < threads; ++k) {
    m[k] = new FasterStereoCuda;
    if (!m[k]->Init(o)) return -2.0;
  }
  const size_t N = (size_t)width * height;
  std::vector<std::vector<float>> d(threads, std::vector<float>(N));
  const double s = timed_threads(
      threads, [&](int k) { for (int i = 0; i < warmup; ++i) m[k]->Match(left, right, d[k].data()); },
      [&](int k) { for (int i = 0; i < n; ++i) m[k]->Match(left, right, d[k].data()); });
  return s > 0 ? (double)threads * n / s : -3.0;
}

}  // extern "C"
