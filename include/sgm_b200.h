/*
 * sgm_b200.h -- C ABI of the B200 semi-global-matching stereo engine.
 *
 * Drop-in boundary for the stereo path of ethan-li-coding/FasterStereoCuda.
 * Every entry point below names the reference interface it replaces
 * (paths are relative to the reference project). Plain pointers and sizes
 * only; no C++ or torch types cross this boundary.
 *
 * Status codes: 0 = success, negative = failure (see sgm_status_t).
 * Threading: one handle is one matcher; calls on a handle must not overlap.
 * Invalid disparity value: -999999.0f. Invalid initial disparity: -32768.
 */
#ifndef SGM_B200_H_
#define SGM_B200_H_

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#if defined(_WIN32)
#define SGM_API __declspec(dllexport)
#else
#define SGM_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SGM_OK = 0,
  SGM_ERR_ARG = -1,         /* bad argument (size, range, null pointer, option combination) */
  SGM_ERR_STATE = -2,       /* handle not initialised / already released */
  SGM_ERR_CUDA = -3,        /* CUDA runtime error (message in sgm_last_error) */
  SGM_ERR_UNSUPPORTED = -4, /* valid in the reference API but not supported by this engine */
  SGM_ERR_NOMEM = -5        /* device or host allocation failed */
} sgm_status_t;

/* Same member order, types and layout as the reference's CuSGMOption
 * (SgmStereoCuda/sgm_types.h:21-65), so a CuSGMOption* may be passed directly. */
typedef struct sgm_option_s {
  int32_t p1;
  int32_t p2_init;
  int32_t p2_max;
  int32_t cs_type;        /* 0 = census 5x5, 1 = census 9x7 */
  int32_t num_paths;
  bool do_median_filter;
  bool do_lr_check;
  float lr_threshold;
  float unique_threshold;
  bool using_constant_p2;
  bool do_remove_peaks;
  float peaks_ratio_threshold;
  int32_t post_filter_type; /* 0 = none, 1 = Gauss, 2 = bilateral (cusgm_df.cu:94-195) */
  int32_t morphology_type;  /* 0 = none, 1 = erosion, 2 = dilation, 3 = open, 4 = close */
} sgm_option_t;

/* Same layout as StereoROI_T (SgmStereoCuda/sgm_types.h:89-92). */
typedef struct sgm_roi_s {
  int32_t x, y, w, h;
} sgm_roi_t;

/* Choices the reference leaves to thread scheduling or to its compiler; fixed here. */
typedef struct sgm_ext_options_s {
  int32_t tie_rule;       /* WTA tie break, plain path: 0 lowest d, 1 highest d, 2 highest lane, 3 lowest lane,
                             4 (default) the reference build's behaviour measured on a B200 */
  int32_t init_tie_rule;  /* the same at initial-disparity (pyramid) levels (default 4) */
  int32_t peaks_strips;   /* strips of small-region removal; <= 0: hardware threads * 3 / 4 */
  int32_t peaks_abs_mode; /* region test: 0 |(int)(a-b)| <= 1 (g++ build), 1 |a-b| <= 1.0f (MSVC build) */
  int32_t p2_div0;        /* P2 / 0 at initial-disparity levels */
} sgm_ext_options_t;

/* Same layout as CamParam_T (SgmStereoCuda/sgm_types.h:70-84). */
typedef struct sgm_camera_s {
  double x0_left, y0_left;
  double x0_right, y0_right;
  double focus;
  double baseline;
} sgm_camera_t;

typedef struct sgm_engine* sgm_handle_t;

/* StereoCuda::StereoCuda() -- SgmStereoCuda/StereoCuda.cpp:4-7 */
SGM_API int sgm_create(sgm_handle_t* out);
/* StereoCuda::~StereoCuda() -- SgmStereoCuda/StereoCuda.cpp:9-16 */
SGM_API int sgm_destroy(sgm_handle_t h);
/* StereoCuda::Init -- SgmStereoCuda/StereoCuda.h:31, StereoCudaImpl.cpp:128-261.
 * Allocates every device buffer for (width, height, min_disparity, disp_range). */
SGM_API int sgm_init(sgm_handle_t h, int32_t width, int32_t height, int32_t min_disparity, int32_t disp_range,
                     const sgm_option_t* option, int32_t print_log);
/* No counterpart in the reference: sets the rules in sgm_ext_options_t (before or after init). */
SGM_API int sgm_set_ext_options(sgm_handle_t h, const sgm_ext_options_t* ext);
SGM_API int sgm_get_ext_options(sgm_handle_t h, sgm_ext_options_t* ext);

/* No counterpart in the reference. Kernel variants and launch shapes; results do not depend on
 * them (every variant is bit-exact), only speed does. 0 everywhere = defaults; a matcher left at
 * the defaults runs, in the synchronous host API (sgm_match, sgm_match2, sgm_pyr_match,
 * sgm_pyr_match2), row_kernel = col_kernel = 4 while at most eight such calls are in flight in
 * the process (a few callers matching one frame at a time) and the defaults below otherwise.
 * While at most eight calls are in flight they also wait for their results by polling; beyond
 * that they sleep on a blocking-sync event. */
typedef struct sgm_tuning_t {
  int32_t row_kernel;   /* horizontal scans: 1 = whole census rows in shared memory,
                           2 = census window and 32-pixel cost chunks in shared memory,
                           3 = cost-volume kernel + row_lanes lanes per scanline (u16x2 SIMD),
                           4 = one warp per scanline with cost chunks staged by bulk async copies
                           and 32-bit path costs: the shortest step chain, for one pair in flight
                           (D <= 128 and tie rule 0, 1 or 4 at plain levels; any tie rule at the
                           32-disparity pyramid levels; elsewhere the default);
                           0 (default) = 3 where it is exact (see below), else 2 */
  int32_t rows_per_cta; /* scanlines per CTA of the horizontal scans: 0 (default), 1, 2 or 4 */
  int32_t col_kernel;   /* vertical scans + WTA: 1 = one warp per column, plain loads, 2 = the same with
                           an 8-row prefetch ring, 3 = col_lanes lanes per column (u16x2 SIMD, WTA in
                           the lanes), 4 = as row_kernel 4 (chunks of 32 rows as tensor-map boxes;
                           at the 32-disparity levels both directions beside the row scans, then a
                           WTA launch: the first such match allocates one more path volume, so it
                           must not run inside a stream capture); 0 (default) = 3
                           where it is exact, else 1. Variant 3 is exact for D <= 128,
                           P1 <= P2 <= 16383 and tie rule 0 or 4 (else 2 / 1 run) */
  int32_t cols_per_cta; /* columns (one warp each) per CTA of the vertical scans: 0 (default) .. 8 */
  int32_t bt_smem;      /* 1: keep bottom-to-top path costs in shared memory when they fit */
  int32_t row_lanes;    /* variant 3: lanes per scanline of the horizontal scans, 1/2/4/8 (0: 8) */
  int32_t col_lanes;    /* variant 3: lanes per column of the vertical scans, 1/2/4/8 (0: 4);
                           D = 128 takes 2 or 4 (default 4) */
} sgm_tuning_t;
SGM_API int sgm_set_tuning(sgm_handle_t h, const sgm_tuning_t* t);
SGM_API int sgm_get_tuning(sgm_handle_t h, sgm_tuning_t* t);
/* StereoCuda::Match -- SgmStereoCuda/StereoCuda.h:44, StereoCudaImpl.cpp:507-546.
 * Host buffers of width*height elements. disp_right, init_disp_left, roi_* may be NULL.
 * Returns after the disparity has been copied back (synchronous, like the reference).
 * roi_left / roi_right (cusgm_cc.cu:478-488, cusgm_ca.cu:3991-3999): a view's rectangle, inside the
 * image, matched as a sub-image whose paths start at its edges (columns from max(x, min_disparity));
 * the WTA covers floor(h/2)*2 of its rows, everything outside is INVALID, small-region removal runs
 * in strips of the left rectangle's rows. roi_right is used with the LR check only. Plain levels
 * with disp_range <= 128, P1 <= P2 <= 16383 and tie rule 0 or 4, else SGM_ERR_UNSUPPORTED.
 * With print_log set at init, prints the time of every stage (CUDA events). */
SGM_API int sgm_match(sgm_handle_t h, const uint8_t* img_left, const uint8_t* img_right, float* disp_left,
                      float* disp_right, const int16_t* init_disp_left, const sgm_roi_t* roi_left,
                      const sgm_roi_t* roi_right);
/* No counterpart in the reference: the same match on device-resident buffers
 * (dense width*height arrays), enqueued on `stream` (a cudaStream_t, NULL = the
 * handle's own stream) without synchronising. */
SGM_API int sgm_match_device(sgm_handle_t h, const uint8_t* d_left, const uint8_t* d_right, float* d_disp_left,
                             float* d_disp_right, const int16_t* d_init_disp_left, void* stream);
/* StereoCuda::Init2 -- SgmStereoCuda/StereoCuda.h:57, StereoCudaImpl.cpp:263-278: Init plus the
 * camera used by sgm_match2. */
SGM_API int sgm_init2(sgm_handle_t h, int32_t width, int32_t height, int32_t min_disparity, int32_t disp_range,
                      const sgm_option_t* option, const sgm_camera_t* camera, int32_t print_log);
/* StereoCuda::Match2 -- SgmStereoCuda/StereoCuda.h:69, StereoCudaImpl.cpp:548-583: match, then
 * depth = baseline*focus / (d + x0_right - x0_left) in double, INVALID kept (cusgm_util.cu:7-34).
 * The disparity is the final map, except with exactly one of post filter / morphology and no
 * small-region removal: then the map before that step (the reference's aggregator buffer). */
SGM_API int sgm_match2(sgm_handle_t h, const uint8_t* img_left, const uint8_t* img_right, float* depth_left,
                       const int16_t* init_disp_left, const sgm_roi_t* roi_left, const sgm_roi_t* roi_right);
/* StereoCuda::Release -- SgmStereoCuda/StereoCuda.h:75, StereoCudaImpl.cpp:281-332 */
SGM_API int sgm_release(sgm_handle_t h);
/* StereoCuda::SetMinDisparity / GetDispartyRange -- SgmStereoCuda/StereoCuda.h:71-72.
 * A minimum disparity at or past the width is refused (SGM_ERR_ARG, the previous value kept). */
SGM_API int sgm_set_min_disparity(sgm_handle_t h, int32_t min_disparity);
SGM_API int32_t sgm_get_disparity_range(sgm_handle_t h);
/* StereoCuda::GetRoiFromDispMap -- SgmStereoCuda/StereoCudaImpl.cpp:585-628 */
SGM_API void sgm_roi_from_disp_map(const float* disp, int32_t width, int32_t height, sgm_roi_t* roi);
/* StereoCuda::get_invad_float / get_invad_short / get_level_range -- StereoCuda.h:87-91 */
SGM_API float sgm_invalid_float(void);
SGM_API int16_t sgm_invalid_short(void);
SGM_API int16_t sgm_level_range(void);
/* StereoCuda::MallocPageLockedPtr / FreePageLockedPtr -- StereoCuda.h:94-97 */
SGM_API int sgm_malloc_page_locked(void** ptr, size_t size);
SGM_API int sgm_free_page_locked(void* ptr);
/* No counterpart in the reference: message of the last failure on h (NULL h: process-wide). */
SGM_API const char* sgm_last_error(sgm_handle_t h);
/* No counterpart in the reference: number of kernel launches issued by the last match on h. */
SGM_API int64_t sgm_kernel_launches(sgm_handle_t h);

/* No counterpart in the reference: copies an internal stage buffer of the last match to host
 * memory, for stage-by-stage parity tests. `which`: 0/1 census left/right (uint64 per pixel,
 * 5x5 zero-extended), 2 cost, 3 left->right, 4 right->left, 5 bottom->top path costs
 * (uint8 [H][W][D]) and 6 the WTA disparity (float [H][W]) of view `view` (0 left, 1 right).
 * `bytes` must equal the buffer size. Synchronises the handle's stream. */
SGM_API int sgm_debug_read(sgm_handle_t h, int32_t which, int32_t view, void* dst, size_t bytes);

/* No counterpart in the reference: fault injection for tests of the out-of-memory paths. After
 * sgm_debug_fail_device_alloc(n) the engine's (n+1)-th device allocation from then on fails as
 * cudaMalloc does when the device is out of memory (once; n < 0 disarms). The reference's Init
 * returns false when an allocation fails (SgmStereoCuda/StereoCudaImpl.cpp:138-207); sgm_init,
 * sgm_pyr_init, sgm_init2, sgm_pyr_init2, sgm_batch_init and sgm_batch_pyr_init return SGM_ERR_NOMEM
 * and free what they had allocated. sgm_debug_live_device_allocations counts the engine's device
 * allocations that are currently held (process-wide). */
SGM_API int sgm_debug_fail_device_alloc(int64_t after);
/* No counterpart in the reference: number of waits on a bulk-copy barrier that the variant-4 scan
 * kernels gave up on (each is bounded; a warp that gives up stops and leaves its outputs
 * incomplete). 0 in every correct run; -1 if it cannot be read. */
SGM_API int64_t sgm_debug_wait_timeouts(void);
/* Tests of that path: every such wait gives up after max_polls polls (<= 0: the default, 2^22),
 * and with short_copy != 0 the warp-per-scanline plain row scans expect 16 bytes more than their
 * first copy delivers, so that wait runs out (no memory is touched beyond the copies). The
 * context stays usable. sgm_debug_reset_wait_timeouts sets the counter back to 0. */
SGM_API int sgm_debug_scan_wait(int64_t max_polls, int32_t short_copy);
SGM_API int sgm_debug_reset_wait_timeouts(void);
SGM_API int64_t sgm_debug_live_device_allocations(void);

/* No counterpart in the reference: per-kernel timing with CUDA events recorded on the launching
 * stream around every launch of every handle in the process. Enabling resets the counters. While
 * it is on, matches run their kernels directly (no graph) and one after another on their stream
 * (the column pass that otherwise overlaps the row scans on a second stream waits for them), so
 * that each launch is timed alone; sgm_batch_run and sgm_batch_pyr_run likewise enqueue the
 * batch's kernels on the given stream one at a time instead of launching its graph. */
SGM_API int sgm_profile_enable(int32_t enable);
/* Writes {"kernel": {"launches": n, "ms": total}, ...} into buf; returns 0, or the size needed
 * (including the terminating NUL) when cap is too small. Synchronises on the recorded events. */
SGM_API int sgm_profile_read(char* buf, size_t cap);

/* No counterpart in the reference. Single-level matching that allocates no memory, for callers
 * that may not call cudaMalloc once they are running: real-time loops that forbid allocation after
 * start-up (an allocation can stall and synchronise the device), and plugin hosts that own the GPU
 * memory budget and hand a plugin only its input and output buffers.
 * Inputs and output are dense device arrays the caller owns (width*height uint8 images, float
 * disparity). All working memory lives in one 64 MiB array inside the library, which every GPU
 * that loads the library keeps until the process exits. The working memory of a call is
 *   2*W*H*(4 or 8, census 5x5 / 9x7) + 4*views*W*H*D + 8*W*H bytes (views = 2 with the LR check),
 * each term rounded up to 256; larger requests are rejected with SGM_ERR_ARG and a message in
 * sgm_last_error(NULL). Supported: D = 32, 64 or 128, census, penalties, uniqueness, LR check,
 * median; small-region removal, morphology, post filters and initial disparities are not
 * (SGM_ERR_UNSUPPORTED). Also refused (SGM_ERR_ARG): heights above 65535 and a minimum disparity
 * at or past the width. Results equal sgm_match_device with the default extended options.
 * Calls share the working memory: calls whose work overlaps on the GPU (two streams, two host
 * threads) race and must be serialised by the caller. The first call on each device does the
 * set-up -- it looks up the array's device address (cudaGetSymbolAddress) and loads the kernels --
 * so make it before any stream capture starts. A CUDA error left pending by earlier work makes the
 * call fail with SGM_ERR_CUDA without clearing it. Enqueued on `stream` (a cudaStream_t), not
 * synchronised. */
SGM_API int sgm_match_noalloc(const uint8_t* d_left, const uint8_t* d_right, float* d_disp_left, int32_t width,
                              int32_t height, int32_t min_disparity, int32_t disp_range, const sgm_option_t* option,
                              void* stream);

/* ---------------- batched matching (many pairs, one graph launch) ---------------- */

/* No counterpart in the reference, which matches one pair per StereoCuda::Match call. A batch
 * holds pairs of different sizes and disparity ranges (D = 32, 64 or 128) under one option set
 * (census, penalties, uniqueness, LR check, median; no small-region removal, morphology, post
 * filters or initial disparities). sgm_batch_init allocates one device arena for all pairs,
 * picks launch shapes per (D, width class) bucket by timing candidates (cached per process) and
 * captures the whole batch into one CUDA graph. Each pair's result is bit-identical to
 * sgm_match_device on that pair. */
typedef struct sgm_batch* sgm_batch_t;
typedef struct sgm_batch_pair_t {
  int32_t width, height, min_disparity, disp_range;
} sgm_batch_pair_t;
typedef struct sgm_batch_info_t {
  int32_t pairs, buckets;
  uint64_t arena_bytes;     /* device memory of the batch */
  int64_t kernels_per_run;  /* kernel launches inside one graph launch */
} sgm_batch_info_t;
typedef struct sgm_batch_bucket_t {
  int32_t disp_range, width_class, pairs;  /* width class 0: <= 640, 1: <= 1280, 2: wider */
  int32_t rows_lanes;                      /* 0: one warp per scanline; G: G lanes per scanline (u16x2) */
  int32_t rows_warps_per_cta, rows_ctas;   /* persistent row-scan kernel shape */
  int32_t cols_lanes;                      /* 0: one warp per column; G: G lanes per column (u16x2) */
  int32_t cols_warps_per_cta, cols_prefetch, cols_ctas;  /* prefetch (one warp per column): 0 plain, 4/8 ring */
} sgm_batch_bucket_t;
SGM_API int sgm_batch_create(sgm_batch_t* out);
SGM_API int sgm_batch_destroy(sgm_batch_t b);
SGM_API const char* sgm_batch_last_error(sgm_batch_t b);
/* ext may be NULL (default rules). */
SGM_API int sgm_batch_init(sgm_batch_t b, const sgm_batch_pair_t* pairs, int32_t count, const sgm_option_t* option,
                           const sgm_ext_options_t* ext);
/* Re-times every bucket's candidates (ignoring the cache) and re-captures the graph. */
SGM_API int sgm_batch_autotune(sgm_batch_t b);
/* Device buffers of pair `index` inside the arena: width*height uint8 images to fill before
 * sgm_batch_run, width*height float disparities to read after it. */
SGM_API int sgm_batch_pair_buffers(sgm_batch_t b, int32_t index, uint8_t** d_left, uint8_t** d_right,
                                   float** d_disp);
/* One graph launch matching every pair, enqueued on `stream` (NULL: the batch's own stream). */
SGM_API int sgm_batch_run(sgm_batch_t b, void* stream);
/* Host buffers (arrays of `count` pointers): copies in, runs, copies out, synchronises. */
SGM_API int sgm_batch_match(sgm_batch_t b, const uint8_t* const* left, const uint8_t* const* right,
                            float* const* disp);
SGM_API int sgm_batch_info(sgm_batch_t b, sgm_batch_info_t* info);
SGM_API int sgm_batch_bucket(sgm_batch_t b, int32_t index, sgm_batch_bucket_t* bucket);

/* ---------------- differentiable float32 SGM (training harness) ---------------- */

/* No counterpart in the reference. Float32 4-path hard-min SGM with per-pixel P1/P2 maps and a
 * soft-argmin disparity: L_p(d) = C_p(d) + min(L_q(d), L_q(d±1)+P1(p), m_q+P2(p)) - m_q,
 * S = ((L_0 + L_1) + L_2) + L_3 over the paths (top->bottom, left->right, bottom->top,
 * right->left), disp = sum_d d*softmax(-S/T). Device pointers: cost [B][H][W][D],
 * p1/p2/disp [B][H][W], sum [B][H][W][D] (S, kept for the backward pass), ckpt of
 * sgm_float_checkpoint_elems floats (path states every 8 pixels, kept for the backward pass),
 * work of sgm_float_workspace_elems floats (scratch, free after the call's work completes on
 * `stream`). D = 32 or 64; cost, sum, ckpt and work 16-byte aligned. */
SGM_API size_t sgm_float_checkpoint_elems(int32_t B, int32_t H, int32_t W, int32_t D);
SGM_API size_t sgm_float_workspace_elems(int32_t B, int32_t H, int32_t W, int32_t D);
SGM_API int sgm_float_forward(const float* cost, const float* p1, const float* p2, int32_t B, int32_t H, int32_t W,
                              int32_t D, float temperature, float* sum, float* ckpt, float* work, float* disp,
                              void* stream);
/* No counterpart in the reference. Gradients of sum(grad_disp * disp) with respect to cost, p1
 * and p2 (written, not accumulated); grad_sum [B][H][W][D] and work (sgm_float_workspace_elems
 * floats) are scratch. Each path's states are recomputed from the checkpoints, 8 pixels at a
 * time. grad_sum and grad_cost 16-byte aligned. */
SGM_API int sgm_float_backward(const float* cost, const float* p1, const float* p2, int32_t B, int32_t H, int32_t W,
                               int32_t D, float temperature, const float* sum, const float* ckpt,
                               const float* grad_disp, float* grad_sum, float* work, float* grad_cost,
                               float* grad_p1, float* grad_p2, void* stream);

/* ---------------- pyramid matcher (FasterStereoCuda) ---------------- */

/* Same layout as FasterStereoCuda::StereoOption1 (FasterStereoCuda/FasterStereoCuda.h:39-51). */
typedef struct sgm_pyr_option1_s {
  int32_t width, height, min_disp, max_disp, num_layers;
  bool do_lr_check, do_rm_peaks, do_smooth;
} sgm_pyr_option1_t;

/* No counterpart in the reference: replaces the census type and penalties that
 * SetSgmParameters (FasterStereoCuda.cpp:169-199) hard-codes for every level. */
typedef struct sgm_level_override_s {
  int32_t cs_type, p1, p2;
} sgm_level_override_t;

/* Same layout as FasterStereoCuda::EpipolarStereoParam and StereoOption2
 * (FasterStereoCuda/FasterStereoCuda.h:28-69). */
typedef struct sgm_epipolar_s {
  double x0_left, y0_left;
  double x0_right, y0_right;
  double baseline;
  double focus;
} sgm_epipolar_t;

typedef struct sgm_pyr_option2_s {
  int32_t width, height;
  float min_depth, max_depth;
  int32_t num_layers;
  bool do_lr_check, do_rm_peaks, do_smooth;
  sgm_epipolar_t epi;
} sgm_pyr_option2_t;

typedef struct sgm_pyramid* sgm_pyr_handle_t;

/* FasterStereoCuda::FasterStereoCuda / ~FasterStereoCuda -- FasterStereoCuda.cpp:693-703 */
SGM_API int sgm_pyr_create(sgm_pyr_handle_t* out);
SGM_API int sgm_pyr_destroy(sgm_pyr_handle_t h);
/* FasterStereoCuda::Init -- FasterStereoCuda.h:95, HierSgmCudaImpl::Init FasterStereoCuda.cpp:201-295.
 * override may be NULL (reference per-level parameters). */
SGM_API int sgm_pyr_init(sgm_pyr_handle_t h, const sgm_pyr_option1_t* option, const sgm_level_override_t* override_,
                         const sgm_ext_options_t* ext);
/* FasterStereoCuda::Match -- FasterStereoCuda.h:114, HierSgmCudaImpl::Match FasterStereoCuda.cpp:408-529.
 * All levels run on the device; no host round trip between levels. */
SGM_API int sgm_pyr_match(sgm_pyr_handle_t h, const uint8_t* img_left, const uint8_t* img_right, float* disp);
/* No counterpart in the reference: device-resident variant, enqueued on `stream` without synchronising. */
SGM_API int sgm_pyr_match_device(sgm_pyr_handle_t h, const uint8_t* d_left, const uint8_t* d_right, float* d_disp,
                                 void* stream);
/* FasterStereoCuda::Init2 -- FasterStereoCuda.h:102, HierSgmCudaImpl::Init2 FasterStereoCuda.cpp:297-406:
 * the coarsest disparity range comes from the depth range and the scaled camera. */
SGM_API int sgm_pyr_init2(sgm_pyr_handle_t h, const sgm_pyr_option2_t* option, const sgm_level_override_t* override_,
                          const sgm_ext_options_t* ext);
/* FasterStereoCuda::Match2 -- FasterStereoCuda.h:123, FasterStereoCuda.cpp:531-635: depth of the finest level. */
SGM_API int sgm_pyr_match2(sgm_pyr_handle_t h, const uint8_t* img_left, const uint8_t* img_right, float* depth);
/* FasterStereoCuda::Release -- FasterStereoCuda.h:105 */
SGM_API int sgm_pyr_release(sgm_pyr_handle_t h);
/* No counterpart in the reference: level geometry chosen by init (for tests and tools). */
SGM_API int sgm_pyr_level_info(sgm_pyr_handle_t h, int32_t level, int32_t* width, int32_t* height,
                               int32_t* min_disp, int32_t* disp_range);
SGM_API int64_t sgm_pyr_kernel_launches(sgm_pyr_handle_t h);
/* No counterpart in the reference. Tuning of one level (level >= 0) or of every level (-1),
 * after sgm_pyr_init. */
SGM_API int sgm_pyr_set_tuning(sgm_pyr_handle_t h, int32_t level, const sgm_tuning_t* t);

/* ---------------- batched pyramids ---------------- */

/* No counterpart in the reference. Batched pyramids: every pair's FasterStereoCuda::Match
 * (FasterStereoCuda.cpp:408-529: decimation, coarsest level with LR / dilation / small-region
 * removal per SetSgmParameters, then 32-disparity levels driven by the coarser map) for many
 * pairs of different sizes in one CUDA graph. pairs[i]: full-resolution width, height,
 * min_disparity and disp_range = max_disp - min_disp; option: num_layers, do_lr_check,
 * do_rm_peaks (do_smooth unsupported; its width/height/disparity fields are ignored); override
 * and ext as for sgm_pyr_init (ext may be NULL). Each pair's result is bit-identical to
 * sgm_pyr_match_device on that pair. */
typedef struct sgm_batch_pyr* sgm_batch_pyr_t;
SGM_API int sgm_batch_pyr_create(sgm_batch_pyr_t* out);
SGM_API int sgm_batch_pyr_destroy(sgm_batch_pyr_t p);
SGM_API const char* sgm_batch_pyr_last_error(sgm_batch_pyr_t p);
SGM_API int sgm_batch_pyr_init(sgm_batch_pyr_t p, const sgm_batch_pair_t* pairs, int32_t count,
                               const sgm_pyr_option1_t* option, const sgm_level_override_t* level_override,
                               const sgm_ext_options_t* ext);
/* Full-resolution input images and final disparity of pair `index` (device, dense). */
SGM_API int sgm_batch_pyr_pair_buffers(sgm_batch_pyr_t p, int32_t index, uint8_t** d_left, uint8_t** d_right,
                                       float** d_disp);
SGM_API int sgm_batch_pyr_run(sgm_batch_pyr_t p, void* stream);
SGM_API int sgm_batch_pyr_match(sgm_batch_pyr_t p, const uint8_t* const* left, const uint8_t* const* right,
                                float* const* disp);
SGM_API int sgm_batch_pyr_info(sgm_batch_pyr_t p, sgm_batch_info_t* info);

#ifdef __cplusplus
}
#endif
#endif
