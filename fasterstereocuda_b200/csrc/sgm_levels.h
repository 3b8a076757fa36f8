// Host-side rules shared by the pyramid matcher and the batched pyramid.
#pragma once
#include <cstring>
#include <thread>

#include "../../include/sgm_b200.h"
#include "sgm_common.cuh"

// Strips of the small-region removal when none are set: 3/4 of the host's hardware threads, as
// the reference sizes its removal thread pool (StereoCudaImpl.cpp:238-249).
inline int default_peaks_strips() {
  const unsigned hc = std::thread::hardware_concurrency();
  const int n = (int)(hc * 3 / 4);
  return n > 0 ? n : 1;
}

// Options, minimum disparity and disparity range of pyramid level `level` of `layers`
// (reference SetSgmParameters, FasterStereoCuda.cpp:169-199, and the range rules of
// HierSgmCudaImpl::Init, FasterStereoCuda.cpp:201-295).
inline void level_options(const sgm_pyr_option1_t* o, const sgm_level_override_t* ov, int level, int layers,
                   sgm_option_t* so, int* dmin_out, int* drange_out) {
  std::memset(so, 0, sizeof(*so));
  so->p1 = ov ? ov->p1 : 8;
  so->p2_init = ov ? ov->p2 : 32;
  so->p2_max = 64;
  so->cs_type = ov ? ov->cs_type : 0;
  so->num_paths = 4;
  so->unique_threshold = level == 0 ? 0.95f : 1.0f;
  so->lr_threshold = 1.0f;
  so->do_median_filter = true;
  so->post_filter_type = (level == 0 && o->do_smooth) ? 1 : 0;  // Gauss at the finest level
  so->using_constant_p2 = true;
  if (layers <= 1) {
    so->do_lr_check = o->do_lr_check;
    so->do_remove_peaks = o->do_rm_peaks;
    so->peaks_ratio_threshold = 0.0005f;
    so->morphology_type = 0;
  } else if (layers <= 2) {
    so->do_lr_check = level == 0 ? false : o->do_lr_check;
    so->do_remove_peaks = level == 0 ? false : o->do_rm_peaks;
    so->peaks_ratio_threshold = level == 0 ? 0.0005f : 0.001f;
    so->morphology_type = level < layers - 1 ? 0 : 2;
  } else {
    so->do_lr_check = level < layers - 1 ? false : o->do_lr_check;
    so->do_remove_peaks = level < layers - 1 ? false : o->do_rm_peaks;
    so->peaks_ratio_threshold = level < layers - 1 ? 0.0005f : 0.005f;
    so->morphology_type = level < layers - 1 ? 0 : 2;
  }
  const int scale = 1 << level;
  if (level == layers - 1) {
    int dmin = o->min_disp / scale, dmax = o->max_disp / scale;
    int range = dmax - dmin;
    int k = 6;
    while ((1 << k) < range) ++k;
    range = 1 << k;
    if (range > 2 * o->width) range /= 2;
    if (dmin >= o->width) {
      dmin = o->width - range;
      if (dmin < -o->width) dmin = -o->width;
    }
    *dmin_out = dmin;
    *drange_out = range;
  } else {
    *dmin_out = 0;
    *drange_out = sgm::kLevelRange;
  }
}
