/*
 * sgm_types.h -- value types of the StereoCuda C++ interface.
 *
 * Interface-compatible with SgmStereoCuda/sgm_types.h of the reference
 * (ethan-li-coding/FasterStereoCuda): the same type names, member order, member
 * types and default values, so that objects built against either header have
 * the same layout and the same mangled symbol names.
 */
#pragma once

#include <cstdint>
#include <vector>

#define INVALID_VALUE -999999.0f

typedef float float32;
typedef double float64;
typedef uint8_t uint8;
typedef uint16_t uint16;
typedef uint32_t uint32;
typedef uint64_t uint64;
typedef int8_t sint8;
typedef int16_t sint16;
typedef int32_t sint32;
typedef int64_t sint64;

#ifndef STEREO_SGM_PARAM_T
#define STEREO_SGM_PARAM_T
/* Matching options (reference: sgm_types.h:21-65). Defaults: P1 8, P2 32, census 5x5,
 * everything else off / zero. The layout equals sgm_option_t of sgm_b200.h. */
class CuSGMOption {
 public:
  enum CS_Type { CS_5x5 = 0, CS_9x7 };
  enum PF_Type { PF_NONE = 0, PF_GAUSS, PF_BILATERAL };
  enum MP_Type { MP_NONE = 0, MP_EROSION, MP_DILATION, MP_OPEN, MP_CLOSE };

  CuSGMOption()
      : p1(8), p2_init(32), p2_max(0), cs_type(CS_5x5), num_paths(0), do_median_filter(false), do_lr_check(false),
        lr_threshold(0), unique_threshold(0), using_constant_p2(false), do_remove_peaks(false),
        peaks_ratio_threshold(0), post_filter_type(PF_NONE), morphology_type(MP_NONE) {}
  ~CuSGMOption() = default;

  sint32 p1;
  sint32 p2_init;
  sint32 p2_max;
  CS_Type cs_type;
  sint32 num_paths;
  bool do_median_filter;
  bool do_lr_check;
  float32 lr_threshold;
  float32 unique_threshold;
  bool using_constant_p2;
  bool do_remove_peaks;
  float32 peaks_ratio_threshold;
  PF_Type post_filter_type;
  MP_Type morphology_type;
};
#endif

#ifndef STEREO_CAMERA_PARAM_T
#define STEREO_CAMERA_PARAM_T
/* Rectified camera parameters (reference: sgm_types.h:70-84). */
typedef struct CameraParam_T {
  float64 x0_left, y0_left;
  float64 x0_right, y0_right;
  float64 focus;
  float64 baseline;

  /* parameters of the image scaled down by s (baseline unchanged) */
  CameraParam_T Scale(const int& s) const {
    CameraParam_T c{};
    c.x0_left = x0_left / s;
    c.y0_left = y0_left / s;
    c.x0_right = x0_right / s;
    c.y0_right = y0_right / s;
    c.focus = focus / s;
    c.baseline = baseline;
    return c;
  }
} CamParam_T;
#endif

#ifndef STEREO_ROI_T
#define STEREO_ROI_T
/* Region of interest (reference: sgm_types.h:89-92). */
struct StereoROI_T {
  sint32 x, y, w, h;
};
#endif
