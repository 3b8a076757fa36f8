/*
 * StereoCuda.h -- C++ single-level matcher, interface-compatible with the reference's
 * SgmStereoCuda/StereoCuda.h (ethan-li-coding/FasterStereoCuda): same class name, same
 * single-pointer layout, same member functions with the same signatures, so code written
 * (or compiled) against the reference links against libsgmb200.so unchanged.
 * Implemented on the C ABI of sgm_b200.h.
 */
#pragma once
#include "sgm_types.h"

#if defined(_WIN32)
#define STEREO_CUDA_DLL __declspec(dllexport)
#else
#define STEREO_CUDA_DLL __attribute__((visibility("default")))
#endif

class STEREO_CUDA_DLL StereoCuda {
 public:
  StereoCuda();
  ~StereoCuda();

  /* Allocates the device buffers for width x height and disparities
   * [min_disparity, min_disparity + disp_range). Returns false on bad arguments,
   * unsupported options or CUDA errors. */
  bool Init(sint32 width, sint32 height, sint32 min_disparity, sint32 disp_range, CuSGMOption sgm_option,
            bool print_log = false) const;

  /* Matches one rectified pair (host buffers of width*height). disp_left receives the left
   * disparity map (INVALID_VALUE where rejected); disp_right, when given, the right map of the
   * consistency check; init_disp_left, when given, per-pixel initial disparities (32-disparity
   * levels). Synchronous. */
  bool Match(uint8* img_left, uint8* img_right, float32* disp_left, float32* disp_right = nullptr,
             sint16* init_disp_left = nullptr, StereoROI_T* ste_roi_left = nullptr,
             StereoROI_T* ste_roi_right = nullptr) const;

  /* As Init, and keeps the camera parameters for Match2 (disparity -> depth). */
  bool Init2(sint32 width, sint32 height, sint32 min_disparity, sint32 disp_range, CuSGMOption sgm_option,
             CamParam_T cam_param, bool print_log = false) const;

  /* Matches and converts the left disparity map into depth = baseline * focus / (d + x0r - x0l). */
  bool Match2(uint8* img_left, uint8* img_right, float32* depth_left, sint16* init_disp_left = nullptr,
              StereoROI_T* ste_roi_left = nullptr, StereoROI_T* ste_roi_right = nullptr) const;

  void SetMinDisparity(const sint32& min_disparty);
  sint32 GetDispartyRange();

  /* Frees the device buffers. */
  void Release() const;

  static void GetRoiFromDispMap(float32* disp_ptr, sint32 width, sint32 height, StereoROI_T& ste_roi);
  static float32 get_invad_float();
  static sint16 get_invad_short();
  static sint16 get_level_range();
  static bool MallocPageLockedPtr(void** ptr, size_t size);
  static bool FreePageLockedPtr(void* ptr);

 private:
  void* impl_;
};
