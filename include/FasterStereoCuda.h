/*
 * FasterStereoCuda.h -- C++ pyramid matcher, interface-compatible with the reference's
 * FasterStereoCuda/FasterStereoCuda.h (ethan-li-coding/FasterStereoCuda): same class name,
 * nested option types, layout and member signatures. Implemented on sgm_b200.h; all pyramid
 * levels run on the GPU.
 */
#ifndef FASTERSTEREOCUDA_STEREO_H_
#define FASTERSTEREOCUDA_STEREO_H_

#if defined(_WIN32)
#define FASTERSTEREOCUDA_DLL __declspec(dllexport)
#else
#define FASTERSTEREOCUDA_DLL __attribute__((visibility("default")))
#endif

#include <cstddef>

class FASTERSTEREOCUDA_DLL FasterStereoCuda {
 public:
  /* rectified pair geometry */
  typedef struct EpipolarStereoParam {
    double x0_left, y0_left;
    double x0_right, y0_right;
    double baseline;
    double focus;
    EpipolarStereoParam() { x0_left = y0_left = x0_right = y0_right = focus = baseline = 0; }
  } epi_ste_t;

  /* options of disparity output */
  typedef struct StereoOption1 {
    int width;
    int height;
    int min_disp;
    int max_disp;
    int num_layers;
    bool do_lr_check;
    bool do_rm_peaks;
    bool do_smooth;
    StereoOption1()
        : width(0), height(0), min_disp(0), max_disp(0), num_layers(1), do_lr_check(true), do_rm_peaks(true),
          do_smooth(false) {}
  } ste_opt1_t;

  /* options of depth output */
  typedef struct StereoOption2 {
    int width;
    int height;
    float min_depth;
    float max_depth;
    int num_layers;
    bool do_lr_check;
    bool do_rm_peaks;
    bool do_smooth;
    epi_ste_t epi;
    StereoOption2()
        : width(0), height(0), min_depth(0), max_depth(0), num_layers(1), do_lr_check(true), do_rm_peaks(true),
          do_smooth(false) {}
  } ste_opt2_t;

 public:
  FasterStereoCuda();
  ~FasterStereoCuda();

  static bool MallocPageLockedPtr(void** ptr, size_t size);
  static bool FreePageLockedPtr(void* ptr);

 public:
  bool Init(const ste_opt1_t& option) const;
  bool Init2(const ste_opt2_t& option) const;
  void Release() const;
  /* disparity map of the finest level (INVALID = -999999.0f), host buffers of width*height */
  bool Match(const unsigned char* bytes_left, const unsigned char* bytes_right, float* disparity_data) const;
  /* depth map */
  bool Match2(const unsigned char* bytes_left, const unsigned char* bytes_right, float* depth_data) const;

 private:
  void* impl_;
};

#endif
