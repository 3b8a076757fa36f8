// C++ classes StereoCuda and FasterStereoCuda (include/StereoCuda.h, include/FasterStereoCuda.h)
// implemented on the C ABI. The classes keep the reference's single-pointer layout; the
// pointer holds the C handle.
#include <cstddef>

#include "../../include/FasterStereoCuda.h"
#include "../../include/StereoCuda.h"
#include "../../include/sgm_b200.h"

static_assert(sizeof(CuSGMOption) == sizeof(sgm_option_t), "CuSGMOption layout");
static_assert(offsetof(CuSGMOption, lr_threshold) == offsetof(sgm_option_t, lr_threshold), "CuSGMOption layout");
static_assert(offsetof(CuSGMOption, morphology_type) == offsetof(sgm_option_t, morphology_type), "CuSGMOption layout");
static_assert(sizeof(StereoROI_T) == sizeof(sgm_roi_t), "StereoROI_T layout");
static_assert(sizeof(CamParam_T) == sizeof(sgm_camera_t), "CamParam_T layout");
static_assert(sizeof(FasterStereoCuda::StereoOption1) == sizeof(sgm_pyr_option1_t), "StereoOption1 layout");
static_assert(sizeof(FasterStereoCuda::StereoOption2) == sizeof(sgm_pyr_option2_t), "StereoOption2 layout");
static_assert(offsetof(FasterStereoCuda::StereoOption2, epi) == offsetof(sgm_pyr_option2_t, epi), "StereoOption2 layout");
static_assert(sizeof(StereoCuda) == sizeof(void*) && sizeof(FasterStereoCuda) == sizeof(void*), "pimpl layout");

namespace {
inline sgm_handle_t H(void* p) { return static_cast<sgm_handle_t>(p); }
inline sgm_pyr_handle_t P(void* p) { return static_cast<sgm_pyr_handle_t>(p); }
inline const sgm_roi_t* roi(const StereoROI_T* r) { return reinterpret_cast<const sgm_roi_t*>(r); }
}  // namespace

StereoCuda::StereoCuda() : impl_(nullptr) {
  sgm_handle_t h = nullptr;
  if (sgm_create(&h) == SGM_OK) impl_ = h;
}

StereoCuda::~StereoCuda() {
  if (impl_) sgm_destroy(H(impl_));
  impl_ = nullptr;
}

bool StereoCuda::Init(sint32 width, sint32 height, sint32 min_disparity, sint32 disp_range, CuSGMOption sgm_option,
                      bool print_log) const {
  return impl_ && sgm_init(H(impl_), width, height, min_disparity, disp_range,
                           reinterpret_cast<const sgm_option_t*>(&sgm_option), print_log) == SGM_OK;
}

bool StereoCuda::Match(uint8* img_left, uint8* img_right, float32* disp_left, float32* disp_right,
                       sint16* init_disp_left, StereoROI_T* ste_roi_left, StereoROI_T* ste_roi_right) const {
  return impl_ && sgm_match(H(impl_), img_left, img_right, disp_left, disp_right, init_disp_left, roi(ste_roi_left),
                            roi(ste_roi_right)) == SGM_OK;
}

bool StereoCuda::Init2(sint32 width, sint32 height, sint32 min_disparity, sint32 disp_range, CuSGMOption sgm_option,
                       CamParam_T cam_param, bool print_log) const {
  return impl_ && sgm_init2(H(impl_), width, height, min_disparity, disp_range,
                            reinterpret_cast<const sgm_option_t*>(&sgm_option),
                            reinterpret_cast<const sgm_camera_t*>(&cam_param), print_log) == SGM_OK;
}

bool StereoCuda::Match2(uint8* img_left, uint8* img_right, float32* depth_left, sint16* init_disp_left,
                        StereoROI_T* ste_roi_left, StereoROI_T* ste_roi_right) const {
  return impl_ && sgm_match2(H(impl_), img_left, img_right, depth_left, init_disp_left, roi(ste_roi_left),
                             roi(ste_roi_right)) == SGM_OK;
}

void StereoCuda::SetMinDisparity(const sint32& min_disparty) {
  if (impl_) sgm_set_min_disparity(H(impl_), min_disparty);
}

sint32 StereoCuda::GetDispartyRange() { return impl_ ? sgm_get_disparity_range(H(impl_)) : 0; }

void StereoCuda::Release() const {
  if (impl_) sgm_release(H(impl_));
}

void StereoCuda::GetRoiFromDispMap(float32* disp_ptr, sint32 width, sint32 height, StereoROI_T& ste_roi) {
  sgm_roi_from_disp_map(disp_ptr, width, height, reinterpret_cast<sgm_roi_t*>(&ste_roi));
}

float32 StereoCuda::get_invad_float() { return sgm_invalid_float(); }
sint16 StereoCuda::get_invad_short() { return sgm_invalid_short(); }
sint16 StereoCuda::get_level_range() { return sgm_level_range(); }
bool StereoCuda::MallocPageLockedPtr(void** ptr, size_t size) { return sgm_malloc_page_locked(ptr, size) == SGM_OK; }
bool StereoCuda::FreePageLockedPtr(void* ptr) { return sgm_free_page_locked(ptr) == SGM_OK; }

FasterStereoCuda::FasterStereoCuda() : impl_(nullptr) {
  sgm_pyr_handle_t h = nullptr;
  if (sgm_pyr_create(&h) == SGM_OK) impl_ = h;
}

FasterStereoCuda::~FasterStereoCuda() {
  if (impl_) sgm_pyr_destroy(P(impl_));
  impl_ = nullptr;
}

bool FasterStereoCuda::MallocPageLockedPtr(void** ptr, size_t size) {
  return sgm_malloc_page_locked(ptr, size) == SGM_OK;
}

bool FasterStereoCuda::FreePageLockedPtr(void* ptr) { return sgm_free_page_locked(ptr) == SGM_OK; }

bool FasterStereoCuda::Init(const ste_opt1_t& option) const {
  return impl_ && sgm_pyr_init(P(impl_), reinterpret_cast<const sgm_pyr_option1_t*>(&option), nullptr, nullptr) ==
                      SGM_OK;
}

bool FasterStereoCuda::Init2(const ste_opt2_t& option) const {
  return impl_ && sgm_pyr_init2(P(impl_), reinterpret_cast<const sgm_pyr_option2_t*>(&option), nullptr, nullptr) ==
                      SGM_OK;
}

void FasterStereoCuda::Release() const {
  if (impl_) sgm_pyr_release(P(impl_));
}

bool FasterStereoCuda::Match(const unsigned char* bytes_left, const unsigned char* bytes_right,
                             float* disparity_data) const {
  return impl_ && sgm_pyr_match(P(impl_), bytes_left, bytes_right, disparity_data) == SGM_OK;
}

bool FasterStereoCuda::Match2(const unsigned char* bytes_left, const unsigned char* bytes_right,
                              float* depth_data) const {
  return impl_ && sgm_pyr_match2(P(impl_), bytes_left, bytes_right, depth_data) == SGM_OK;
}
