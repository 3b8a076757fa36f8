/*
 * CPU oracle for the SGM stereo path. TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's algorithm
 * (ethan-li-coding/FasterStereoCuda, SgmStereoCuda/ + FasterStereoCuda/).
 * It exists to check the CUDA product path and to serve as the timed host
 * baseline. Nothing in the product library links, loads or calls it.
 *
 * Parity pin: the host-side stages (small-region removal, decimation,
 * next-level initial disparity) are checked against the reference's own
 * compiled functions; the device stages are checked against dumps produced by
 * the reference's CUDA build run on a B200 (tests/golden/).
 *
 * Buffer conventions (all dense, row-major, no pitch):
 *   images        uint8  [H][W]
 *   census        uint64 [H][W]   (5x5 census zero-extended from 32 bits)
 *   cost / paths  uint8  [H][W][D] (disparity fastest)
 *   disparity     float  [H][W]   (INVALID = -999999.0f)
 *   init disparity int16 [H][W]   (INVALID = -32768)
 */
#ifndef SGM_ORACLE_H_
#define SGM_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_INVALID_FLOAT (-999999.0f)
#define ORC_INVALID_SHORT (-32768)
#define ORC_INVALID_COST 127
#define ORC_LEVEL_RANGE 32

/* WTA tie rules: which disparity wins when several share the minimum. */
enum {
  ORC_TIE_LOWEST = 0,     /* smallest d */
  ORC_TIE_HIGHEST = 1,    /* largest d */
  ORC_TIE_LANE_HIGH = 2,  /* warp mapping d = lane + 32*j: highest lane wins, lowest j within it */
  ORC_TIE_LANE_LOW = 3,   /* warp mapping d = lane + 32*j: lowest lane wins, lowest j within it */
  ORC_TIE_REF_B200 = 4    /* the reference build's behaviour measured on a B200 (see orc_wta_plain/init) */
};

/* Region-growing neighbour test used by small-region removal. */
enum {
  ORC_PEAKS_ABS_INT = 0,   /* |(int)(a-b)| <= 1  (reference built with g++: int abs overload) */
  ORC_PEAKS_ABS_FLOAT = 1  /* fabsf(a-b) <= 1.0f (reference built with MSVC: float abs overload) */
};

typedef struct {
  int32_t width, height;
  int32_t min_disp, disp_range;
  int32_t cs_type;          /* 0 = 5x5 (uint32), 1 = 9x7 (uint64) */
  int32_t p1, p2;
  float uniqueness;
  int32_t do_lr_check;
  float lr_threshold;
  int32_t do_median;
  int32_t morphology_dilation; /* 1 = dilation after median (pyramid coarsest level) */
  int32_t do_remove_peaks;
  float peaks_ratio;
  int32_t peaks_strips;     /* number of horizontal strips (reference: hardware threads * 3/4) */
  int32_t peaks_abs_mode;   /* ORC_PEAKS_ABS_* */
  int32_t tie_rule;         /* plain-path WTA tie rule */
  int32_t init_tie_rule;    /* init-disparity WTA tie rule */
  int32_t p2_div0;          /* value of P2 / 0 at init-disparity levels */
  int32_t threads;          /* OpenMP threads, <= 0: runtime default */
  int32_t post_filter;      /* 0 none, 1 Gauss, 2 bilateral (after the median) */
  int32_t morphology;       /* 0: as morphology_dilation; 1 erosion, 2 dilation, 3 open, 4 close */
  /* regions of interest (StereoROI_T of StereoCuda::Match) of the left and the right view; the
   * rectangle must lie inside the image. Plain levels only. */
  int32_t roi_l_enable, roi_l_x, roi_l_y, roi_l_w, roi_l_h;
  int32_t roi_r_enable, roi_r_x, roi_r_y, roi_r_w, roi_r_h;
} orc_config_t;

/* ---- stages ---- */
void orc_census(const uint8_t* img, int W, int H, int cs_type, int is_right, uint64_t* out);
void orc_cost_plain(const uint64_t* cl, const uint64_t* cr, int W, int H, int min_d, int D, int cs_type,
                    int left2right, uint8_t* cost);
void orc_cost_init(const uint64_t* cl, const uint64_t* cr, const int16_t* init, int W, int H, int x0, int D,
                   int cs_type, int left2right, uint8_t* cost);
/* dir: 0 = top->bottom, 1 = left->right, 2 = bottom->top, 3 = right->left */
void orc_path_plain(const uint8_t* cost, int W, int H, int x0, int D, int32_t p1, int32_t p2, int dir,
                    uint8_t* out);
void orc_path_init(const uint8_t* cost, const int16_t* init, int W, int H, int x0, int D, int32_t p1, int32_t p2,
                   int32_t p2_div0, int dir, uint8_t* out);
void orc_wta_plain(const uint8_t* const paths[4], int W, int H, int x0, int min_d, int D, float uniqueness,
                   int tie_rule, float* disp);
void orc_wta_init(const uint8_t* const paths[4], const int16_t* init, int W, int H, int x0, int D,
                  float uniqueness, int tie_rule, float* disp);
void orc_lr_check(float* disp_l, const float* disp_r_snapshot, float* disp_r_out, int W, int H, float threshold);
void orc_median3x3(const float* in, float* out, int W, int H);
void orc_dilation(const float* in, float* out, int W, int H, int wnd);
void orc_erosion(const float* in, float* out, int W, int H, int wnd);
void orc_gauss(const float* in, float* out, int W, int H, float sigma_d, float sigma_r);
void orc_bilateral(const uint8_t* img, const float* in, float* out, int W, int H, float sigma_d, float sigma_r);
int orc_remove_peaks(float* disp, int W, int H, int strips, float ratio, int abs_mode);
int orc_remove_peaks_strip(float* disp, int w, int h, int threshold, int abs_mode);
void orc_zoom_half(const uint8_t* src, int w_src, int h_src, uint8_t* dst);
void orc_init_next_level(const float* cur, int w_cur, int h_cur, int16_t* next, int width, int height);
uint8_t orc_cost_adjust(int d);

/* ---- whole single-level match (StereoCuda::Match) ----
 * init may be NULL (plain path). disp_r may be NULL. Returns 0 on success. */
int orc_match(const orc_config_t* cfg, const uint8_t* left, const uint8_t* right, const int16_t* init,
              float* disp_l, float* disp_r);

/* Stage dump variant used by tests: any output pointer may be NULL.
 * cost_* are [H][W][D], paths_* [4][H][W][D] (left view: *_lr, right view: *_rl, the latter
 * only computed with the LR check); wta_* are the WTA maps before LR/median. */
int orc_match_dump(const orc_config_t* cfg, const uint8_t* left, const uint8_t* right, const int16_t* init,
                   uint64_t* census_l, uint64_t* census_r, uint8_t* cost_lr, uint8_t* paths_lr, float* wta_l,
                   uint8_t* cost_rl, uint8_t* paths_rl, float* wta_r, float* disp_l, float* disp_r);

/* ---- pyramid (FasterStereoCuda::Match) ---- */
typedef struct {
  int32_t width, height, min_disp, max_disp, num_layers;
  int32_t do_lr_check, do_rm_peaks, do_smooth;
  /* override of the per-level census/penalties (the reference hard-codes 5x5, 8/32) */
  int32_t override_enable, cs_type, p1, p2;
  int32_t peaks_strips, peaks_abs_mode, tie_rule, init_tie_rule, p2_div0, threads;
} orc_pyr_config_t;

/* Per-level configuration the pyramid driver derives (FasterStereoCuda.cpp:201-295). */
int orc_pyr_level_config(const orc_pyr_config_t* pc, int level, orc_config_t* out);
int orc_pyr_match(const orc_pyr_config_t* pc, const uint8_t* left, const uint8_t* right, float* disp);

void orc_set_threads(int n);
int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
