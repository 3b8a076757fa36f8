/*
 * CPU oracle for the SGM stereo path -- TEST INFRASTRUCTURE ONLY (see sgm_oracle.h).
 *
 * Each function restates one stage of the reference, with the reference file:line it
 * follows. Where the reference is racy or reads memory it never wrote, the oracle
 * implements one fixed, documented rule instead (noted at each function).
 *
 * Build: gcc -O3 -march=native -fopenmp -ffp-contract=off -fPIC -shared
 * (-ffp-contract=off keeps every float operation individually rounded, as the
 *  reference's device code does for the expressions restated here).
 */
#include "sgm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
static int nthreads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

static inline uint32_t umin(uint32_t a, uint32_t b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }

/* Census transform. SgmStereoCuda/cusgm_cc.cu:30-67 (5x5) and :68-106 (9x7).
 * Bit order: row-major over the window, MSB first; bit set when neighbour < centre.
 * Border pixels take the kernel's invalid_val: 0 for the left view and the 32-bit
 * 0xFFFFFFFF (zero-extended into 64 bits for 9x7) for the right view
 * (cusgm_cc.cu:450-465). */
void orc_census(const uint8_t* img, int W, int H, int cs_type, int is_right, uint64_t* out) {
  const int csw = cs_type ? 4 : 2, csh = cs_type ? 3 : 2;
  const uint64_t border = is_right ? 0xFFFFFFFFull : 0ull;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      uint64_t v = 0;
      if (x < csw || x >= W - csw || y < csh || y >= H - csh) {
        v = border;
      } else {
        const uint8_t c = img[(size_t)y * W + x];
        for (int dy = -csh; dy <= csh; ++dy) {
          const uint8_t* row = img + (size_t)(y + dy) * W + x;
          for (int dx = -csw; dx <= csw; ++dx) v = (v << 1) | (uint64_t)(row[dx] < c);
        }
      }
      out[(size_t)y * W + x] = v;
    }
  }
}

static inline uint8_t hamming(uint64_t a, uint64_t b) { return (uint8_t)__builtin_popcountll(a ^ b); }

/* Plain Hamming cost. cusgm_cc.cu:118-172 (9x7), :238-293 (5x5), launch :472-523.
 * left2right:  C(x,d) = popc(cl[x] ^ cr[x - min_d - d])   (out of range -> cr[0])
 * right2left:  C(x,d) = popc(cl[x] ^ cr[x + min_d + d])   (out of range -> cr[0]);
 *              the caller passes (census_right, census_left) as (cl, cr) for this pass.
 * Only x in [max(0,min_d), W) is written. The 5x5 right-to-left kernel stops one pixel
 * short in every block of D pixels (cusgm_cc.cu:288): those pixels keep what the
 * buffer held before (the left-to-right cost of the same call), so `cost` is in/out. */
/* blk_x0: first column of the kernel's D-pixel blocks (x0, or the ROI's x for the right view of a
 * match with a region of interest, cusgm_cc.cu:478-488 via LRCheck :4191). */
static void cost_plain_blocks(const uint64_t* cl, const uint64_t* cr, int W, int H, int min_d, int D, int cs_type,
                              int left2right, int blk_x0, uint8_t* cost) {
  const int x0 = imax(0, min_d);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 0; y < H; ++y) {
    const uint64_t* l = cl + (size_t)y * W;
    const uint64_t* r = cr + (size_t)y * W;
    for (int x = x0; x < W; ++x) {
      if (!left2right && cs_type == 0 && x >= blk_x0) {
        const int blk_start = blk_x0 + ((x - blk_x0) / D) * D;
        const int iend = imin(D, W - blk_start);
        if (x == blk_start + iend - 1) continue; /* stale pixel */
      }
      uint8_t* c = cost + ((size_t)y * W + x) * D;
      for (int d = 0; d < D; ++d) {
        const int pos = left2right ? x - min_d - d : x + min_d + d;
        const uint64_t rv = (pos >= 0 && pos < W) ? r[pos] : r[0];
        c[d] = hamming(l[x], rv);
      }
    }
  }
}

void orc_cost_plain(const uint64_t* cl, const uint64_t* cr, int W, int H, int min_d, int D, int cs_type,
                    int left2right, uint8_t* cost) {
  cost_plain_blocks(cl, cr, W, H, min_d, D, cs_type, left2right, imax(0, min_d), cost);
}

/* CostAdjust, cusgm_cc.cu:14-21: (uint8)expf(4*|d-16|/16) with integer division, i.e.
 * floor(e^k) for k = 0..4 (1, 2, 7, 20, 54); none of these is near an integer boundary. */
uint8_t orc_cost_adjust(int d) {
  static const uint8_t tab[5] = {1, 2, 7, 20, 54};
  int k = 4 * abs(d - ORC_LEVEL_RANGE / 2) / (ORC_LEVEL_RANGE / 2);
  if (k < 0) k = 0;
  if (k > 4) k = 4;
  return tab[k];
}

/* Cost with a per-pixel initial disparity. cusgm_cc.cu:173-237 (9x7), :294-360 (5x5).
 * left2right:  pos = x - d - init[x]; valid iff 0 < pos < W (strict);
 *              C = popc(cl[x]^cr[pos]) + CostAdjust(d), else 0xFF (9x7) / 127 (5x5).
 * right2left:  pos = x + d + init[x]; C = popc(cl[x] ^ (0<pos<W ? cr[pos] : cr[0])) + CostAdjust(d). */
void orc_cost_init(const uint64_t* cl, const uint64_t* cr, const int16_t* init, int W, int H, int x0, int D,
                   int cs_type, int left2right, uint8_t* cost) {
  const uint8_t invalid = cs_type ? 0xFF : ORC_INVALID_COST;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 0; y < H; ++y) {
    const uint64_t* l = cl + (size_t)y * W;
    const uint64_t* r = cr + (size_t)y * W;
    const int16_t* iv = init + (size_t)y * W;
    for (int x = x0; x < W; ++x) {
      uint8_t* c = cost + ((size_t)y * W + x) * D;
      for (int d = 0; d < D; ++d) {
        if (left2right) {
          const int pos = x - d - iv[x];
          c[d] = (pos > 0 && pos < W) ? (uint8_t)(hamming(l[x], r[pos]) + orc_cost_adjust(d)) : invalid;
        } else {
          const int pos = x + d + iv[x];
          const uint64_t rv = (pos > 0 && pos < W) ? r[pos] : r[0];
          c[d] = (uint8_t)(hamming(l[x], rv) + orc_cost_adjust(d));
        }
      }
    }
  }
}

/* One recurrence step of the plain path (cusgm_ca.cu:1517-1564 for D=64; same for 32/128):
 * L_p(d) = C_p(d) + min(L_q(d), L_q(d-1)+P1, L_q(d+1)+P1, m_q+P2) - m_q in uint32,
 * where the out-of-range neighbour candidates are the constant 127 (INVALID_COST). */
static inline uint32_t step_plain(const uint8_t* c, const uint32_t* Lq, uint32_t mq, int D, uint32_t p1, uint32_t p2,
                                  uint32_t* Lp) {
  uint32_t m = 0xFFFFFFFFu;
  const uint32_t l4 = mq + p2;
  for (int d = 0; d < D; ++d) {
    const uint32_t a = d > 0 ? Lq[d - 1] + p1 : ORC_INVALID_COST;
    const uint32_t b = d < D - 1 ? Lq[d + 1] + p1 : ORC_INVALID_COST;
    const uint32_t t = umin(umin(umin(Lq[d], a), b), l4);
    const uint32_t v = (uint32_t)c[d] + (t - mq);
    Lp[d] = v;
    m = umin(m, v);
  }
  return m;
}

/* Plain path aggregation, one direction. Kernels cusgm_ca.cu:1343-1888, launched at
 * :4082-4123 (directions: 0 top->bottom, 1 left->right, 2 bottom->top, 3 right->left).
 * Paths cover x in [x0, W) and every row. The stored value is (uint8)L.
 * The reference never stores the first pixel of a path; here it stores (uint8)C there. */
/* The same over a region of interest (StereoCuda::Match with a StereoROI_T): horizontal paths run
 * along rows [y0, y1) from x0 to x1-1 (or back), vertical paths along columns [x0, x1) from y0 to
 * y1-1 (or back): the kernels' xoffset / xEnd / yoffset / yend (cusgm_ca.cu:3991-3999, :1478-1598). */
static void path_plain_region(const uint8_t* cost, int W, int x0, int x1, int y0, int y1, int D, int32_t p1,
                              int32_t p2, int dir, uint8_t* out) {
  const int horizontal = (dir == 1 || dir == 3);
  const int forward = (dir == 0 || dir == 1);
  const int nlines = horizontal ? (y1 - y0) : (x1 - x0);
  const int len = horizontal ? (x1 - x0) : (y1 - y0);
  if (nlines <= 0 || len <= 0) return;
#pragma omp parallel num_threads(nthreads())
  {
    uint32_t* Lq = (uint32_t*)malloc(sizeof(uint32_t) * D);
    uint32_t* Lp = (uint32_t*)malloc(sizeof(uint32_t) * D);
#pragma omp for schedule(static)
    for (int line = 0; line < nlines; ++line) {
      uint32_t m = 0xFFFFFFFFu;
      for (int s = 0; s < len; ++s) {
        const int k = forward ? s : len - 1 - s;
        const int x = horizontal ? x0 + k : x0 + line;
        const int y = horizontal ? y0 + line : y0 + k;
        const size_t off = ((size_t)y * W + x) * D;
        const uint8_t* c = cost + off;
        if (s == 0) {
          m = 0xFFFFFFFFu;
          for (int d = 0; d < D; ++d) { Lq[d] = c[d]; m = umin(m, Lq[d]); }
          for (int d = 0; d < D; ++d) out[off + d] = (uint8_t)Lq[d];
          continue;
        }
        m = step_plain(c, Lq, m, D, (uint32_t)p1, (uint32_t)p2, Lp);
        for (int d = 0; d < D; ++d) { out[off + d] = (uint8_t)Lp[d]; Lq[d] = Lp[d]; }
      }
    }
    free(Lq);
    free(Lp);
  }
}

void orc_path_plain(const uint8_t* cost, int W, int H, int x0, int D, int32_t p1, int32_t p2, int dir,
                    uint8_t* out) {
  path_plain_region(cost, W, x0, W, 0, H, D, p1, p2, dir, out);
}

/* Path aggregation with per-pixel base disparities (D = 32 levels of the pyramid).
 * cusgm_ca.cu:1181-1261 (horizontal) and :1263-1338 (vertical), launched :4055-4069.
 *   neighbour indices are realigned by base - last_base and must fall in [0, 32);
 *   the same-d candidate uses the unaligned previous L(d);
 *   P2' = max(P1, P2 / |last_base - base + 1|) (integer; a zero divisor gives p2_div0);
 *   a pixel whose base is INVALID is skipped: nothing stored, state kept, m := 127;
 *   the vertical kernels start last_base from row 0 in both directions (:1291).
 * All arithmetic is uint32 as in the reference (wraps are kept). */
void orc_path_init(const uint8_t* cost, const int16_t* init, int W, int H, int x0, int D, int32_t p1, int32_t p2,
                   int32_t p2_div0, int dir, uint8_t* out) {
  const int horizontal = (dir == 1 || dir == 3);
  const int forward = (dir == 0 || dir == 1);
  const int nlines = horizontal ? H : (W - x0);
  const int len = horizontal ? (W - x0) : H;
  if (nlines <= 0 || len <= 0) return;
#pragma omp parallel num_threads(nthreads())
  {
    uint32_t* Lq = (uint32_t*)malloc(sizeof(uint32_t) * D);
    uint32_t* Lp = (uint32_t*)malloc(sizeof(uint32_t) * D);
#pragma omp for schedule(static)
    for (int line = 0; line < nlines; ++line) {
      uint32_t m = 0;
      int last_base = 0;
      for (int s = 0; s < len; ++s) {
        const int k = forward ? s : len - 1 - s;
        const int x = horizontal ? x0 + k : x0 + line;
        const int y = horizontal ? line : k;
        const size_t off = ((size_t)y * W + x) * D;
        const uint8_t* c = cost + off;
        if (s == 0) {
          m = 0xFFFFFFFFu;
          for (int d = 0; d < D; ++d) { Lq[d] = c[d]; m = umin(m, Lq[d]); }
          for (int d = 0; d < D; ++d) out[off + d] = (uint8_t)Lq[d];
          last_base = horizontal ? init[(size_t)y * W + x] : init[x]; /* vertical: row 0 */
          continue;
        }
        const int base = init[(size_t)y * W + x];
        if (base == ORC_INVALID_SHORT) { m = ORC_INVALID_COST; continue; }
        const int div = abs(last_base - base + 1);
        const int32_t q = div ? p2 / div : p2_div0;
        const uint32_t l4 = m + (uint32_t)(p1 > q ? p1 : q);
        uint32_t mn = 0xFFFFFFFFu;
        for (int d = 0; d < D; ++d) {
          const int i1 = d + base - 1 - last_base;
          const int i2 = d + base + 1 - last_base;
          const uint32_t a = (i1 >= 0 && i1 < ORC_LEVEL_RANGE) ? Lq[i1] + (uint32_t)p1 : ORC_INVALID_COST;
          const uint32_t b = (i2 >= 0 && i2 < ORC_LEVEL_RANGE) ? Lq[i2] + (uint32_t)p1 : ORC_INVALID_COST;
          const uint32_t t = umin(umin(umin(Lq[d], a), b), l4);
          Lp[d] = (uint32_t)c[d] + (t - m);
          mn = umin(mn, Lp[d]);
        }
        for (int d = 0; d < D; ++d) { Lq[d] = Lp[d]; out[off + d] = (uint8_t)Lp[d]; }
        m = mn;
        last_base = base;
      }
    }
    free(Lq);
    free(Lp);
  }
}

/* Parabola through (d-1, c1), (d, c0), (d+1, c2), as written at cusgm_ca.cu:150-154. */
static inline float subpix_bias(float c1, float c0, float c2) {
  float den = c1 + c2 - 2.0f * c0;
  if (den < 1.0f) den = 1.0f;
  return (c1 - c2 + den) / (2.0f * den);
}

/* y: image row (the measured reference rule depends on its parity). */
static int pick_tie(const uint32_t* S, int D, uint32_t m, int rule, int y) {
  int best = -1;
  if (rule == ORC_TIE_REF_B200) {
    /* Warpfor64 (cusgm_ca.cu:3666-3675): lanes t with S(t)==m store t, lanes with only
     * S(t+32)==m store t+32; within one store the lowest lane wins; the later of the two
     * stores wins, and the compiled order differs between the two rows of a WTA block:
     * on even rows the t+32 store is later, on odd rows the t store. Other D: lowest d. */
    if (D != 64) rule = ORC_TIE_LOWEST;
    else {
      int a = -1, b = -1;
      for (int t = 0; t < 32; ++t) {
        if (S[t] == m) { if (a < 0) a = t; }
        else if (S[t + 32] == m) { if (b < 0) b = t + 32; }
      }
      if (y % 2 == 0) return b >= 0 ? b : a;
      return a >= 0 ? a : b;
    }
  }
  switch (rule) {
    case ORC_TIE_HIGHEST:
      for (int d = D - 1; d >= 0; --d) if (S[d] == m) return d;
      break;
    case ORC_TIE_LANE_HIGH:
    case ORC_TIE_LANE_LOW: {
      const int per = D / 32 > 0 ? D / 32 : 1;
      const int lanes = D < 32 ? D : 32;
      for (int i = 0; i < lanes; ++i) {
        const int lane = rule == ORC_TIE_LANE_HIGH ? lanes - 1 - i : i;
        for (int j = 0; j < per; ++j)
          if (S[lane + 32 * j] == m) return lane + 32 * j;
      }
      break;
    }
    default:
      for (int d = 0; d < D; ++d) if (S[d] == m) return d;
  }
  return best;
}

/* Plain WTA + uniqueness + subpixel. cusgm_ca.cu:3514-3699 (D=32/64), :3701-3809 (D=128),
 * generic :3149-3232; launches :4139-4165.
 *   rows: D in {32,64,128} launch floor(H/2)*2 rows, other D all rows; x from x0;
 *   pixels never written (x < x0, last row when H is odd) are INVALID here;
 *   x<5, y<5, x>W-5, y>H-5 -> INVALID;
 *   d* <= 0 or d* >= D (generic: d* >= D-1) -> INVALID;
 *   c3 at d* = D-1 reads the slot that holds the winning index, i.e. the value D-1;
 *   min(c1-c2, c3-c2) <= c2*(1-u) -> INVALID; else d* + min_d + bias. */
/* With a region of interest (columns [x0, x1), rows [y0, y1)) the launch covers the region's
 * columns and floor((y1-y0)/2)*2 rows from y0 (cusgm_ca.cu:4139-4165 with roi_x/roi_y/roi_w/roi_h);
 * the border test stays in image coordinates, and the measured tie rule's row parity is the row's
 * position in its two-row block, i.e. y - y0. Everything outside is INVALID. */
static void wta_plain_region(const uint8_t* const paths[4], int W, int H, int x0, int x1, int y0, int y1, int min_d,
                             int D, float uniqueness, int tie_rule, float* disp) {
  const int warp_kernel = (D == 32 || D == 64 || D == 128);
  const int rows = warp_kernel ? ((y1 - y0) / 2) * 2 : (y1 - y0);
  const float ut = 1.0f - uniqueness;
#pragma omp parallel num_threads(nthreads())
  {
    uint32_t* S = (uint32_t*)malloc(sizeof(uint32_t) * D);
#pragma omp for schedule(static)
    for (int y = 0; y < H; ++y) {
      for (int x = 0; x < W; ++x) {
        float* out = disp + (size_t)y * W + x;
        *out = ORC_INVALID_FLOAT;
        if (y < y0 || y >= y0 + rows || x < x0 || x >= x1) continue;
        if (x > W - 5 || y > H - 5 || x < 5 || y < 5) continue;
        const size_t off = ((size_t)y * W + x) * D;
        uint32_t m = 0xFFFFFFFFu;
        for (int d = 0; d < D; ++d) {
          S[d] = (uint32_t)paths[0][off + d] + paths[1][off + d] + paths[2][off + d] + paths[3][off + d];
          m = umin(m, S[d]);
        }
        const int ds = pick_tie(S, D, m, tie_rule, y - y0);
        if (ds <= 0 || ds >= (warp_kernel ? D : D - 1)) continue;
        const float c1 = (float)S[ds - 1];
        const float c2 = (float)m;
        const float c3 = (ds + 1 < D) ? (float)S[ds + 1] : (float)ds;
        const float d12 = c1 - c2, d32 = c3 - c2;
        const float uniq = d12 < d32 ? d12 : d32;
        if (uniq <= c2 * ut) continue;
        *out = (float)(ds + min_d) + subpix_bias(c1, c2, c3);
      }
    }
    free(S);
  }
}

void orc_wta_plain(const uint8_t* const paths[4], int W, int H, int x0, int min_d, int D, float uniqueness,
                   int tie_rule, float* disp) {
  wta_plain_region(paths, W, H, x0, W, 0, H, min_d, D, uniqueness, tie_rule, disp);
}

/* Output of one winning candidate d at an init-disparity level (cusgm_ca.cu:3488-3509). */
static float init_candidate(const uint32_t* S, int D, int ds, int base, float ut) {
  if (ds <= 1 || ds >= D - 1) return ORC_INVALID_FLOAT;
  const float c1 = (float)S[ds - 1];
  const float c2 = (float)S[ds];
  const float c3 = (float)S[ds + 1];
  const float d12 = c1 - c2, d32 = c3 - c2;
  const float uniq = d12 < d32 ? d12 : d32;
  if (uniq <= c2 * ut) return ORC_INVALID_FLOAT;
  return (float)(ds + base) + subpix_bias(c1, c2, c3);
}

/* WTA at init-disparity levels. cusgm_ca.cu:3425-3512 (launched with 4 lines, :4073-4077).
 *   rows [0, floor(H/4)*4); d* <= 1 or d* >= D-1 -> INVALID; base INVALID -> INVALID;
 *   disp = d* + base + bias (min_d is not added).
 * In the reference every tied lane writes its own result; tie_rule picks which one. */
void orc_wta_init(const uint8_t* const paths[4], const int16_t* init, int W, int H, int x0, int D,
                  float uniqueness, int tie_rule, float* disp) {
  const int rows = (H / 4) * 4;
  const float ut = 1.0f - uniqueness;
#pragma omp parallel num_threads(nthreads())
  {
    uint32_t* S = (uint32_t*)malloc(sizeof(uint32_t) * D);
#pragma omp for schedule(static)
    for (int y = 0; y < H; ++y) {
      for (int x = 0; x < W; ++x) {
        float* out = disp + (size_t)y * W + x;
        *out = ORC_INVALID_FLOAT;
        if (y >= rows || x < x0) continue;
        if (x > W - 5 || y > H - 5 || x < 5 || y < 5) continue;
        const int base = init[(size_t)y * W + x];
        if (base == ORC_INVALID_SHORT) continue;
        const size_t off = ((size_t)y * W + x) * D;
        uint32_t m = 0xFFFFFFFFu;
        for (int d = 0; d < D; ++d) {
          S[d] = (uint32_t)paths[0][off + d] + paths[1][off + d] + paths[2][off + d] + paths[3][off + d];
          m = umin(m, S[d]);
        }
        if (tie_rule == ORC_TIE_REF_B200) {
          /* every tied lane stores its own result (cusgm_ca.cu:3488-3509); measured on a B200:
           * a valid disparity wins over INVALID, and the lowest lane wins among valid ones */
          for (int d = 0; d < D; ++d) {
            if (S[d] != m) continue;
            const float v = init_candidate(S, D, d, base, ut);
            if (v != ORC_INVALID_FLOAT) { *out = v; break; }
          }
          continue;
        }
        const int ds = pick_tie(S, D, m, tie_rule, y);
        *out = init_candidate(S, D, ds, base, ut);
        continue;
      }
    }
    free(S);
  }
}

/* Left-right consistency. cusgm_ca.cu:3873-3898 (launch :4345-4347).
 * xr = round-half-away(x - dL) (computed in double as in the reference);
 * out of range -> dL = INVALID; |dL - dR| > thr -> dL = dR[xr] = INVALID, else dL = (dL+dR)/2.
 * The reference reads dR while other threads invalidate it and also reads x == W;
 * here dR is read from a snapshot and x ranges over [0, W). disp_r_out may be NULL. */
void orc_lr_check(float* disp_l, const float* disp_r_snapshot, float* disp_r_out, int W, int H, float threshold) {
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 0; y < H; ++y) {
    float* l = disp_l + (size_t)y * W;
    const float* r = disp_r_snapshot + (size_t)y * W;
    float* ro = disp_r_out ? disp_r_out + (size_t)y * W : NULL;
    for (int x = 0; x < W; ++x) {
      const float dl = l[x];
      if (dl == ORC_INVALID_FLOAT) continue;
      const float xrf = (float)x - dl;
      const int xr = (xrf > 0) ? (int)((double)xrf + 0.5) : (int)((double)xrf - 0.5);
      if (xr < 0 || xr >= W) { l[x] = ORC_INVALID_FLOAT; continue; }
      const float dr = r[xr];
      if (fabsf(dl - dr) > threshold) {
        l[x] = ORC_INVALID_FLOAT;
        if (ro) ro[xr] = ORC_INVALID_FLOAT;
      } else {
        l[x] = (dl + dr) / 2.0f;
      }
    }
  }
}

static inline float median9(float* v) {
  /* insertion sort of 9 values; for non-NaN inputs the middle element equals the
   * result of the reference's compare-exchange network (cusgm_df.cu:48-71) */
  for (int i = 1; i < 9; ++i) {
    float t = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > t) { v[j + 1] = v[j]; --j; }
    v[j + 1] = t;
  }
  return v[4];
}

/* 3x3 median. cusgm_df.cu:16-75, launched :346-355 with a grid whose y extent is
 * derived from the WIDTH: rows 1..min(H-2, 2*ceil((W-2)/2)) and columns 1..W-2 are
 * filtered; all other pixels keep their input value. The reference filters in place
 * (neighbouring blocks race on the halo); here the input is a snapshot. */
void orc_median3x3(const float* in, float* out, int W, int H) {
  if (out != in) memcpy(out, in, sizeof(float) * (size_t)W * H);
  if (W < 3 || H < 3) return;
  int ylim = 2 * ((W - 2 + 1) / 2);
  if (ylim > H - 2) ylim = H - 2;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 1; y <= ylim; ++y) {
    for (int x = 1; x <= W - 2; ++x) {
      float v[9];
      int k = 0;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) v[k++] = in[(size_t)(y + dy) * W + x + dx];
      out[(size_t)y * W + x] = median9(v);
    }
  }
}

/* Erosion. cusgm_df.cu:165-195: an interior pixel (wth < x < W-wth, wth < y < H-wth) whose
 * window holds an INVALID value becomes INVALID; every other pixel is copied. */
void orc_erosion(const float* in, float* out, int W, int H, int wnd) {
  const int wth = (wnd - 1) / 2;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      const float v = in[(size_t)y * W + x];
      float mn = v;
      if (x > wth && x < W - wth && y > wth && y < H - wth) {
        for (int dx = -wth; dx <= wth; ++dx)
          for (int dy = -wth; dy <= wth; ++dy) {
            const float u = in[(size_t)(y + dy) * W + x + dx];
            if (u < mn) mn = u;
          }
      }
      out[(size_t)y * W + x] = mn == ORC_INVALID_FLOAT ? mn : v;
    }
  }
}

/* Range-limited Gaussian smoothing. cusgm_df.cu:93-121 (sigma_d 1.5, sigma_r 2.0 at :294):
 * over a (2*ceil(2 sd)+1)^2 window (columns outer, rows inner), valid neighbours within sr of a
 * valid centre weigh expf(-(dx^2+dy^2)/(2 sd^2)); INVALID when no weight. */
void orc_gauss(const float* in, float* out, int W, int H, float sigma_d, float sigma_r) {
  const int r = (int)ceil(2.0 * sigma_d);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      float result = ORC_INVALID_FLOAT, sum = 0.0f, sum_w = 0.0f;
      const float c = in[(size_t)y * W + x];
      if (c != ORC_INVALID_FLOAT) {
        for (int m = x - r; m <= x + r; ++m)
          for (int n = y - r; n <= y + r; ++n)
            if (m >= 0 && n >= 0 && m < W && n < H) {
              const float v = in[(size_t)n * W + m];
              if (v != ORC_INVALID_FLOAT && fabsf(c - v) < sigma_r) {
                const int dx = m - x, dy = n - y;
                const float w = expf(-((float)(dx * dx + dy * dy) / (2.0f * sigma_d * sigma_d)));
                sum_w += w;
                sum = fmaf(w, v, sum);
              }
            }
      }
      if (sum_w > 0.0f) result = sum / sum_w;
      out[(size_t)y * W + x] = result;
    }
  }
}

/* Bilateral smoothing guided by the left image. cusgm_df.cu:123-162 (sigma_d 2.5, sigma_r 10.0
 * at :298): spatial weight times exp(-g^2/(2 sr^2)) of the grey difference g (in double) for
 * valid neighbours with |g| < sr. */
void orc_bilateral(const uint8_t* img, const float* in, float* out, int W, int H, float sigma_d, float sigma_r) {
  const int r = (int)ceil(2.0 * sigma_d);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      float result = ORC_INVALID_FLOAT, sum = 0.0f, sum_w = 0.0f;
      const float c = in[(size_t)y * W + x];
      const int gc = img[(size_t)y * W + x];
      if (c != ORC_INVALID_FLOAT) {
        for (int m = x - r; m <= x + r; ++m)
          for (int n = y - r; n <= y + r; ++n)
            if (m >= 0 && n >= 0 && m < W && n < H) {
              const float v = in[(size_t)n * W + m];
              const int g = img[(size_t)n * W + m];
              if (v != ORC_INVALID_FLOAT && fabsf((float)(g - gc)) < sigma_r) {
                const int dx = m - x, dy = n - y;
                const float dist = (float)(g - gc);
                const float wd = expf(-((float)(dx * dx + dy * dy) / (2.0f * sigma_d * sigma_d)));
                const float wr = (float)exp(-(double)(dist * dist) / (2.0 * sigma_r * sigma_r));
                const float w = wd * wr;
                sum_w += w;
                sum = fmaf(w, v, sum);
              }
            }
        if (sum_w > 0.0f) result = sum / sum_w;
      }
      out[(size_t)y * W + x] = result;
    }
  }
}

/* Dilation of INVALID pixels. cusgm_df.cu:197-222; window size rule :302-303.
 * An INVALID (or -32768) pixel with wth < x < W-wth and wth < y < H-wth takes the max
 * over its window; every other pixel is copied. */
void orc_dilation(const float* in, float* out, int W, int H, int wnd) {
  const int wth = (wnd - 1) / 2;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      float v = in[(size_t)y * W + x];
      if (v == ORC_INVALID_FLOAT || v == (float)ORC_INVALID_SHORT) {
        if (x > wth && x < W - wth && y > wth && y < H - wth) {
          for (int dx = -wth; dx <= wth; ++dx)
            for (int dy = -wth; dy <= wth; ++dy) {
              const float u = in[(size_t)(y + dy) * W + x + dx];
              if (u > v) v = u;
            }
        }
      }
      out[(size_t)y * W + x] = v;
    }
  }
}

static inline int peaks_adjacent(float a, float b, int abs_mode) {
  if (abs_mode == ORC_PEAKS_ABS_FLOAT) return fabsf(a - b) <= 1.0f;
  return abs((int)(a - b)) <= 1;
}

/* Small-region ("peaks") removal on one strip. StereoCudaImpl.cpp:32-97.
 * 4-connected regions of valid pixels whose neighbours differ by at most 1 (see
 * peaks_adjacent); regions smaller than threshold become INVALID. Returns the count. */
static int remove_peaks_strip(float* disp, int w, int h, int threshold, int abs_mode, int32_t* label,
                              int32_t* queue) {
  int peaks = 0;
  for (int i = 0; i < w * h; ++i) label[i] = 0;
  int next_label = 0;
  for (int seed = 0; seed < w * h; ++seed) {
    if (disp[seed] == ORC_INVALID_FLOAT || label[seed] != 0) continue;
    ++next_label;
    int qh = 0, qt = 0;
    queue[qt++] = seed;
    label[seed] = next_label;
    while (qh < qt) {
      const int p = queue[qh++];
      const int py = p / w, px = p - py * w;
      const float base = disp[p];
      static const int oy[4] = {-1, 0, 0, 1}, ox[4] = {0, -1, 1, 0};
      for (int n = 0; n < 4; ++n) {
        const int ny = py + oy[n], nx = px + ox[n];
        if (ny < 0 || ny >= h || nx < 0 || nx >= w) continue;
        const int q = ny * w + nx;
        if (label[q] != 0) continue;
        const float s = disp[q];
        if (s == ORC_INVALID_FLOAT) continue;
        if (peaks_adjacent(s, base, abs_mode)) { label[q] = next_label; queue[qt++] = q; }
      }
    }
    if (qt < threshold) {
      for (int k = 0; k < qt; ++k) disp[queue[k]] = ORC_INVALID_FLOAT;
      peaks += qt;
    }
  }
  return peaks;
}

/* One strip with an explicit threshold (the reference's RemovePeaks, StereoCudaImpl.cpp:32-97). */
int orc_remove_peaks_strip(float* disp, int w, int h, int threshold, int abs_mode) {
  if (w <= 0 || h <= 0) return 0;
  int32_t* label = (int32_t*)malloc(sizeof(int32_t) * (size_t)w * h);
  int32_t* queue = (int32_t*)malloc(sizeof(int32_t) * (size_t)w * h);
  const int n = remove_peaks_strip(disp, w, h, threshold, abs_mode, label, queue);
  free(label);
  free(queue);
  return n;
}

/* Strip partition and thresholds as in StereoCudaImpl.cpp:463-498 (no ROI):
 * rm_tiles = floor(H / strips); strip i covers rows [i*rm_tiles, (i+1)*rm_tiles);
 * rows at and below strips*rm_tiles are not processed;
 * threshold = (int)((float)(W*h_strip) * ratio). */
/* With a region of interest the strips cover the region's rows: rm_tiles = floor(roi_h / strips),
 * strip i rows [roi_y + i*rm_tiles, min(H, roi_y + (i+1)*rm_tiles)) (StereoCudaImpl.cpp:463-498). */
static int remove_peaks_rows(float* disp, int W, int H, int y_off, int rows_h, int strips, float ratio,
                             int abs_mode) {
  if (strips <= 0) return 0;
  const int tiles = rows_h / strips;
  if (tiles <= 0) return 0;
  int total = 0;
#pragma omp parallel num_threads(nthreads()) reduction(+ : total)
  {
    int32_t* label = (int32_t*)malloc(sizeof(int32_t) * (size_t)W * tiles);
    int32_t* queue = (int32_t*)malloc(sizeof(int32_t) * (size_t)W * tiles);
#pragma omp for schedule(dynamic, 1)
    for (int i = 0; i < strips; ++i) {
      const int start = imax(0, y_off + i * tiles);
      const int end = imin(H, y_off + (i + 1) * tiles);
      if (end <= start) continue;
      const int h = end - start;
      const int threshold = (int)((float)(W * h) * ratio);
      total += remove_peaks_strip(disp + (size_t)start * W, W, h, threshold, abs_mode, label, queue);
    }
    free(label);
    free(queue);
  }
  return total;
}

int orc_remove_peaks(float* disp, int W, int H, int strips, float ratio, int abs_mode) {
  return remove_peaks_rows(disp, W, H, 0, H, strips, ratio, abs_mode);
}

/* Even-sample decimation by 2. FasterStereoCuda.cpp:114-136. */
void orc_zoom_half(const uint8_t* src, int w_src, int h_src, uint8_t* dst) {
  const int wd = w_src / 2, hd = h_src / 2;
  for (int y = 0; y < hd; ++y)
    for (int x = 0; x < wd; ++x) dst[(size_t)y * wd + x] = src[(size_t)(2 * y) * w_src + 2 * x];
}

/* Initial disparity of the next finer level. FasterStereoCuda.cpp:138-166.
 * Even rows (except the last row): (short)(2*d - 16) from cur at flat index
 * (y/2)*(width/2) + x/2, INVALID -> -32768; odd rows and the last row copy the row above.
 * With an odd `width` the flat index runs into the next row of `cur`; at the very end it
 * runs past the buffer, which the oracle reads as INVALID. */
void orc_init_next_level(const float* cur, int w_cur, int h_cur, int16_t* next, int width, int height) {
  const int half = ORC_LEVEL_RANGE >> 1;
  const int wid2 = width >> 1;
  const long ncur = (long)w_cur * h_cur;
  for (int i = 0; i < height; ++i) {
    int16_t* row = next + (size_t)i * width;
    for (int j = 0; j < width; ++j) {
      if (i % 2 == 1 || i == height - 1) {
        row[j] = i > 0 ? next[(size_t)(i - 1) * width + j] : (int16_t)ORC_INVALID_SHORT;
      } else {
        const long idx = (long)(i >> 1) * wid2 + (j >> 1);
        const float d = idx < ncur ? cur[idx] : ORC_INVALID_FLOAT;
        row[j] = d != ORC_INVALID_FLOAT ? (int16_t)(2.0f * d - (float)half) : (int16_t)ORC_INVALID_SHORT;
      }
    }
  }
}

/* Right-view initial disparities for LR checking at an init level.
 * cusgm_util.cu:47-59 then a 5x5 int16 dilation (StereoCudaImpl.cpp:375-381).
 * The reference scatters concurrently; here every target is cleared first and the
 * scatter runs in increasing x, so the largest source x wins. */
static void right_init(const int16_t* init_l, int16_t* init_r, int W, int H) {
  int16_t* tmp = (int16_t*)malloc(sizeof(int16_t) * (size_t)W * H);
  const int half = ORC_LEVEL_RANGE >> 1;
  for (int y = 0; y < H; ++y) {
    int16_t* r = tmp + (size_t)y * W;
    const int16_t* l = init_l + (size_t)y * W;
    for (int x = 0; x < W; ++x) r[x] = ORC_INVALID_SHORT;
    for (int x = 0; x < W; ++x) {
      const int16_t xl = (int16_t)x;
      const int16_t il = (int16_t)(l[x] + half);
      const int t = xl - il;
      if (t > 0 && t < W) r[t] = (int16_t)(il - half);
    }
  }
  const int wth = 2;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      int16_t v = tmp[(size_t)y * W + x];
      if (v == ORC_INVALID_SHORT && x > wth && x < W - wth && y > wth && y < H - wth) {
        for (int dx = -wth; dx <= wth; ++dx)
          for (int dy = -wth; dy <= wth; ++dy) {
            const int16_t u = tmp[(size_t)(y + dy) * W + x + dx];
            if (u > v) v = u;
          }
      }
      init_r[(size_t)y * W + x] = v;
    }
  free(tmp);
}

/* Region of one view: columns [x0, x1), rows [y0, y1), and the origin of the cost kernel's
 * D-pixel blocks. Without an ROI: columns from max(0, min_disp), every row (cusgm_ca.cu:3991-3999).
 * With an ROI: its rectangle, columns clipped to start at max(0, min_disp) (the left view's cost,
 * computed without the ROI, covers only those, StereoCudaImpl.cpp:403). */
typedef struct { int x0, x1, y0, y1, bx; } orc_region_t;

static orc_region_t view_region(const orc_config_t* c, int left_view) {
  const int xmin = imax(0, c->min_disp);
  orc_region_t r = {xmin, c->width, 0, c->height, xmin};
  const int en = left_view ? c->roi_l_enable : c->roi_r_enable;
  if (en) {
    const int rx = left_view ? c->roi_l_x : c->roi_r_x, ry = left_view ? c->roi_l_y : c->roi_r_y;
    const int rw = left_view ? c->roi_l_w : c->roi_r_w, rh = left_view ? c->roi_l_h : c->roi_r_h;
    r.x0 = imax(rx, xmin);
    r.x1 = rx + rw;
    r.y0 = ry;
    r.y1 = ry + rh;
    r.bx = rx;
  }
  return r;
}

static int roi_ok(int en, int x, int y, int w, int h, int W, int H) {
  return !en || (x >= 0 && y >= 0 && w > 0 && h > 0 && x + w <= W && y + h <= H);
}

static int run_view(const orc_config_t* c, const uint64_t* cl, const uint64_t* cr, const int16_t* init,
                    int left2right, uint8_t* cost, uint8_t* paths, float* wta, uint8_t* cost_dump,
                    uint8_t* paths_dump) {
  const int W = c->width, H = c->height, D = c->disp_range;
  const size_t V = (size_t)W * H * D;
  const int x0 = imax(0, c->min_disp);
  const orc_region_t r = view_region(c, left2right);
  if (init) orc_cost_init(cl, cr, init, W, H, x0, D, c->cs_type, left2right, cost);
  else cost_plain_blocks(cl, cr, W, H, c->min_disp, D, c->cs_type, left2right, r.bx, cost);
  if (cost_dump) memcpy(cost_dump, cost, V);
  const uint8_t* P[4];
  for (int dir = 0; dir < 4; ++dir) {
    uint8_t* out = paths + (size_t)dir * V;
    if (init) orc_path_init(cost, init, W, H, x0, D, c->p1, c->p2, c->p2_div0, dir, out);
    else path_plain_region(cost, W, r.x0, r.x1, r.y0, r.y1, D, c->p1, c->p2, dir, out);
    P[dir] = out;
  }
  if (paths_dump) memcpy(paths_dump, paths, 4 * V);
  if (init) orc_wta_init(P, init, W, H, x0, D, c->uniqueness, c->init_tie_rule, wta);
  else wta_plain_region(P, W, H, r.x0, r.x1, r.y0, r.y1, c->min_disp, D, c->uniqueness, c->tie_rule, wta);
  return 0;
}

/* StereoCuda::Match: StereoCudaImpl.cpp:507-546 (cost :363-416, aggregation :418-446,
 * filter :448-461, D2H then small-region removal :463-498). */
int orc_match_dump(const orc_config_t* c, const uint8_t* left, const uint8_t* right, const int16_t* init,
                   uint64_t* census_l, uint64_t* census_r, uint8_t* cost_lr, uint8_t* paths_lr, float* wta_l,
                   uint8_t* cost_rl, uint8_t* paths_rl, float* wta_r, float* disp_l, float* disp_r) {
  const int W = c->width, H = c->height, D = c->disp_range;
  if (W <= 0 || H <= 0 || D <= 0 || !left || !right || !disp_l) return -1;
  if (!roi_ok(c->roi_l_enable, c->roi_l_x, c->roi_l_y, c->roi_l_w, c->roi_l_h, W, H) ||
      !roi_ok(c->roi_r_enable, c->roi_r_x, c->roi_r_y, c->roi_r_w, c->roi_r_h, W, H))
    return -1;
  if (init && (c->roi_l_enable || c->roi_r_enable)) return -3; /* ROI at initial-disparity levels: not built */
  const size_t N = (size_t)W * H, V = N * D;
  uint64_t* cl = (uint64_t*)malloc(sizeof(uint64_t) * N);
  uint64_t* cr = (uint64_t*)malloc(sizeof(uint64_t) * N);
  uint8_t* cost = (uint8_t*)calloc(V, 1);
  uint8_t* paths = (uint8_t*)calloc(4 * V, 1);
  float* dl = (float*)malloc(sizeof(float) * N);
  float* dr = (float*)malloc(sizeof(float) * N);
  float* tmp = (float*)malloc(sizeof(float) * N);
  int rc = 0;
  if (!cl || !cr || !cost || !paths || !dl || !dr || !tmp) { rc = -2; goto done; }
  orc_census(left, W, H, c->cs_type, 0, cl);
  orc_census(right, W, H, c->cs_type, 1, cr);
  if (census_l) memcpy(census_l, cl, sizeof(uint64_t) * N);
  if (census_r) memcpy(census_r, cr, sizeof(uint64_t) * N);
  run_view(c, cl, cr, init, 1, cost, paths, dl, cost_lr, paths_lr);
  if (wta_l) memcpy(wta_l, dl, sizeof(float) * N);
  for (size_t i = 0; i < N; ++i) dr[i] = ORC_INVALID_FLOAT;
  if (c->do_lr_check) {
    int16_t* init_r = NULL;
    if (init) {
      init_r = (int16_t*)malloc(sizeof(int16_t) * N);
      right_init(init, init_r, W, H);
    }
    /* right view: census roles swapped, same cost buffer (stale 5x5 pixels keep L->R cost) */
    run_view(c, cr, cl, init_r, 0, cost, paths, dr, cost_rl, paths_rl);
    if (wta_r) memcpy(wta_r, dr, sizeof(float) * N);
    memcpy(tmp, dr, sizeof(float) * N);
    orc_lr_check(dl, tmp, dr, W, H, c->lr_threshold);
    free(init_r);
  } else if (wta_r) {
    memcpy(wta_r, dr, sizeof(float) * N);
  }
  if (c->do_median) {
    orc_median3x3(dl, tmp, W, H);
    memcpy(dl, tmp, sizeof(float) * N);
  }
  if (c->post_filter == 1 || c->post_filter == 2) {
    if (c->post_filter == 1) orc_gauss(dl, tmp, W, H, 1.5f, 2.0f);
    else orc_bilateral(left, dl, tmp, W, H, 2.5f, 10.0f);
    memcpy(dl, tmp, sizeof(float) * N);
  }
  {
    /* cusgm_df.cu:301-338: OPEN and CLOSE run both steps from the same input into the same
     * output, leaving the dilation (OPEN) or the erosion (CLOSE) */
    const int mp = c->morphology ? c->morphology : (c->morphology_dilation ? 2 : 0);
    const int op = mp == 3 ? 2 : (mp == 4 ? 1 : mp);
    if (op) {
      const int s = W < H ? W : H;
      const int wnd = s < 360 ? 3 : (s < 720 ? 5 : 7);
      if (op == 2) orc_dilation(dl, tmp, W, H, wnd);
      else orc_erosion(dl, tmp, W, H, wnd);
      memcpy(dl, tmp, sizeof(float) * N);
    }
  }
  if (c->do_remove_peaks) {
    if (c->roi_l_enable)
      remove_peaks_rows(dl, W, H, c->roi_l_y, c->roi_l_h, c->peaks_strips, c->peaks_ratio, c->peaks_abs_mode);
    else
      orc_remove_peaks(dl, W, H, c->peaks_strips, c->peaks_ratio, c->peaks_abs_mode);
  }
  memcpy(disp_l, dl, sizeof(float) * N);
  if (disp_r) memcpy(disp_r, dr, sizeof(float) * N);
done:
  free(cl); free(cr); free(cost); free(paths); free(dl); free(dr); free(tmp);
  return rc;
}

int orc_match(const orc_config_t* cfg, const uint8_t* left, const uint8_t* right, const int16_t* init,
              float* disp_l, float* disp_r) {
  return orc_match_dump(cfg, left, right, init, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, disp_l, disp_r);
}

/* Per-level options and disparity ranges: SetSgmParameters (FasterStereoCuda.cpp:169-199)
 * and the range rules of HierSgmCudaImpl::Init (:229-291). The optional override replaces
 * the hard-coded census type and penalties on every level. */
int orc_pyr_level_config(const orc_pyr_config_t* pc, int level, orc_config_t* o) {
  const int layers = pc->num_layers < 1 ? 1 : pc->num_layers;
  if (level < 0 || level >= layers) return -1;
  memset(o, 0, sizeof(*o));
  const int scale = 1 << level;
  o->width = pc->width / scale;
  o->height = pc->height / scale;
  o->cs_type = pc->override_enable ? pc->cs_type : 0;
  o->p1 = pc->override_enable ? pc->p1 : 8;
  o->p2 = pc->override_enable ? pc->p2 : 32;
  o->uniqueness = level == 0 ? 0.95f : 1.0f;
  o->lr_threshold = 1.0f;
  o->do_median = 1;
  o->post_filter = (level == 0 && pc->do_smooth) ? 1 : 0;
  o->morphology = 0;
  if (layers <= 1) {
    o->do_lr_check = pc->do_lr_check;
    o->do_remove_peaks = pc->do_rm_peaks;
    o->peaks_ratio = 0.0005f;
    o->morphology_dilation = 0;
  } else if (layers <= 2) {
    o->do_lr_check = level == 0 ? 0 : pc->do_lr_check;
    o->do_remove_peaks = level == 0 ? 0 : pc->do_rm_peaks;
    o->peaks_ratio = level == 0 ? 0.0005f : 0.001f;
    o->morphology_dilation = level < layers - 1 ? 0 : 1;
  } else {
    o->do_lr_check = level < layers - 1 ? 0 : pc->do_lr_check;
    o->do_remove_peaks = level < layers - 1 ? 0 : pc->do_rm_peaks;
    o->peaks_ratio = level < layers - 1 ? 0.0005f : 0.005f;
    o->morphology_dilation = level < layers - 1 ? 0 : 1;
  }
  if (level == layers - 1) {
    int dmin = pc->min_disp / scale, dmax = pc->max_disp / scale;
    int range = dmax - dmin;
    int k = 6;
    while ((1 << k) < range) ++k;
    range = 1 << k;
    if (range > 2 * pc->width) range /= 2;
    if (dmin >= pc->width) {
      dmin = pc->width - range;
      if (dmin < -pc->width) dmin = -pc->width;
    }
    o->min_disp = dmin;
    o->disp_range = range;
  } else {
    o->min_disp = 0;
    o->disp_range = ORC_LEVEL_RANGE;
  }
  o->peaks_strips = pc->peaks_strips;
  o->peaks_abs_mode = pc->peaks_abs_mode;
  o->tie_rule = pc->tie_rule;
  o->init_tie_rule = pc->init_tie_rule;
  o->p2_div0 = pc->p2_div0;
  o->threads = pc->threads;
  return 0;
}

/* FasterStereoCuda::Match: HierSgmCudaImpl::Match, FasterStereoCuda.cpp:408-529. */
int orc_pyr_match(const orc_pyr_config_t* pc, const uint8_t* left, const uint8_t* right, float* disp) {
  const int layers = pc->num_layers < 1 ? 1 : pc->num_layers;
  uint8_t* L[16] = {0};
  uint8_t* R[16] = {0};
  int16_t* init[16] = {0};
  float* dl[16] = {0};
  int w[16], h[16];
  if (layers > 16) return -1;
  for (int i = 0; i < layers; ++i) {
    w[i] = pc->width >> i;
    h[i] = pc->height >> i;
    L[i] = (uint8_t*)malloc((size_t)w[i] * h[i] + 1);
    R[i] = (uint8_t*)malloc((size_t)w[i] * h[i] + 1);
    dl[i] = (float*)malloc(sizeof(float) * ((size_t)w[i] * h[i] + 1));
    if (i < layers - 1) init[i] = (int16_t*)malloc(sizeof(int16_t) * ((size_t)w[i] * h[i] + 1));
  }
  memcpy(L[0], left, (size_t)w[0] * h[0]);
  memcpy(R[0], right, (size_t)w[0] * h[0]);
  for (int i = 1; i < layers; ++i) {
    orc_zoom_half(L[i - 1], w[i - 1], h[i - 1], L[i]);
    orc_zoom_half(R[i - 1], w[i - 1], h[i - 1], R[i]);
  }
  int rc = 0;
  for (int n = layers - 1; n >= 0 && rc == 0; --n) {
    orc_config_t c;
    orc_pyr_level_config(pc, n, &c);
    rc = orc_match(&c, L[n], R[n], init[n], n > 0 ? dl[n] : disp, NULL);
    if (n > 0) orc_init_next_level(dl[n], w[n], h[n], init[n - 1], w[n - 1], h[n - 1]);
  }
  for (int i = 0; i < layers; ++i) { free(L[i]); free(R[i]); free(dl[i]); free(init[i]); }
  return rc;
}
