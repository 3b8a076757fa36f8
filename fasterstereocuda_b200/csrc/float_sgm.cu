// Differentiable float32 SGM: 4-path hard-min recurrence with per-pixel P1/P2 maps, summed over the
// paths, followed by a soft-argmin disparity; and its adjoint.
//
// No counterpart in the reference (it is the training/serving addition beside the bit-exact path).
// The recurrence is the reference's path recurrence (cusgm_ca.cu:1517-1564) in float with the
// penalties read at the current pixel and +inf beyond d = 0 and d = D-1:
//   L_p(d) = C_p(d) + min(L_q(d), L_q(d-1)+P1(p), L_q(d+1)+P1(p), m_q+P2(p)) - m_q,  m_q = min_k L_q(k)
//   S(p,d) = sum over the four paths;  disp(p) = sum_d d * softmax_d(-S(p,d)/T)
// Ties of the hard minima are broken in the fixed order same d, d-1, d+1, jump (lowest k for m_q).
//
// Backward: per path, scanlines are walked backwards segment by segment; each segment of
// kSeg pixels is recomputed from the state stored when the forward pass entered it, so no
// D-deep path volume is kept (only one state per kSeg pixels). The adjoint routes the gradient
// of every L_p(d) to C_p(d), to P1(p) or P2(p) through the recorded minimum, and to L_q.
//
// Layouts: cost/sum/grad volumes float [B][H][W][D]; maps float [B][H][W]; checkpoints float
// [4 paths][lines][segments][D]. Paths: 0 top->bottom, 1 left->right, 2 bottom->top, 3 right->left.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/sgm_b200.h"

void sgm_set_process_error(const char* msg);

namespace {

constexpr unsigned kFullMask = 0xFFFFFFFFu;
constexpr int kSeg = 16;
#define kInf __int_as_float(0x7f800000)

struct Geo {
  int B, H, W, D;
  int dir;
  int lines, len, nseg;
};

__host__ __device__ inline Geo make_geo(int B, int H, int W, int D, int dir) {
  Geo g;
  g.B = B; g.H = H; g.W = W; g.D = D; g.dir = dir;
  const bool horiz = dir == 1 || dir == 3;
  g.lines = horiz ? B * H : B * W;
  g.len = horiz ? W : H;
  g.nseg = (g.len + kSeg - 1) / kSeg;
  return g;
}

// pixel index (b*H + y)*W + x of scan position s on line `line`
__device__ __forceinline__ size_t pix(const Geo& g, int line, int s) {
  const bool fwd = g.dir == 0 || g.dir == 1;
  const int k = fwd ? s : g.len - 1 - s;
  if (g.dir == 1 || g.dir == 3) return (size_t)line * g.W + k;  // line = b*H + y
  const int b = line / g.W, x = line - b * g.W;
  return ((size_t)b * g.H + k) * g.W + x;
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(kFullMask, v, o));
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
  return v;
}

// lane holds d = lane*K + j
template <int K>
__device__ __forceinline__ void neighbours(const float (&L)[K], int lane, float (&lm)[K], float (&lp)[K]) {
  const float left = __shfl_up_sync(kFullMask, L[K - 1], 1);
  const float right = __shfl_down_sync(kFullMask, L[0], 1);
#pragma unroll
  for (int j = 0; j < K; ++j) {
    lm[j] = j > 0 ? L[j - 1] : (lane > 0 ? left : kInf);
    lp[j] = j < K - 1 ? L[j + 1] : (lane < 31 ? right : kInf);
  }
}

// One forward step: returns the new minimum. ch receives 0 same, 1 d-1, 2 d+1, 3 jump.
template <int K>
__device__ __forceinline__ float fstep(float (&L)[K], const float (&c)[K], float m, float p1, float p2, int lane,
                                       int (&ch)[K]) {
  float lm[K], lp[K];
  neighbours<K>(L, lane, lm, lp);
  const float jump = m + p2;
  float mn = kInf;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    float t = L[j];
    int k = 0;
    const float a = lm[j] + p1, b = lp[j] + p1;
    if (a < t) { t = a; k = 1; }
    if (b < t) { t = b; k = 2; }
    if (jump < t) { t = jump; k = 3; }
    ch[j] = k;
    L[j] = c[j] + t - m;
    mn = fminf(mn, L[j]);
  }
  return warp_min(mn);
}

// Inputs of the next kPF pixels are loaded ahead in a register ring (each line owns its pixels, so
// the running sum can be read ahead of the stores of earlier pixels).
constexpr int kPF = 4;

template <int K>
__global__ void __launch_bounds__(256) k_float_fwd(const float* __restrict__ cost, const float* __restrict__ p1m,
                                                   const float* __restrict__ p2m, float* __restrict__ sum,
                                                   float* __restrict__ ckpt, Geo g, int first) {
  const int line = blockIdx.x * blockDim.y + threadIdx.y;
  const int lane = threadIdx.x;
  if (line >= g.lines) return;
  const int D = 32 * K;
  float* ck = ckpt + (size_t)line * g.nseg * D;
  float L[K];
  int ch[K];
  float m = 0.f;
  float rc[kPF][K], rs[kPF][K], rp1[kPF], rp2[kPF];
  auto fetch = [&](int j, int s) {
    const size_t p = pix(g, line, s);
#pragma unroll
    for (int i = 0; i < K; ++i) {
      rc[j][i] = cost[p * D + lane * K + i];
      rs[j][i] = first ? 0.f : sum[p * D + lane * K + i];
    }
    rp1[j] = p1m[p];
    rp2[j] = p2m[p];
  };
#pragma unroll
  for (int j = 0; j < kPF; ++j)
    if (j < g.len) fetch(j, j);
  for (int s0 = 0; s0 < g.len; s0 += kPF) {
#pragma unroll
    for (int j = 0; j < kPF; ++j) {
      const int s = s0 + j;
      if (s < g.len) {
        const size_t p = pix(g, line, s);
        float c[K], old[K];
#pragma unroll
        for (int i = 0; i < K; ++i) { c[i] = rc[j][i]; old[i] = rs[j][i]; }
        const float P1 = rp1[j], P2 = rp2[j];
        if (s + kPF < g.len) fetch(j, s + kPF);
        if (s % kSeg == 0 && s > 0) {  // state entering this segment
#pragma unroll
          for (int i = 0; i < K; ++i) ck[(size_t)(s / kSeg) * D + lane * K + i] = L[i];
        }
        if (s == 0) {
          float mn = kInf;
#pragma unroll
          for (int i = 0; i < K; ++i) { L[i] = c[i]; mn = fminf(mn, c[i]); }
          m = warp_min(mn);
        } else {
          m = fstep<K>(L, c, m, P1, P2, lane, ch);
        }
        float* sp = sum + p * D + lane * K;
#pragma unroll
        for (int i = 0; i < K; ++i) sp[i] = first ? L[i] : old[i] + L[i];
      }
    }
  }
}

// disp = sum_d d softmax(-S/T); dS = -gdisp/T * w(d) * (d - disp) when gdisp is given
template <int K>
__global__ void __launch_bounds__(256) k_soft_argmin(const float* __restrict__ sum, float* __restrict__ disp,
                                                     const float* __restrict__ gdisp, float* __restrict__ gsum,
                                                     size_t npix, float inv_t) {
  const size_t p = (size_t)blockIdx.x * blockDim.y + threadIdx.y;
  const int lane = threadIdx.x;
  if (p >= npix) return;
  const int D = 32 * K;
  const float* sp = sum + p * D + lane * K;
  float S[K], mn = kInf;
#pragma unroll
  for (int j = 0; j < K; ++j) { S[j] = sp[j]; mn = fminf(mn, S[j]); }
  mn = warp_min(mn);
  float e[K], z = 0.f, num = 0.f;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    e[j] = expf(-(S[j] - mn) * inv_t);
    z += e[j];
    num += e[j] * (float)(lane * K + j);
  }
  z = warp_sum(z);
  num = warp_sum(num);
  const float d = num / z;
  if (!gdisp) {
    if (lane == 0) disp[p] = d;
    return;
  }
  const float gd = gdisp[p];
  float* gp = gsum + p * D + lane * K;
#pragma unroll
  for (int j = 0; j < K; ++j) gp[j] = -gd * inv_t * (e[j] / z) * ((float)(lane * K + j) - d);
}

template <int K>
__global__ void __launch_bounds__(128) k_float_bwd(const float* __restrict__ cost, const float* __restrict__ p1m,
                                                   const float* __restrict__ p2m, const float* __restrict__ ckpt,
                                                   const float* __restrict__ gsum, float* __restrict__ gcost,
                                                   float* __restrict__ gp1, float* __restrict__ gp2, Geo g,
                                                   int first) {
  const int D = 32 * K;
  extern __shared__ float seg_smem[];
  const int line = blockIdx.x * blockDim.y + threadIdx.y;
  const int lane = threadIdx.x;
  if (line >= g.lines) return;
  // per warp: (kSeg + 1) states of D floats; slot 0 = state entering the segment
  float* st = seg_smem + (size_t)threadIdx.y * (kSeg + 1) * D;
  const float* ck = ckpt + (size_t)line * g.nseg * D;
  float gnext[K];
#pragma unroll
  for (int j = 0; j < K; ++j) gnext[j] = 0.f;
  for (int k = g.nseg - 1; k >= 0; --k) {
    const int s0 = k * kSeg, s1 = min(g.len, s0 + kSeg);
    // recompute the segment: st[1 + (s - s0)] = L(s)
    float L[K], c[K];
    int ch[K];
    float m = 0.f;
    if (k > 0) {
#pragma unroll
      for (int j = 0; j < K; ++j) {
        L[j] = ck[(size_t)k * D + lane * K + j];
        st[lane * K + j] = L[j];
      }
      float mn = kInf;
#pragma unroll
      for (int j = 0; j < K; ++j) mn = fminf(mn, L[j]);
      m = warp_min(mn);
    }
    {
      // inputs of the segment's pixels through a kPF-deep register ring
      float rc[kPF][K], rp1[kPF], rp2[kPF];
      auto fetch = [&](int j, int s) {
        const size_t p = pix(g, line, s);
#pragma unroll
        for (int i = 0; i < K; ++i) rc[j][i] = cost[p * D + lane * K + i];
        rp1[j] = p1m[p];
        rp2[j] = p2m[p];
      };
#pragma unroll
      for (int j = 0; j < kPF; ++j)
        if (s0 + j < s1) fetch(j, s0 + j);
      for (int b = s0; b < s1; b += kPF) {
#pragma unroll
        for (int j = 0; j < kPF; ++j) {
          const int s = b + j;
          if (s < s1) {
#pragma unroll
            for (int i = 0; i < K; ++i) c[i] = rc[j][i];
            const float P1 = rp1[j], P2 = rp2[j];
            if (s + kPF < s1) fetch(j, s + kPF);
            if (s == 0) {
              float mn = kInf;
#pragma unroll
              for (int i = 0; i < K; ++i) { L[i] = c[i]; mn = fminf(mn, c[i]); }
              m = warp_min(mn);
            } else {
              m = fstep<K>(L, c, m, P1, P2, lane, ch);
            }
#pragma unroll
            for (int i = 0; i < K; ++i) st[(size_t)(1 + s - s0) * D + lane * K + i] = L[i];
          }
        }
      }
    }
    __syncwarp();
    // adjoint through the segment, last pixel first; its inputs through a register ring
    float rg[kPF][K], rgc[kPF][K], rq1[kPF], rq2[kPF];
    auto fetch_b = [&](int j, int s) {
      const size_t p = pix(g, line, s);
#pragma unroll
      for (int i = 0; i < K; ++i) {
        rg[j][i] = gsum[p * D + lane * K + i];
        rgc[j][i] = first ? 0.f : gcost[p * D + lane * K + i];
      }
      rq1[j] = p1m[p];
      rq2[j] = p2m[p];
    };
#pragma unroll
    for (int j = 0; j < kPF; ++j)
      if (s1 - 1 - j >= s0) fetch_b(j, s1 - 1 - j);
    for (int b = s1 - 1; b >= s0; b -= kPF)
#pragma unroll
    for (int jj = 0; jj < kPF; ++jj) {
      const int s = b - jj;
      if (s < s0) break;
      const size_t p = pix(g, line, s);
      float gl[K], gco[K];
#pragma unroll
      for (int j = 0; j < K; ++j) { gl[j] = rg[jj][j] + gnext[j]; gco[j] = rgc[jj][j]; }
      const float P1 = rq1[jj], P2 = rq2[jj];
      if (s - kPF >= s0) fetch_b(jj, s - kPF);
      float* gc = gcost + p * D + lane * K;
#pragma unroll
      for (int j = 0; j < K; ++j) gc[j] = first ? gl[j] : gco[j] + gl[j];
      if (s == 0) break;
      // previous state L_q = L(s-1): slot (s - s0) (slot 0 = checkpoint when s == s0)
      const float* q = st + (size_t)(s - s0) * D;
      float Lq[K];
#pragma unroll
      for (int j = 0; j < K; ++j) Lq[j] = q[lane * K + j];
      // m_q and its (lowest) index
      float mn = kInf;
      int mi = 0;
#pragma unroll
      for (int j = 0; j < K; ++j)
        if (Lq[j] < mn) { mn = Lq[j]; mi = lane * K + j; }
      const float mq = warp_min(mn);
      const unsigned hit = __ballot_sync(kFullMask, mn == mq);
      const int src = __ffs(hit) - 1;
      const int kq = __shfl_sync(kFullMask, mi, src);
      // choices at p
      float lm[K], lp[K];
      neighbours<K>(Lq, lane, lm, lp);
      const float jump = mq + P2;
      float g1 = 0.f, g2 = 0.f, gall = 0.f;
      float gsame[K], gm1[K], gp1v[K];
#pragma unroll
      for (int j = 0; j < K; ++j) {
        float t = Lq[j];
        int c3 = 0;
        if (lm[j] + P1 < t) { t = lm[j] + P1; c3 = 1; }
        if (lp[j] + P1 < t) { t = lp[j] + P1; c3 = 2; }
        if (jump < t) { c3 = 3; }
        gsame[j] = c3 == 0 ? gl[j] : 0.f;
        gm1[j] = c3 == 1 ? gl[j] : 0.f;   // flows to L_q(d-1)
        gp1v[j] = c3 == 2 ? gl[j] : 0.f;  // flows to L_q(d+1)
        if (c3 == 1 || c3 == 2) g1 += gl[j];
        if (c3 == 3) g2 += gl[j];
        gall += gl[j];
      }
      g1 = warp_sum(g1);
      g2 = warp_sum(g2);
      gall = warp_sum(gall);
      if (lane == 0) {
        gp1[p] += g1;
        gp2[p] += g2;
      }
      // gradient of L_q: same d, from d+1 choosing d-1 (i.e. d), from d-1 choosing d+1 (i.e. d)
      const float from_up = __shfl_down_sync(kFullMask, gm1[0], 1);     // d = lane*K+K-1 receives gm1 of d+1
      const float from_down = __shfl_up_sync(kFullMask, gp1v[K - 1], 1); // d = lane*K receives gp1 of d-1
#pragma unroll
      for (int j = 0; j < K; ++j) {
        float v = gsame[j];
        v += j < K - 1 ? gm1[j + 1] : (lane < 31 ? from_up : 0.f);
        v += j > 0 ? gp1v[j - 1] : (lane > 0 ? from_down : 0.f);
        if (lane * K + j == kq) v += g2 - gall;
        gnext[j] = v;
      }
    }
    __syncwarp();
  }
}

int check(const char* what) {
  const cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(st);
    sgm_set_process_error(m.c_str());
    return SGM_ERR_CUDA;
  }
  return SGM_OK;
}

int validate(int B, int H, int W, int D) {
  if (B <= 0 || H <= 0 || W <= 0 || (D != 32 && D != 64)) {
    sgm_set_process_error("float SGM: B, H, W > 0 and D in {32, 64} required");
    return SGM_ERR_ARG;
  }
  return SGM_OK;
}

}  // namespace

extern "C" {

size_t sgm_float_checkpoint_elems(int32_t B, int32_t H, int32_t W, int32_t D) {
  size_t n = 0;
  for (int dir = 0; dir < 4; ++dir) {
    const Geo g = make_geo(B, H, W, D, dir);
    n = n > (size_t)g.lines * g.nseg * D ? n : (size_t)g.lines * g.nseg * D;
  }
  return 4 * n;
}

int sgm_float_forward(const float* cost, const float* p1, const float* p2, int32_t B, int32_t H, int32_t W,
                      int32_t D, float temperature, float* sum, float* ckpt, float* disp, void* stream) {
  int st = validate(B, H, W, D);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // path checkpoints are laid out with the largest per-path size so every path has its own slab
  const size_t slab = sgm_float_checkpoint_elems(B, H, W, D) / 4;
  const int order[4] = {0, 1, 2, 3};
  for (int i = 0; i < 4; ++i) {
    Geo g = make_geo(B, H, W, D, order[i]);
    float* ck = ckpt + slab * order[i];
    dim3 blk(32, 8), grd((g.lines + 7) / 8);
    if (D == 64) k_float_fwd<2><<<grd, blk, 0, s>>>(cost, p1, p2, sum, ck, g, i == 0);
    else k_float_fwd<1><<<grd, blk, 0, s>>>(cost, p1, p2, sum, ck, g, i == 0);
    if ((st = check("float forward"))) return st;
  }
  const size_t npix = (size_t)B * H * W;
  dim3 blk(32, 8), grd((unsigned)((npix + 7) / 8));
  if (D == 64) k_soft_argmin<2><<<grd, blk, 0, s>>>(sum, disp, nullptr, nullptr, npix, 1.0f / temperature);
  else k_soft_argmin<1><<<grd, blk, 0, s>>>(sum, disp, nullptr, nullptr, npix, 1.0f / temperature);
  return check("soft argmin");
}

int sgm_float_backward(const float* cost, const float* p1, const float* p2, int32_t B, int32_t H, int32_t W, int32_t D,
                       float temperature, const float* sum, const float* ckpt, const float* grad_disp,
                       float* grad_sum, float* grad_cost, float* grad_p1, float* grad_p2, void* stream) {
  int st = validate(B, H, W, D);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t npix = (size_t)B * H * W;
  {
    dim3 blk(32, 8), grd((unsigned)((npix + 7) / 8));
    if (D == 64) k_soft_argmin<2><<<grd, blk, 0, s>>>(sum, nullptr, grad_disp, grad_sum, npix, 1.0f / temperature);
    else k_soft_argmin<1><<<grd, blk, 0, s>>>(sum, nullptr, grad_disp, grad_sum, npix, 1.0f / temperature);
    if ((st = check("soft argmin backward"))) return st;
  }
  // P1/P2 gradients accumulate over the paths; the first pixel of a path adds nothing
  if (cudaMemsetAsync(grad_p1, 0, npix * sizeof(float), s) != cudaSuccess ||
      cudaMemsetAsync(grad_p2, 0, npix * sizeof(float), s) != cudaSuccess)
    return check("float backward memset");
  const size_t slab = sgm_float_checkpoint_elems(B, H, W, D) / 4;
  for (int i = 0; i < 4; ++i) {
    Geo g = make_geo(B, H, W, D, i);
    const float* ck = ckpt + slab * i;
    dim3 blk(32, 4), grd((g.lines + 3) / 4);
    const size_t smem = (size_t)4 * (kSeg + 1) * D * sizeof(float);
    if (D == 64)
      k_float_bwd<2><<<grd, blk, smem, s>>>(cost, p1, p2, ck, grad_sum, grad_cost, grad_p1, grad_p2, g, i == 0);
    else
      k_float_bwd<1><<<grd, blk, smem, s>>>(cost, p1, p2, ck, grad_sum, grad_cost, grad_p1, grad_p2, g, i == 0);
    if ((st = check("float backward"))) return st;
  }
  return SGM_OK;
}

}  // extern "C"
