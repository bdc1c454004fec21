// unet.cu - the learned warm start: a 4-level convolutional U-Net that maps
// Re and the obstacle's signed distance on a coarse grid to the developed
// velocity and density, trained on the solver's own snapshots.
//
// Activations are NHWC BF16; every 3x3 convolution is an implicit GEMM on
// the tensor cores (mma.sync m16n8k16, BF16 operands, FP32 accumulation):
// M = pixels, N = output channels, K = 9 taps x input channels.  The input
// gradient is the same kernel on the gradient with flipped, transposed
// weights; the weight gradient is a GEMM over pixels (M = output channels,
// N = input channels of one tap, K = pixels) split over pixel chunks with
// FP32 atomics.  Parameters are FP32 masters updated by Adam; BF16 copies
// feed the tensor cores.  No reference counterpart.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/mblbm.h"
#include "unet_umma.cuh"

#define UN_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      std::fprintf(stderr, "mblbm unet: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), \
                   __FILE__, __LINE__);                                                        \
      return MB_ERR_CUDA;                                                                      \
    }                                                                                          \
  } while (0)

namespace {

using bf16 = __nv_bfloat16;
constexpr int CIN_RAW = 4;   // sdf, Re, inside, x
constexpr int CIN_PAD = 16;  // first layer input, padded for the K step of 16
constexpr int COUT_HEAD = 3;

// A view of an NHWC tensor: pixel p, channel c at ptr[p * cs + co + c].
struct View {
  void *ptr;
  int cs, co;  // channel stride (elements per pixel) and channel offset
};

// ---------------------------------------------------------------------------
// Tensor-core building block
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(float *c, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ uint32_t ld_pair(const bf16 *p) { return *(const uint32_t *)p; }
__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// ---------------------------------------------------------------------------
// 3x3 convolution, stride 1, zero padding 1, as an implicit GEMM.
// CTA: 4 warps, 64 pixels x 64 output channels; warp: 32 x 32 (2 x 4 MMA
// tiles).  Cin is a multiple of 16 and Cout of 32.  Weights W[Cout][9][Cin].
// OUT_F32 = false: Y = relu?(conv + bias) as BF16 (forward).
// OUT_F32 = true : Y (+)= conv as FP32, no bias (input gradient, with the
// flipped transposed weights).
// ---------------------------------------------------------------------------
template <bool OUT_F32>
__global__ void __launch_bounds__(128) k_conv3x3(View X, const bf16 *__restrict__ Wt, const float *__restrict__ bias,
                                                 View Y, int NP, int H, int W, int Cin, int Cout, int relu,
                                                 int accumulate) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tig = lane & 3;
  const int p_base = blockIdx.x * 64 + (warp >> 1) * 32;
  const int n_base = blockIdx.y * 64 + (warp & 1) * 32;
  if (n_base >= Cout) return;  // warp-uniform
  const int HW = H * W;
  // the four pixel rows this thread feeds into A: m-tile mt, half h
  int py[4], px[4], pn[4];
  bool pv[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int p = p_base + (q >> 1) * 16 + g + (q & 1) * 8;
    pv[q] = p < NP;
    const int pp = pv[q] ? p : 0;
    pn[q] = pp / HW;
    const int r = pp - pn[q] * HW;
    py[q] = r / W;
    px[q] = r - py[q] * W;
  }
  float acc[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[a][b][c] = 0.f;
  const bf16 *xb = (const bf16 *)X.ptr;
  for (int t = 0; t < 9; t++) {
    const int dy = t / 3 - 1, dx = t % 3 - 1;
    const bf16 *src[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int yy = py[q] + dy, xx = px[q] + dx;
      const bool ok = pv[q] && yy >= 0 && yy < H && xx >= 0 && xx < W;
      src[q] = ok ? xb + ((long long)(pn[q] * HW + yy * W + xx)) * X.cs + X.co : nullptr;
    }
    for (int k0 = 0; k0 < Cin; k0 += 16) {
      uint32_t af[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; mt++) {
        const bf16 *s0 = src[mt * 2], *s1 = src[mt * 2 + 1];
        af[mt][0] = s0 ? ld_pair(s0 + k0 + tig * 2) : 0u;
        af[mt][1] = s1 ? ld_pair(s1 + k0 + tig * 2) : 0u;
        af[mt][2] = s0 ? ld_pair(s0 + k0 + tig * 2 + 8) : 0u;
        af[mt][3] = s1 ? ld_pair(s1 + k0 + tig * 2 + 8) : 0u;
      }
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const int n = n_base + nt * 8 + g;
        uint32_t bfr[2] = {0u, 0u};
        if (n < Cout) {
          const bf16 *w = Wt + ((long long)n * 9 + t) * Cin + k0 + tig * 2;
          bfr[0] = ld_pair(w);
          bfr[1] = ld_pair(w + 8);
        }
#pragma unroll
        for (int mt = 0; mt < 2; mt++) mma_bf16(acc[mt][nt], af[mt], bfr);
      }
    }
  }
  // epilogue: acc[mt][nt][h*2 + e] is pixel row (g + 8h) of m-tile mt, channel nt*8 + tig*2 + e
#pragma unroll
  for (int mt = 0; mt < 2; mt++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int p = p_base + mt * 16 + g + h * 8;
      if (p >= NP) continue;
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const int n = n_base + nt * 8 + tig * 2;
        if (n >= Cout) continue;
        float v0 = acc[mt][nt][h * 2], v1 = acc[mt][nt][h * 2 + 1];
        if constexpr (OUT_F32) {
          float *y = (float *)Y.ptr + (long long)p * Y.cs + Y.co + n;
          if (accumulate) {
            v0 += y[0];
            v1 += y[1];
          }
          y[0] = v0;
          y[1] = v1;
        } else {
          v0 += bias[n];
          v1 += bias[n + 1];
          if (relu) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          bf16 *y = (bf16 *)Y.ptr + (long long)p * Y.cs + Y.co + n;
          *(__nv_bfloat162 *)y = __floats2bfloat162_rn(v0, v1);
        }
      }
    }
}

// ---------------------------------------------------------------------------
// Weight gradient of a 3x3 convolution: dW[co][t][ci] += sum_p dY[p][co] X[p+off_t][ci].
// CTA: 4 warps, 64 co x 64 ci of one tap over a chunk of pixels; warp 32 x 32.
// MMA: A[m = co][k = pixel], B[k = pixel][n = ci]; fragments packed from
// single BF16 loads.  Partial sums go to FP32 dW with atomics.
// ---------------------------------------------------------------------------
constexpr int WG_CHUNK = 256;
__global__ void __launch_bounds__(128) k_conv3x3_wgrad(View X, const bf16 *__restrict__ dY, float *dW, int NP, int H,
                                                       int W, int Cin, int Cout) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tig = lane & 3;
  const int t = blockIdx.y % 9;
  const int cig = blockIdx.y / 9;  // 64-wide input-channel group
  const int co_base = blockIdx.z * 64 + (warp >> 1) * 32;
  const int ci_base = cig * 64 + (warp & 1) * 32;
  if (co_base >= Cout || ci_base >= Cin) return;
  const int dy = t / 3 - 1, dx = t % 3 - 1;
  const int HW = H * W;
  const bf16 *xb = (const bf16 *)X.ptr;
  float acc[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[a][b][c] = 0.f;
  const int p0 = blockIdx.x * WG_CHUNK;
  const int p1 = min(NP, p0 + WG_CHUNK);
  const bf16 zero = __float2bfloat16(0.f);
  for (int kb = p0; kb < p1; kb += 16) {
    // the four pixels of this thread's k slots: kb + tig*2 + {0,1} and +8
    const bf16 *xs[4];
    int pk[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int p = kb + tig * 2 + (q & 1) + (q >> 1) * 8;
      pk[q] = p;
      xs[q] = nullptr;
      if (p < p1) {
        const int n = p / HW, r = p - n * HW, y = r / W, x = r - y * W;
        const int yy = y + dy, xx = x + dx;
        if (yy >= 0 && yy < H && xx >= 0 && xx < W) xs[q] = xb + ((long long)(n * HW + yy * W + xx)) * X.cs + X.co;
      }
    }
    uint32_t af[2][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
      const int c0 = co_base + mt * 16 + g, c1 = c0 + 8;
      bf16 v[2][4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const bool okp = pk[q] < p1;
        v[0][q] = (okp && c0 < Cout) ? dY[(long long)pk[q] * Cout + c0] : zero;
        v[1][q] = (okp && c1 < Cout) ? dY[(long long)pk[q] * Cout + c1] : zero;
      }
      af[mt][0] = pack2(v[0][0], v[0][1]);
      af[mt][1] = pack2(v[1][0], v[1][1]);
      af[mt][2] = pack2(v[0][2], v[0][3]);
      af[mt][3] = pack2(v[1][2], v[1][3]);
    }
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
      const int ci = ci_base + nt * 8 + g;
      bf16 v[4];
#pragma unroll
      for (int q = 0; q < 4; q++) v[q] = (xs[q] && ci < Cin) ? xs[q][ci] : zero;
      uint32_t bfr[2] = {pack2(v[0], v[1]), pack2(v[2], v[3])};
#pragma unroll
      for (int mt = 0; mt < 2; mt++) mma_bf16(acc[mt][nt], af[mt], bfr);
    }
  }
#pragma unroll
  for (int mt = 0; mt < 2; mt++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int co = co_base + mt * 16 + g + h * 8;
      if (co >= Cout) continue;
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const int ci = ci_base + nt * 8 + tig * 2;
        if (ci >= Cin) continue;
        float *d = dW + ((long long)co * 9 + t) * Cin + ci;
        atomicAdd(d, acc[mt][nt][h * 2]);
        atomicAdd(d + 1, acc[mt][nt][h * 2 + 1]);
      }
    }
}

// bias gradient: db[c] += sum_p dY[p][c]
__global__ void k_bias_grad(const bf16 *__restrict__ dY, float *db, int NP, int C) {
  const int c = threadIdx.x % C;  // blockDim is a multiple of C (C <= 256)
  const int lanes = blockDim.x / C;
  const int sub = threadIdx.x / C;
  float s = 0.f;
  for (int p = blockIdx.x * lanes + sub; p < NP; p += gridDim.x * lanes) s += __bfloat162float(dY[(long long)p * C + c]);
  atomicAdd(db + c, s);
}

// g (FP32, gradient w.r.t. a ReLU output T) -> BF16 gradient w.r.t. the pre-activation
__global__ void k_relu_grad(const float *__restrict__ g, const bf16 *__restrict__ T, bf16 *out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(__bfloat162float(T[i]) > 0.f ? g[i] : 0.f);
}

// 2x2 average pooling (forward on BF16, backward accumulates FP32)
__global__ void k_pool_fwd(const bf16 *__restrict__ X, bf16 *Y, int N, int H, int W, int C) {
  const int Ho = H / 2, Wo = W / 2;
  const long long n = (long long)N * Ho * Wo * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    long long r = i / C;
    const int x = (int)(r % Wo);
    r /= Wo;
    const int y = (int)(r % Ho);
    const int b = (int)(r / Ho);
    const bf16 *s = X + (((long long)b * H + 2 * y) * W + 2 * x) * C + c;
    const float v = __bfloat162float(s[0]) + __bfloat162float(s[C]) + __bfloat162float(s[(long long)W * C]) +
                    __bfloat162float(s[(long long)W * C + C]);
    Y[i] = __float2bfloat16(0.25f * v);
  }
}
__global__ void k_pool_bwd(const float *__restrict__ gY, float *gX, int N, int H, int W, int C) {
  const long long n = (long long)N * H * W * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    long long r = i / C;
    const int x = (int)(r % W);
    r /= W;
    const int y = (int)(r % H);
    const int b = (int)(r / H);
    gX[i] += 0.25f * gY[(((long long)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
  }
}

// nearest x2 upsampling of X (N, H/2, W/2, C) into channels [co, co+C) of Y (N, H, W, cs)
__global__ void k_up_fwd(const bf16 *__restrict__ X, View Y, int N, int H, int W, int C) {
  const long long n = (long long)N * H * W * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long p = i / C;
    const int x = (int)(p % W);
    const long long r = p / W;
    const int y = (int)(r % H);
    const int b = (int)(r / H);
    ((bf16 *)Y.ptr)[p * Y.cs + Y.co + c] = X[(((long long)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
  }
}
// gX (N, H/2, W/2, C) += sum over the 4 children of channels [co, co+C) of gY
__global__ void k_up_bwd(View gY, float *gX, int N, int H, int W, int C) {
  const int Ho = H / 2, Wo = W / 2;
  const long long n = (long long)N * Ho * Wo * C;
  const float *g = (const float *)gY.ptr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    long long r = i / C;
    const int x = (int)(r % Wo);
    r /= Wo;
    const int y = (int)(r % Ho);
    const int b = (int)(r / Ho);
    const long long p = ((long long)b * H + 2 * y) * W + 2 * x;
    gX[i] += g[p * gY.cs + gY.co + c] + g[(p + 1) * gY.cs + gY.co + c] + g[(p + W) * gY.cs + gY.co + c] +
             g[(p + W + 1) * gY.cs + gY.co + c];
  }
}
// copy X (N*H*W, C) into channels [co, co+C) of Y / add channels back
__global__ void k_chan_copy(const bf16 *__restrict__ X, View Y, long long NP, int C) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NP * C; i += (long long)gridDim.x * blockDim.x)
    ((bf16 *)Y.ptr)[(i / C) * Y.cs + Y.co + i % C] = X[i];
}
__global__ void k_chan_add(View gY, float *gX, long long NP, int C) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NP * C; i += (long long)gridDim.x * blockDim.x)
    gX[i] += ((const float *)gY.ptr)[(i / C) * gY.cs + gY.co + i % C];
}

// network input: FP32 [NP][4] -> BF16 [NP][16] (zero padded)
__global__ void k_input(const float *__restrict__ in, bf16 *out, long long NP) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NP * CIN_PAD;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % CIN_PAD);
    out[i] = __float2bfloat16(c < CIN_RAW ? in[(i / CIN_PAD) * CIN_RAW + c] : 0.f);
  }
}

// head: 1x1 convolution 32 -> 3 in FP32 on the BF16 features; with a target,
// the masked mean squared error and its gradients:
//   loss = sum_p m_p sum_o (y_po - t_po)^2 / (3 sum_p m_p)
struct HeadArgs {
  const bf16 *X;        // [NP][C]
  const float *Wh;      // [3][C]
  const float *bh;      // [3]
  float *out;           // [NP][3] (may be null)
  const float *target;  // [NP][3] (null: no loss)
  const float *mask;    // [NP]
  float inv_count;      // 1 / (3 sum m)
  float *loss;          // accumulated
  float *gX;            // [NP][C] gradient w.r.t. X (FP32, overwritten)
  float *gW, *gb;       // accumulated
  long long NP;
  int C;
};
__global__ void __launch_bounds__(256) k_head(HeadArgs a) {
  __shared__ float sW[COUT_HEAD * 64];
  for (int q = threadIdx.x; q < COUT_HEAD * a.C; q += blockDim.x) sW[q] = a.Wh[q];
  __syncthreads();
  float lsum = 0.f, gWl[COUT_HEAD * 32], gbl[COUT_HEAD];
  for (int q = 0; q < COUT_HEAD * 32; q++) gWl[q] = 0.f;
  for (int o = 0; o < COUT_HEAD; o++) gbl[o] = 0.f;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < a.NP; p += (long long)gridDim.x * blockDim.x) {
    float x[32];
    for (int c = 0; c < a.C; c++) x[c] = __bfloat162float(a.X[p * a.C + c]);
    float y[COUT_HEAD];
    for (int o = 0; o < COUT_HEAD; o++) {
      float s = a.bh[o];
      for (int c = 0; c < a.C; c++) s += sW[o * a.C + c] * x[c];
      y[o] = s;
      if (a.out) a.out[p * COUT_HEAD + o] = s;
    }
    if (!a.target) continue;
    const float m = a.mask[p];
    float gy[COUT_HEAD];
    for (int o = 0; o < COUT_HEAD; o++) {
      const float d = y[o] - a.target[p * COUT_HEAD + o];
      lsum += m * d * d * a.inv_count;
      gy[o] = 2.f * m * d * a.inv_count;
      gbl[o] += gy[o];
      for (int c = 0; c < a.C; c++) gWl[o * 32 + c] += gy[o] * x[c];
    }
    for (int c = 0; c < a.C; c++) {
      float s = 0.f;
      for (int o = 0; o < COUT_HEAD; o++) s += sW[o * a.C + c] * gy[o];
      a.gX[p * a.C + c] = s;
    }
  }
  if (!a.target) return;
  // block reductions, then one atomic per value
  __shared__ float red[256];
  auto reduce = [&](float v) -> float {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    const float r = red[0];
    __syncthreads();
    return r;
  };
  const float L = reduce(lsum);
  if (threadIdx.x == 0) atomicAdd(a.loss, L);
  for (int o = 0; o < COUT_HEAD; o++) {
    const float b = reduce(gbl[o]);
    if (threadIdx.x == 0) atomicAdd(a.gb + o, b);
    for (int c = 0; c < a.C; c++) {
      const float w = reduce(gWl[o * 32 + c]);
      if (threadIdx.x == 0) atomicAdd(a.gW + o * a.C + c, w);
    }
  }
}

// FP32 master weights of a 3x3 layer -> BF16 W[Cout][9][Cin] and the input-
// gradient weights Wt[Cin][9][Cout] = W[co][8 - t][ci]
__global__ void k_weights_bf16(const float *__restrict__ w, bf16 *wb, bf16 *wt, int Cout, int Cin) {
  const long long n = (long long)Cout * 9 * Cin;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(i % Cin);
    const int t = (int)((i / Cin) % 9);
    const int co = (int)(i / ((long long)Cin * 9));
    const bf16 v = __float2bfloat16(w[i]);
    wb[i] = v;
    wt[((long long)ci * 9 + (8 - t)) * Cout + co] = v;
  }
}

// Adam (Kingma and Ba), bias-corrected, on every parameter
__global__ void k_adam(float *w, float *m, float *v, const float *g, long long n, float lr, float b1, float b2,
                       float c1, float c2, float eps) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void k_zero(float *p, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = 0.f;
}

int grid_for(long long n, int th = 256) { return (int)std::max<long long>(1, std::min<long long>((n + th - 1) / th, 148LL * 16)); }

}  // namespace

// ===========================================================================
// The network
// ===========================================================================
namespace {
struct ConvLayer {
  int cin, cout, level;  // level: resolution H >> level
  long long w_off, b_off;  // offsets in the parameter array
  bf16 *wb = nullptr, *wt = nullptr;
};
// activation buffers per level
}  // namespace

struct mb_unet {
  int H, W, maxN, C0;
  int gemm = 1;                  // 3x3 convolutions: 1 tcgen05 (where the layer's shape fits), 0 mma.sync
  unsigned int *d_err = nullptr; // error word of the tcgen05 kernels' bounded waits
  std::vector<ConvLayer> conv;  // 14 layers, in forward order
  long long head_w = 0, head_b = 0, nparam = 0;
  float *P = nullptr, *M = nullptr, *V = nullptr, *G = nullptr;  // params, Adam moments, gradients
  long long step = 0;
  std::vector<void *> allocs;
  // activations (BF16) and gradients (FP32)
  bf16 *x_in = nullptr;
  bf16 *act[14] = {};        // outputs of the 14 conv layers
  bf16 *pool[3] = {};        // pooled e0b, e1b, e2b
  bf16 *cat[3] = {};         // concat inputs of d2a, d1a, d0a (level 2, 1, 0)
  float *gact[14] = {};      // gradient w.r.t. each conv output
  float *gpool[3] = {}, *gcat[3] = {};
  bf16 *gbf = nullptr;       // BF16 gradient w.r.t. a pre-activation (scratch, largest layer)
  float *d_loss = nullptr;
  float *h_loss = nullptr;
};

namespace {
// layer table: (cin, cout, level)
const int kLayers[14][3] = {{16, 32, 0},   {32, 32, 0},   {32, 64, 1},   {64, 64, 1},  {64, 128, 2},
                            {128, 128, 2}, {128, 256, 3}, {256, 256, 3}, {384, 128, 2}, {128, 128, 2},
                            {192, 64, 1},  {64, 64, 1},   {96, 32, 0},   {32, 32, 0}};

template <typename T>
int ualloc(mb_unet *n, T **p, size_t count) {
  void *q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return MB_ERR_NOMEM;
  n->allocs.push_back(q);
  *p = (T *)q;
  return MB_OK;
}

uint64_t sm64(uint64_t &s) {
  s += 0x9E3779B97F4A7C15ull;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

long long npix(const mb_unet *n, int N, int level) { return (long long)N * (n->H >> level) * (n->W >> level); }

// ---- tcgen05 path: tensor maps and launch --------------------------------
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiled)p;
  }
  return fn;
}

// Pixel tile, channel step and channel tile of a layer on the tcgen05 path;
// false when the layer's shape does not fit it (the mma.sync kernel runs).
struct UmmaShape {
  int Cw, R, CH, NT;
};
bool umma_shape(int H, int W, int Cin, int Cout, UmmaShape *u) {
  u->Cw = W >= umma::TM ? umma::TM : W;
  if (u->Cw < 8 || umma::TM % u->Cw || W % u->Cw) return false;
  u->R = umma::TM / u->Cw;
  if (H % u->R) return false;
  u->CH = Cin % 64 == 0 ? 64 : (Cin % 32 == 0 ? 32 : (Cin % 16 == 0 ? 16 : 0));
  if (!u->CH) return false;
  u->NT = Cout <= 256 ? Cout : (Cout % 2 == 0 && Cout / 2 <= 256 ? Cout / 2 : 0);
  return u->NT >= 32 && u->NT % 16 == 0 && Cout % u->NT == 0;
}

// Weight gradient of a 3x3 layer on the tensor cores (umma::k_wgrad_umma):
// dW [Cout][9][Cin] += sum_p dY[p][co] X[p + off_t][ci].  MB_ERR_UNSUPPORTED
// when the shape does not fit (fewer than 64 channels on either side, or
// images that do not split into 64-pixel boxes).
int wgrad_umma(mb_unet *n, View X, const bf16 *dY, float *dW, int N, int H, int W, int Cin, int Cout,
               cudaStream_t s) {
  EncodeTiled enc = encode_fn();
  if (!enc || Cin < 64 || Cin % 64 || Cout < 64 || (X.co % 8) || (X.cs % 8)) return MB_ERR_UNSUPPORTED;
  const int Cw = W >= umma::WG_KP ? umma::WG_KP : W;
  if (Cw < 8 || umma::WG_KP % Cw || W % Cw) return MB_ERR_UNSUPPORTED;
  const int R = umma::WG_KP / Cw;
  if (H % R) return MB_ERR_UNSUPPORTED;
  const int NT = Cin <= 256 ? Cin : (Cin % 128 == 0 && Cin / 2 <= 256 ? Cin / 2 : 0);
  if (!NT || NT % 64) return MB_ERR_UNSUPPORTED;
  CUtensorMap gmap, xmap;
  const cuuint32_t box[4] = {64, (cuuint32_t)Cw, (cuuint32_t)R, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  {
    const cuuint64_t dims[4] = {(cuuint64_t)Cout, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    const cuuint64_t st[3] = {(cuuint64_t)Cout * 2, (cuuint64_t)Cout * 2 * W, (cuuint64_t)Cout * 2 * W * H};
    if (enc(&gmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)dY, dims, st, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return MB_ERR_CUDA;
  }
  {
    const cuuint64_t dims[4] = {(cuuint64_t)Cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    const cuuint64_t st[3] = {(cuuint64_t)X.cs * 2, (cuuint64_t)X.cs * 2 * W, (cuuint64_t)X.cs * 2 * W * H};
    if (enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (bf16 *)X.ptr + X.co, dims, st, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return MB_ERR_CUDA;
  }
  umma::WgradArgs a{};
  a.H = H;
  a.W = W;
  a.Cw = Cw;
  a.R = R;
  a.bx = W / Cw;
  a.by = H / R;
  a.nboxes = a.bx * a.by * N;
  const int mt = (Cout + umma::TM - 1) / umma::TM, nt = Cin / NT;
  // split-K: about two CTAs per SM over (pixel runs x channel tiles x taps)
  const long long want = std::max<long long>(1, (long long)a.nboxes * 9 * mt * nt / (148 * 2));
  a.boxes_per_cta = (int)std::min<long long>(128, std::max<long long>(4, want));
  a.Cin = Cin;
  a.Cout = Cout;
  a.NT = NT;
  a.dW = dW;
  a.err = n->d_err;
  const dim3 grid((unsigned)((a.nboxes + a.boxes_per_cta - 1) / a.boxes_per_cta), (unsigned)mt, (unsigned)(9 * nt));
  const size_t smem = umma::wgrad_smem(NT);
  UN_CUDA(cudaFuncSetAttribute((const void *)umma::k_wgrad_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  void *args[3] = {&gmap, &xmap, &a};
  UN_CUDA(cudaLaunchKernel((const void *)umma::k_wgrad_umma, grid, dim3(umma::THREADS), args, smem, s));
  return MB_OK;
}

// 3x3 convolution of X (view, Cin channels, N images of H x W) with weights
// wt [Cout][9][Cin] on the tensor cores: BF16 output with bias and ReLU, or
// FP32 output (accumulated when asked).  Returns MB_ERR_UNSUPPORTED when the
// shape or the driver's tensor-map entry point rules it out.
int conv_umma(mb_unet *n, View X, const bf16 *wt, const float *bias, View Y, int N, int H, int W, int Cin, int Cout,
              bool out_f32, bool accumulate, cudaStream_t s) {
  UmmaShape u;
  EncodeTiled enc = encode_fn();
  if (!enc || !umma_shape(H, W, Cin, Cout, &u)) return MB_ERR_UNSUPPORTED;
  if ((X.co % 8) || (X.cs % 8) || (Y.co % 8) || (Y.cs % 8)) return MB_ERR_UNSUPPORTED;  // 16-byte alignment
  const CUtensorMapSwizzle sw = u.CH == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                           : (u.CH == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
  CUtensorMap xmap, wmap;
  {
    const cuuint64_t dims[4] = {(cuuint64_t)Cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    const cuuint64_t strides[3] = {(cuuint64_t)X.cs * 2, (cuuint64_t)X.cs * 2 * W, (cuuint64_t)X.cs * 2 * W * H};
    const cuuint32_t box[4] = {(cuuint32_t)u.CH, (cuuint32_t)u.Cw, (cuuint32_t)u.R, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    if (enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (bf16 *)X.ptr + X.co, dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return MB_ERR_CUDA;
  }
  {
    const cuuint64_t dims[2] = {(cuuint64_t)9 * Cin, (cuuint64_t)Cout};
    const cuuint64_t strides[1] = {(cuuint64_t)9 * Cin * 2};
    const cuuint32_t box[2] = {(cuuint32_t)u.CH, (cuuint32_t)u.NT};
    const cuuint32_t es[2] = {1, 1};
    if (enc(&wmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)wt, dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return MB_ERR_CUDA;
  }
  umma::ConvArgs a{};
  a.H = H;
  a.W = W;
  a.Cw = u.Cw;
  a.R = u.R;
  a.tiles_x = W / u.Cw;
  a.tiles_y = H / u.R;
  a.Cin = Cin;
  a.NT = u.NT;
  a.relu = out_f32 ? 0 : 1;
  a.out_f32 = out_f32;
  a.accumulate = accumulate;
  a.bias = bias;
  a.Y = Y.ptr;
  a.ycs = Y.cs;
  a.yco = Y.co;
  a.Cout = Cout;
  a.err = n->d_err;
  const dim3 grid((unsigned)(a.tiles_x * a.tiles_y * N), (unsigned)(Cout / u.NT));
  void *args[3] = {&xmap, &wmap, &a};
  const void *fn = u.CH == 64 ? (const void *)umma::k_conv3x3_umma<64>
                              : (u.CH == 32 ? (const void *)umma::k_conv3x3_umma<32> : (const void *)umma::k_conv3x3_umma<16>);
  const size_t smem = u.CH == 64 ? umma::Cfg<64>::smem(u.NT) : (u.CH == 32 ? umma::Cfg<32>::smem(u.NT) : umma::Cfg<16>::smem(u.NT));
  UN_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  UN_CUDA(cudaLaunchKernel(fn, grid, dim3(umma::THREADS), args, smem, s));
  return MB_OK;
}

int conv_fwd(mb_unet *n, int li, View X, View Y, int N, cudaStream_t s) {
  const ConvLayer &L = n->conv[li];
  const int H = n->H >> L.level, W = n->W >> L.level;
  const long long NP = (long long)N * H * W;
  if (n->gemm == 1) {
    const int e = conv_umma(n, X, L.wb, n->P + L.b_off, Y, N, H, W, L.cin, L.cout, false, false, s);
    if (e != MB_ERR_UNSUPPORTED) return e;
  }
  dim3 grid((unsigned)((NP + 63) / 64), (unsigned)((L.cout + 63) / 64));
  k_conv3x3<false><<<grid, 128, 0, s>>>(X, L.wb, n->P + L.b_off, Y, (int)NP, H, W, L.cin, L.cout, 1, 0);
  UN_CUDA(cudaGetLastError());
  return MB_OK;
}

// backward of conv layer li given g (FP32 gradient w.r.t. its ReLU output):
// weight and bias gradients, and (if gX) the input gradient accumulated into gX
int conv_bwd(mb_unet *n, int li, View X, const float *g, View gX, bool need_gx, int N, cudaStream_t s) {
  const ConvLayer &L = n->conv[li];
  const int H = n->H >> L.level, W = n->W >> L.level;
  const long long NP = (long long)N * H * W;
  k_relu_grad<<<grid_for(NP * L.cout), 256, 0, s>>>(g, n->act[li], n->gbf, NP * L.cout);
  int ew = MB_ERR_UNSUPPORTED;
  if (n->gemm == 1) ew = wgrad_umma(n, X, n->gbf, n->G + L.w_off, N, H, W, L.cin, L.cout, s);
  if (ew == MB_ERR_UNSUPPORTED) {
    dim3 wg((unsigned)((NP + WG_CHUNK - 1) / WG_CHUNK), (unsigned)(9 * ((L.cin + 63) / 64)),
            (unsigned)((L.cout + 63) / 64));
    k_conv3x3_wgrad<<<wg, 128, 0, s>>>(X, n->gbf, n->G + L.w_off, (int)NP, H, W, L.cin, L.cout);
  } else if (ew) {
    return ew;
  }
  const int bt = 256 / L.cout * L.cout;
  k_bias_grad<<<grid_for(NP, 256), bt > 0 ? bt : L.cout, 0, s>>>(n->gbf, n->G + L.b_off, (int)NP, L.cout);
  if (need_gx) {
    View gy{n->gbf, L.cout, 0};
    int e = MB_ERR_UNSUPPORTED;
    if (n->gemm == 1) e = conv_umma(n, gy, L.wt, nullptr, gX, N, H, W, L.cout, L.cin, true, true, s);
    if (e == MB_ERR_UNSUPPORTED) {
      dim3 grid((unsigned)((NP + 63) / 64), (unsigned)((L.cin + 63) / 64));
      k_conv3x3<true><<<grid, 128, 0, s>>>(gy, L.wt, nullptr, gX, (int)NP, H, W, L.cout, L.cin, 0, 1);
    } else if (e) {
      return e;
    }
  }
  UN_CUDA(cudaGetLastError());
  return MB_OK;
}

int refresh_weights(mb_unet *n, cudaStream_t s) {
  for (auto &L : n->conv) {
    const long long cnt = (long long)L.cout * 9 * L.cin;
    k_weights_bf16<<<grid_for(cnt), 256, 0, s>>>(n->P + L.w_off, L.wb, L.wt, L.cout, L.cin);
  }
  UN_CUDA(cudaGetLastError());
  return MB_OK;
}

int forward(mb_unet *n, const float *d_in, int N, cudaStream_t s) {
  const long long NP0 = npix(n, N, 0);
  k_input<<<grid_for(NP0 * CIN_PAD), 256, 0, s>>>(d_in, n->x_in, NP0);
  auto V = [](void *p, int cs, int co = 0) { return View{p, cs, co}; };
  int e;
  // encoder
  if ((e = conv_fwd(n, 0, V(n->x_in, CIN_PAD), V(n->act[0], 32), N, s))) return e;
  if ((e = conv_fwd(n, 1, V(n->act[0], 32), V(n->act[1], 32), N, s))) return e;
  k_pool_fwd<<<grid_for(npix(n, N, 1) * 32), 256, 0, s>>>(n->act[1], n->pool[0], N, n->H, n->W, 32);
  if ((e = conv_fwd(n, 2, V(n->pool[0], 32), V(n->act[2], 64), N, s))) return e;
  if ((e = conv_fwd(n, 3, V(n->act[2], 64), V(n->act[3], 64), N, s))) return e;
  k_pool_fwd<<<grid_for(npix(n, N, 2) * 64), 256, 0, s>>>(n->act[3], n->pool[1], N, n->H >> 1, n->W >> 1, 64);
  if ((e = conv_fwd(n, 4, V(n->pool[1], 64), V(n->act[4], 128), N, s))) return e;
  if ((e = conv_fwd(n, 5, V(n->act[4], 128), V(n->act[5], 128), N, s))) return e;
  k_pool_fwd<<<grid_for(npix(n, N, 3) * 128), 256, 0, s>>>(n->act[5], n->pool[2], N, n->H >> 2, n->W >> 2, 128);
  if ((e = conv_fwd(n, 6, V(n->pool[2], 128), V(n->act[6], 256), N, s))) return e;
  if ((e = conv_fwd(n, 7, V(n->act[6], 256), V(n->act[7], 256), N, s))) return e;
  // decoder: cat[lv] = [up(previous), skip]
  const int upC[3] = {256, 128, 64}, skC[3] = {128, 64, 32}, skip[3] = {5, 3, 1}, prev[3] = {7, 9, 11};
  for (int q = 0; q < 3; q++) {
    const int lv = 2 - q, H = n->H >> lv, W = n->W >> lv, cs = upC[q] + skC[q];
    k_up_fwd<<<grid_for(npix(n, N, lv) * upC[q]), 256, 0, s>>>(n->act[prev[q]], V(n->cat[q], cs, 0), N, H, W, upC[q]);
    k_chan_copy<<<grid_for(npix(n, N, lv) * skC[q]), 256, 0, s>>>(n->act[skip[q]], V(n->cat[q], cs, upC[q]),
                                                                  npix(n, N, lv), skC[q]);
    if ((e = conv_fwd(n, 8 + 2 * q, V(n->cat[q], cs), V(n->act[8 + 2 * q], skC[q]), N, s))) return e;
    if ((e = conv_fwd(n, 9 + 2 * q, V(n->act[8 + 2 * q], skC[q]), V(n->act[9 + 2 * q], skC[q]), N, s))) return e;
  }
  UN_CUDA(cudaGetLastError());
  return MB_OK;
}

int head(mb_unet *n, int N, float *out, const float *target, const float *mask, float inv_count, cudaStream_t s) {
  HeadArgs a{};
  a.X = n->act[13];
  a.Wh = n->P + n->head_w;
  a.bh = n->P + n->head_b;
  a.out = out;
  a.target = target;
  a.mask = mask;
  a.inv_count = inv_count;
  a.loss = n->d_loss;
  a.gX = n->gact[13];
  a.gW = n->G + n->head_w;
  a.gb = n->G + n->head_b;
  a.NP = npix(n, N, 0);
  a.C = 32;
  k_head<<<grid_for(a.NP, 256), 256, 0, s>>>(a);
  UN_CUDA(cudaGetLastError());
  return MB_OK;
}

int backward(mb_unet *n, int N, cudaStream_t s) {
  auto V = [](void *p, int cs, int co = 0) { return View{p, cs, co}; };
  int e;
  const int upC[3] = {256, 128, 64}, skC[3] = {128, 64, 32}, skip[3] = {5, 3, 1}, prev[3] = {7, 9, 11};
  // gradient buffers of layers fed by more than one consumer start at zero
  for (int li : {1, 3, 5, 7, 9, 11})
    k_zero<<<grid_for(npix(n, N, n->conv[li].level) * n->conv[li].cout), 256, 0, s>>>(
        n->gact[li], npix(n, N, n->conv[li].level) * n->conv[li].cout);
  for (int q = 2; q >= 0; q--) {
    const int lv = 2 - q, H = n->H >> lv, W = n->W >> lv, cs = upC[q] + skC[q];
    const long long NP = npix(n, N, lv);
    const int lb = 9 + 2 * q, la = 8 + 2 * q;
    // d?b: input act[la]; its input gradient overwrites gact[la]
    k_zero<<<grid_for(NP * skC[q]), 256, 0, s>>>(n->gact[la], NP * skC[q]);
    if ((e = conv_bwd(n, lb, V(n->act[la], skC[q]), n->gact[lb], V(n->gact[la], skC[q]), true, N, s))) return e;
    // d?a: input cat[q]
    k_zero<<<grid_for(NP * cs), 256, 0, s>>>(n->gcat[q], NP * cs);
    if ((e = conv_bwd(n, la, V(n->cat[q], cs), n->gact[la], V(n->gcat[q], cs), true, N, s))) return e;
    // split the concat gradient: up part -> previous layer (coarser), skip part -> encoder layer
    k_up_bwd<<<grid_for(npix(n, N, lv + 1) * upC[q]), 256, 0, s>>>(V(n->gcat[q], cs, 0), n->gact[prev[q]], N, H, W,
                                                                   upC[q]);
    k_chan_add<<<grid_for(NP * skC[q]), 256, 0, s>>>(V(n->gcat[q], cs, upC[q]), n->gact[skip[q]], NP, skC[q]);
  }
  // encoder, deepest first: layer pairs (6,7), (4,5), (2,3), (0,1)
  for (int lv = 3; lv >= 0; lv--) {
    const int la = 2 * lv, lb = 2 * lv + 1;
    const long long NP = npix(n, N, lv);
    const int ca = n->conv[la].cout, cin = n->conv[la].cin;
    k_zero<<<grid_for(NP * ca), 256, 0, s>>>(n->gact[la], NP * ca);
    if ((e = conv_bwd(n, lb, V(n->act[la], ca), n->gact[lb], V(n->gact[la], ca), true, N, s))) return e;
    if (lv == 0) {
      if ((e = conv_bwd(n, la, V(n->x_in, CIN_PAD), n->gact[la], V(nullptr, 0), false, N, s))) return e;
    } else {
      // input of layer la is pool[lv-1]; its gradient flows back through the pooling into gact[lb - 2]
      k_zero<<<grid_for(NP * cin), 256, 0, s>>>(n->gpool[lv - 1], NP * cin);
      if ((e = conv_bwd(n, la, V(n->pool[lv - 1], cin), n->gact[la], V(n->gpool[lv - 1], cin), true, N, s))) return e;
      k_pool_bwd<<<grid_for(npix(n, N, lv - 1) * cin), 256, 0, s>>>(n->gpool[lv - 1], n->gact[la - 1], N,
                                                                     n->H >> (lv - 1), n->W >> (lv - 1), cin);
    }
  }
  UN_CUDA(cudaGetLastError());
  return MB_OK;
}
}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" int mb_unet_create(int H, int W, int max_batch, unsigned long long seed, mb_unet **out) {
  if (!out || H < 8 || W < 8 || H % 8 || W % 8 || max_batch < 1) return MB_ERR_INVALID;
  *out = nullptr;
  auto n = std::make_unique<mb_unet>();
  n->H = H;
  n->W = W;
  n->maxN = max_batch;
  n->C0 = 32;
  long long off = 0;
  for (int q = 0; q < 14; q++) {
    ConvLayer L;
    L.cin = kLayers[q][0];
    L.cout = kLayers[q][1];
    L.level = kLayers[q][2];
    L.w_off = off;
    off += (long long)L.cout * 9 * L.cin;
    L.b_off = off;
    off += L.cout;
    n->conv.push_back(L);
  }
  n->head_w = off;
  off += COUT_HEAD * 32;
  n->head_b = off;
  off += COUT_HEAD;
  n->nparam = off;
  int e;
  if ((e = ualloc(n.get(), &n->P, off)) || (e = ualloc(n.get(), &n->M, off)) || (e = ualloc(n.get(), &n->V, off)) ||
      (e = ualloc(n.get(), &n->G, off)))
    return e;
  // He-normal weights (splitmix64 + Box-Muller), zero biases
  std::vector<float> h(off, 0.f);
  uint64_t st = seed;
  auto normal = [&]() {
    const double u1 = ((sm64(st) >> 11) + 0.5) / 9007199254740992.0, u2 = (sm64(st) >> 11) / 9007199254740992.0;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  };
  for (auto &L : n->conv) {
    const double sd = std::sqrt(2.0 / (9.0 * L.cin));
    for (long long q = 0; q < (long long)L.cout * 9 * L.cin; q++) h[L.w_off + q] = (float)(sd * normal());
  }
  for (int q = 0; q < COUT_HEAD * 32; q++) h[n->head_w + q] = (float)(std::sqrt(1.0 / 32) * normal());
  UN_CUDA(cudaMemcpy(n->P, h.data(), off * sizeof(float), cudaMemcpyHostToDevice));
  UN_CUDA(cudaMemset(n->M, 0, off * sizeof(float)));
  UN_CUDA(cudaMemset(n->V, 0, off * sizeof(float)));
  UN_CUDA(cudaMemset(n->G, 0, off * sizeof(float)));
  for (auto &L : n->conv) {
    if ((e = ualloc(n.get(), &L.wb, (size_t)L.cout * 9 * L.cin)) || (e = ualloc(n.get(), &L.wt, (size_t)L.cout * 9 * L.cin)))
      return e;
  }
  const int N = max_batch;
  long long maxg = 0;
  if ((e = ualloc(n.get(), &n->x_in, npix(n.get(), N, 0) * CIN_PAD))) return e;
  for (int q = 0; q < 14; q++) {
    const long long cnt = npix(n.get(), N, n->conv[q].level) * n->conv[q].cout;
    maxg = std::max(maxg, cnt);
    if ((e = ualloc(n.get(), &n->act[q], cnt)) || (e = ualloc(n.get(), &n->gact[q], cnt))) return e;
  }
  const int poolC[3] = {32, 64, 128};
  for (int q = 0; q < 3; q++) {
    const long long cnt = npix(n.get(), N, q + 1) * poolC[q];
    if ((e = ualloc(n.get(), &n->pool[q], cnt)) || (e = ualloc(n.get(), &n->gpool[q], cnt))) return e;
  }
  const int catC[3] = {384, 192, 96};
  for (int q = 0; q < 3; q++) {
    const long long cnt = npix(n.get(), N, 2 - q) * catC[q];
    if ((e = ualloc(n.get(), &n->cat[q], cnt)) || (e = ualloc(n.get(), &n->gcat[q], cnt))) return e;
  }
  if ((e = ualloc(n.get(), &n->gbf, maxg))) return e;
  if ((e = ualloc(n.get(), &n->d_loss, 1))) return e;
  if ((e = ualloc(n.get(), &n->d_err, 1))) return e;
  UN_CUDA(cudaMemset(n->d_err, 0, sizeof(unsigned int)));
  UN_CUDA(cudaMallocHost(&n->h_loss, sizeof(float)));
  if ((e = refresh_weights(n.get(), 0))) return e;
  UN_CUDA(cudaDeviceSynchronize());
  *out = n.release();
  return MB_OK;
}

extern "C" int mb_unet_destroy(mb_unet *n) {
  if (!n) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  for (void *p : n->allocs) cudaFree(p);
  if (n->h_loss) cudaFreeHost(n->h_loss);
  delete n;
  return MB_OK;
}

extern "C" int mb_unet_param_count(mb_unet *n, long long *count) {
  if (!n || !count) return MB_ERR_INVALID;
  *count = n->nparam;
  return MB_OK;
}

extern "C" int mb_unet_get_params(mb_unet *n, float *host, long long count, int which) {
  if (!n || !host || count != n->nparam || which < 0 || which > 1) return MB_ERR_INVALID;
  UN_CUDA(cudaMemcpy(host, which ? n->G : n->P, count * sizeof(float), cudaMemcpyDeviceToHost));
  return MB_OK;
}

extern "C" int mb_unet_set_params(mb_unet *n, const float *host, long long count) {
  if (!n || !host || count != n->nparam) return MB_ERR_INVALID;
  UN_CUDA(cudaMemcpy(n->P, host, count * sizeof(float), cudaMemcpyHostToDevice));
  if (int e = refresh_weights(n, 0)) return e;
  UN_CUDA(cudaDeviceSynchronize());
  return MB_OK;
}

extern "C" int mb_unet_set_gemm(mb_unet *n, int kind) {
  if (!n || kind < 0 || kind > 1) return MB_ERR_INVALID;
  n->gemm = kind;
  return MB_OK;
}

extern "C" int mb_unet_status(mb_unet *n, mb_stream stream) {
  if (!n) return MB_ERR_INVALID;
  unsigned int h = 0;
  cudaStream_t s = (cudaStream_t)stream;
  UN_CUDA(cudaMemcpyAsync(&h, n->d_err, sizeof(h), cudaMemcpyDeviceToHost, s));
  UN_CUDA(cudaStreamSynchronize(s));
  if (!h) return MB_OK;
  UN_CUDA(cudaMemset(n->d_err, 0, sizeof(unsigned int)));
  return MB_ERR_TIMEOUT;
}

extern "C" int mb_unet_forward(mb_unet *n, const float *d_in, int N, float *d_out, mb_stream stream) {
  if (!n || !d_in || !d_out || N < 1 || N > n->maxN) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (int e = forward(n, d_in, N, s)) return e;
  return head(n, N, d_out, nullptr, nullptr, 0.f, s);
}

extern "C" int mb_unet_train_step(mb_unet *n, const float *d_in, const float *d_target, const float *d_mask, int N,
                                  float lr, int apply, float *loss, mb_stream stream) {
  if (!n || !d_in || !d_target || !d_mask || N < 1 || N > n->maxN || !(lr >= 0)) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  int e;
  if ((e = forward(n, d_in, N, s))) return e;
  k_zero<<<grid_for(n->nparam), 256, 0, s>>>(n->G, n->nparam);
  UN_CUDA(cudaMemsetAsync(n->d_loss, 0, sizeof(float), s));
  // loss = sum_p mask_p |y_p - t_p|^2 / (3 N H W)
  if ((e = head(n, N, nullptr, d_target, d_mask, 1.f / (3.f * (float)npix(n, N, 0)), s))) return e;
  if ((e = backward(n, N, s))) return e;
  if (apply) {
    n->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
    k_adam<<<grid_for(n->nparam), 256, 0, s>>>(n->P, n->M, n->V, n->G, n->nparam, lr, b1, b2, c1, c2, 1e-8f);
    if ((e = refresh_weights(n, s))) return e;
  }
  UN_CUDA(cudaMemcpyAsync(n->h_loss, n->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  UN_CUDA(cudaStreamSynchronize(s));
  if (loss) *loss = *n->h_loss;
  return MB_OK;
}
