// kernels.cuh - sm_100a kernels of the multi-block D2Q9 BGK step.
//
// Storage precisions (template parameter P):
//   MB_PREC_F64  : double storage, double arithmetic (the reference's precision)
//   MB_PREC_F32  : float storage, float arithmetic
//   MB_PREC_F16S : half storage of h = f - w_k, float arithmetic in the
//                  shifted variables (rho = 1 + sum h)
// Distributions live in structure-of-arrays planes: element (k, cell) of a
// block is F[k*plane + j*pitch + i] with pitch a multiple of 128 bytes.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mblbm.h"

namespace mblbm {
namespace dev {

// D2Q9 lattice (lbm/lbm.h:43-45); folded into immediates by unrolled loops
__host__ __device__ constexpr int ex(int k) { return k == 1 || k == 5 || k == 8 ? 1 : (k == 3 || k == 6 || k == 7 ? -1 : 0); }
__host__ __device__ constexpr int ey(int k) { return k == 2 || k == 5 || k == 6 ? 1 : (k == 4 || k == 7 || k == 8 ? -1 : 0); }
__host__ __device__ constexpr int opp(int k) { return k == 0 ? 0 : (k <= 4 ? ((k + 1) & 3) + 1 : ((k - 3) & 3) + 5); }
__host__ __device__ constexpr double wd(int k) { return k == 0 ? 4. / 9 : (k <= 4 ? 1. / 9 : 1. / 36); }

template <int P> struct Prec;
template <> struct Prec<MB_PREC_F64> { using S = double; using R = double; static constexpr bool shifted = false; };
template <> struct Prec<MB_PREC_F32> { using S = float; using R = float; static constexpr bool shifted = false; };
template <> struct Prec<MB_PREC_F16S> { using S = __half; using R = float; static constexpr bool shifted = true; };

template <int P> __device__ __forceinline__ typename Prec<P>::R wk(int k) { return (typename Prec<P>::R)wd(k); }

// value of distribution k from its stored form
template <int P>
__device__ __forceinline__ typename Prec<P>::R ld_f(const typename Prec<P>::S *p, long long idx, int k) {
  if constexpr (Prec<P>::shifted) return __half2float(p[idx]) + wk<P>(k);
  else return p[idx];
}
template <int P>
__device__ __forceinline__ void st_f(typename Prec<P>::S *p, long long idx, int k, typename Prec<P>::R v) {
  if constexpr (Prec<P>::shifted) p[idx] = __float2half_rn(v - wk<P>(k));
  else p[idx] = v;
}

// feq, lbm/assit_func.h:2-9
template <typename R>
__device__ __forceinline__ R feq(int k, R rh, R uxx, R uyy) {
  const R eu = (R)ex(k) * uxx + (R)ey(k) * uyy;
  const R uv = uxx * uxx + uyy * uyy;
  return (R)wd(k) * rh * ((R)1.0 + (R)3.0 * eu + (R)4.5 * eu * eu - (R)1.5 * uv);
}

// ----------------------------------------------------------------------------
// Block step: evolution_area_stb1/2/3 (multi/FH/evolution_block.h:3-126) fused
// into one pull collide-stream pass from buffer Fin into Fout.
// ----------------------------------------------------------------------------
constexpr int STB_MAX_BLOCKS = 16;

struct StbBlk {
  const void *Fin;
  void *Fout;
  void *rho, *ux, *uy;
  const uint8_t *flags;
  int nx, ny, pitch, pad_;
  long long plane;
  long long cell0;  // first linear cell index of this block in the launch
  double rv_tau;
};

struct StbParams {
  int nblk;
  int macro_all;     // write rho/u of every FLUID cell (else only CF_MACRO cells)
  int write_macros;  // 0: never write rho/u (kernel timing only)
  int pad_;
  long long total;   // cells in the launch
  double feqc[9];    // feq(rho0, U0): block-edge FLUID cells and stale f of edge solids
  double rho0, u0x, u0y;
  StbBlk b[STB_MAX_BLOCKS];
};

template <int P>
__global__ void __launch_bounds__(256) k_block_step(const __grid_constant__ StbParams p) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= p.total) return;
  int t = 0;
#pragma unroll 1
  while (t + 1 < p.nblk && g >= p.b[t + 1].cell0) t++;
  const StbBlk &B = p.b[t];
  const int local = int(g - B.cell0);
  const int j = local / B.nx;
  const int i = local - j * B.nx;
  const long long c = (long long)j * B.pitch + i;
  const S *__restrict__ Fin = (const S *)B.Fin;
  S *__restrict__ Fout = (S *)B.Fout;
  const long long plane = B.plane;
  const uint8_t fl = B.flags[c];
  const int type = fl & 3;
  const bool wm = p.write_macros && (p.macro_all || (fl & 8));

  if (type == 0) {  // FLUID
    if (fl & 4) {   // block edge: equilibrium at rho0, U0 (stb2 :47-57), collide keeps it
#pragma unroll
      for (int k = 0; k < 9; k++) st_f<P>(Fout, k * plane + c, k, (R)p.feqc[k]);
      if (wm) {
        ((R *)B.rho)[c] = (R)p.rho0;
        ((R *)B.ux)[c] = (R)p.u0x;
        ((R *)B.uy)[c] = (R)p.u0y;
      }
      return;
    }
    R f[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const long long src = k * plane + c - ((long long)ey(k) * B.pitch + ex(k));
      if constexpr (Prec<P>::shifted) f[k] = __half2float(Fin[src]);  // h = f - w
      else f[k] = Fin[src];
    }
    const R rv = (R)B.rv_tau;
    if constexpr (!Prec<P>::shifted) {
      // Macros (lbm/assit_func.h:23-31)
      R rh = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
      R ux = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
      R uy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
      ux = ux / rh;
      uy = uy / rh;
      if (wm) {
        ((R *)B.rho)[c] = rh;
        ((R *)B.ux)[c] = ux;
        ((R *)B.uy)[c] = uy;
      }
      // BGK, stb3 :103-111 (the forcing term is zero)
#pragma unroll
      for (int k = 0; k < 9; k++) Fout[k * plane + c] = f[k] - (f[k] - feq<R>(k, rh, ux, uy)) * rv;
    } else {
      // same scheme in h = f - w: rho = 1 + sum h, j = sum e h, heq = feq - w
      const R drh = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
      const R rh = (R)1.0 + drh;
      R ux = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
      R uy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
      ux = ux / rh;
      uy = uy / rh;
      if (wm) {
        ((R *)B.rho)[c] = rh;
        ((R *)B.ux)[c] = ux;
        ((R *)B.uy)[c] = uy;
      }
      const R uv = ux * ux + uy * uy;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const R eu = (R)ex(k) * ux + (R)ey(k) * uy;
        const R heq = wk<P>(k) * (drh + rh * ((R)3.0 * eu + (R)4.5 * eu * eu - (R)1.5 * uv));
        Fout[k * plane + c] = __float2half_rn(f[k] - (f[k] - heq) * rv);
      }
    }
    return;
  }
  if (type == 1) {  // SOLID_SBB: pull (stale f = feq(rho0,U0) off-block), then on-node bounce-back
    S fr[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const int id = i - ex(k), jd = j - ey(k);
      if (id >= 0 && id < B.nx && jd >= 0 && jd < B.ny)
        fr[k] = Fin[k * plane + c - ((long long)ey(k) * B.pitch + ex(k))];
      else if constexpr (Prec<P>::shifted)
        fr[k] = __float2half_rn((float)(p.feqc[k] - wd(k)));
      else
        fr[k] = (S)p.feqc[k];
    }
#pragma unroll
    for (int k = 0; k < 9; k++) Fout[k * plane + c] = fr[opp(k)];  // w_k = w_opp(k): raw move is exact
    return;
  }
  // C_BOUNDARY and row padding: untouched by the step, carried to the new buffer
#pragma unroll
  for (int k = 0; k < 9; k++) Fout[k * plane + c] = Fin[k * plane + c];
}

// ----------------------------------------------------------------------------
// Per-block table used by the interface, drag and diagnostic kernels.
// ----------------------------------------------------------------------------
struct IfBlk {
  void *F[2];
  void *rho, *ux, *uy;
  void *upx, *upy;
  const uint8_t *flags;
  int nx, ny, pitch, m;
  long long plane;
  double tau;
};

// ----------------------------------------------------------------------------
// Interface point records: c_c_boundary_transfer, temporal_interpolation,
// c_f_boundary_transfer, f_c_boundary_transfer (multi/FH/assit_multi.h).
// ----------------------------------------------------------------------------
struct RecDev {
  uint8_t type, bits, dst_block, src_block;
  uint8_t m0, m1, m2, pad;
  int32_t dst_cell, src;
};
struct RecParams {
  const RecDev *recs;
  int n, pad_;
  const IfBlk *blk;
  void *slots;
  double tw[4][3];
};

template <int P>
__global__ void __launch_bounds__(256) k_records(const __grid_constant__ RecParams p) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.n) return;
  const RecDev r = p.recs[t];
  const IfBlk &D = p.blk[r.dst_block];
  S *Fd = (S *)D.F[(r.bits >> 1) & 1];
  const long long dc = r.dst_cell;
  const bool wF = r.bits & 4, wM = r.bits & 8;
  if (r.type == 0) {  // same-level copy (assit_multi.h:2-46)
    const IfBlk &A = p.blk[r.src_block];
    const S *Fs = (const S *)A.F[r.bits & 1];
    const long long sc = r.src;
    if (wM) {
      ((R *)D.rho)[dc] = ((const R *)A.rho)[sc];
      ((R *)D.ux)[dc] = ((const R *)A.ux)[sc];
      ((R *)D.uy)[dc] = ((const R *)A.uy)[sc];
    }
    if (wF) {
#pragma unroll
      for (int k = 0; k < 9; k++) Fd[k * D.plane + dc] = Fs[k * A.plane + sc];
    }
    return;
  }
  if (r.type == 1 || r.type == 2) {  // temporal interpolation (:213-247) / c_f (:249-271)
    if (!wF) return;
    const R *s = (const R *)p.slots + (long long)r.src * 27;
    if (r.type == 1) {
      const int wi = (r.bits >> 4) & 3;
      const R a = (R)p.tw[wi][0], b = (R)p.tw[wi][1], cc = (R)p.tw[wi][2];
#pragma unroll
      for (int k = 0; k < 9; k++)
        st_f<P>(Fd, k * D.plane + dc, k, a * s[r.m0 * 9 + k] - b * s[r.m1 * 9 + k] + cc * s[r.m2 * 9 + k]);
    } else {
#pragma unroll
      for (int k = 0; k < 9; k++) st_f<P>(Fd, k * D.plane + dc, k, s[r.m2 * 9 + k]);
    }
    return;
  }
  // f_c (:273-314): coarse edge <- fine point, f_neq scaled by r (tau_c-1)/(tau_f-1)
  const IfBlk &Fb = p.blk[r.src_block];
  const S *Fs = (const S *)Fb.F[r.bits & 1];
  const long long sc = r.src;
  const R rh = ((const R *)Fb.rho)[sc], ux = ((const R *)Fb.ux)[sc], uy = ((const R *)Fb.uy)[sc];
  if (wM) {
    ((R *)D.rho)[dc] = rh;
    ((R *)D.ux)[dc] = ux;
    ((R *)D.uy)[dc] = uy;
  }
  if (wF) {
    const R para = (R)((double)(Fb.m / D.m) * (D.tau - 1.0) / (Fb.tau - 1.0));
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const R ft = ld_f<P>(Fs, k * Fb.plane + sc, k);
      const R fe = feq<R>(k, rh, ux, uy);
      st_f<P>(Fd, k * D.plane + dc, k, fe + para * (ft - fe));
    }
  }
}

// ----------------------------------------------------------------------------
// Spatial interpolation: init_Spline3 + tridiagonal solve + calculate_Spline3_gpu
// (assit_multi.h:48-211) for one coarse-fine line per CTA.
// ----------------------------------------------------------------------------
struct SplLineDev {
  int coarse, fine, Nc, Nf, r;
  int ci0, cj0, cdi, cdj;
  int fi0, fj0, fdi, fdj;
  int slot0;
  double para;
};
struct SplTaskDev {
  int line, src_buf, m0, mask_off;
};
struct SplParams {
  const SplTaskDev *tasks;
  const SplLineDev *lines;
  const uint8_t *mask;
  const IfBlk *blk;
  void *slots;
};

// Spline3_S (:118-134), with its 0.1666667 constant
template <typename R>
__device__ __forceinline__ R spline3_s(R xx, R x_1, R h, R fi_1, R fi, R mi_1, R mi) {
  const R x = x_1 + h;
  const R s6 = (R)0.1666667;
  const R a = mi_1 * (x - xx) * (x - xx) * (x - xx) * s6;
  const R b = mi * (xx - x_1) * (xx - x_1) * (xx - x_1) * s6;
  const R c = (fi_1 - mi_1 * h * h * s6) * (x - xx);
  const R d = (fi - mi * h * h * s6) * (xx - x_1);
  return a + b + c + d;
}

// gather the 12 fields (rho, ux, uy, F0..F8) of coarse point ip
template <int P>
__device__ __forceinline__ void spl_gather(const SplLineDev &L, const IfBlk &C, const typename Prec<P>::S *Fc,
                                           int ip, typename Prec<P>::R *v) {
  using R = typename Prec<P>::R;
  const long long c = (long long)(L.cj0 + ip * L.cdj) * C.pitch + (L.ci0 + ip * L.cdi);
  v[0] = ((const R *)C.rho)[c];
  v[1] = ((const R *)C.ux)[c];
  v[2] = ((const R *)C.uy)[c];
#pragma unroll
  for (int k = 0; k < 9; k++) v[3 + k] = ld_f<P>(Fc, k * C.plane + c, k);
}

constexpr int SPL_THREADS = 1024;

// Parallel cyclic reduction of A x_{i-1} + B x_i + C x_{i+1} = D_i for the 12
// right-hand sides at once; the matrix is (0.5, 2, 0.5) with the decoupled
// natural end rows of init_tri_A (multi/init_multi.h:30-51).  ROWS rows per
// thread; shared memory holds A, B, C and D (15 N values).
template <int P, int ROWS>
__global__ void __launch_bounds__(SPL_THREADS) k_spline(const __grid_constant__ SplParams p) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SplTaskDev task = p.tasks[blockIdx.x];
  const SplLineDev L = p.lines[task.line];
  const int N = L.Nc;
  R *A = (R *)smem_raw;
  R *Bd = A + N;
  R *Cu = Bd + N;
  R *D = Cu + N;  // D[f*N + i]
  const IfBlk &C = p.blk[L.coarse];
  const S *Fc = (const S *)C.F[task.src_buf];
  const int tid = threadIdx.x;

  // gather (the race-free reading of init_Spline3 :54-80)
  for (int i = tid; i < N; i += blockDim.x) {
    R v[12];
    spl_gather<P>(L, C, Fc, i, v);
#pragma unroll
    for (int f = 0; f < 12; f++) D[f * N + i] = v[f];
  }
  __syncthreads();
  // right-hand sides 6 f_i - 3 f_{i-1} - 3 f_{i+1}, zero at both ends (:82-107)
  R rhs[ROWS][12];
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const int i = tid + q * blockDim.x;
#pragma unroll
    for (int f = 0; f < 12; f++) {
      R v = 0;
      if (i > 0 && i < N - 1) v = ((R)6.0 * D[f * N + i] - (R)3.0 * D[f * N + i - 1] - (R)3.0 * D[f * N + i + 1]);
      rhs[q][f] = v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const int i = tid + q * blockDim.x;
    if (i < N) {
      A[i] = (i == 0 || i == 1 || i == N - 1) ? (R)0 : (R)0.5;
      Cu[i] = (i == 0 || i == N - 2 || i == N - 1) ? (R)0 : (R)0.5;
      Bd[i] = (R)2.0;
#pragma unroll
      for (int f = 0; f < 12; f++) D[f * N + i] = rhs[q][f];
    }
  }
  __syncthreads();
  for (int s = 1; s < N; s <<= 1) {
    R na[ROWS], nb[ROWS], nc[ROWS];
#pragma unroll
    for (int q = 0; q < ROWS; q++) {
      const int i = tid + q * blockDim.x;
      if (i >= N) continue;
      const R a = A[i], c = Cu[i];
      R al = 0, ga = 0, aa = 0, cc = 0, bb = Bd[i];
      if (i - s >= 0) { al = -a / Bd[i - s]; aa = al * A[i - s]; bb += al * Cu[i - s]; }
      if (i + s < N) { ga = -c / Bd[i + s]; cc = ga * Cu[i + s]; bb += ga * A[i + s]; }
      na[q] = aa;
      nb[q] = bb;
      nc[q] = cc;
#pragma unroll
      for (int f = 0; f < 12; f++) {
        R d = D[f * N + i];
        if (i - s >= 0) d += al * D[f * N + i - s];
        if (i + s < N) d += ga * D[f * N + i + s];
        rhs[q][f] = d;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < ROWS; q++) {
      const int i = tid + q * blockDim.x;
      if (i >= N) continue;
      A[i] = na[q];
      Bd[i] = nb[q];
      Cu[i] = nc[q];
#pragma unroll
      for (int f = 0; f < 12; f++) D[f * N + i] = rhs[q][f];
    }
    __syncthreads();
  }
  for (int i = tid; i < N; i += blockDim.x) {
    const R inv = Bd[i];
#pragma unroll
    for (int f = 0; f < 12; f++) D[f * N + i] = D[f * N + i] / inv;
  }
  __syncthreads();

  // evaluate at the fine points (calculate_Spline3_gpu :136-185)
  const IfBlk &Fb = p.blk[L.fine];
  R *slots = (R *)p.slots;
  const R para = (R)L.para;
  for (int ip = tid; ip < L.Nf; ip += blockDim.x) {
    const R xx = (R)ip / (R)L.r;
    int I = (int)ceil(xx);
    if (I == 0) I = 1;
    R v0[12], v1[12];
    spl_gather<P>(L, C, Fc, I - 1, v0);
    spl_gather<P>(L, C, Fc, I, v1);
    R out[12];
#pragma unroll
    for (int f = 0; f < 12; f++)
      out[f] = spline3_s<R>(xx, (R)(I - 1), (R)1.0, v0[f], v1[f], D[f * N + I - 1], D[f * N + I]);
    const long long fc = (long long)(L.fj0 + ip * L.fdj) * Fb.pitch + (L.fi0 + ip * L.fdi);
    if (task.mask_off < 0 || p.mask[task.mask_off + ip]) {
      ((R *)Fb.rho)[fc] = out[0];
      ((R *)Fb.ux)[fc] = out[1];
      ((R *)Fb.uy)[fc] = out[2];
    }
    R *sl = slots + ((long long)(L.slot0 + ip) * 3 + task.m0) * 9;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const R fe = feq<R>(k, out[0], out[1], out[2]);
      sl[k] = fe + para * (out[3 + k] - fe);
    }
  }
}

// ----------------------------------------------------------------------------
// Momentum-exchange drag (lbm/force_block.h:129-216) over stored links, from
// the buffer the last block step read: the post-stream f of the solid cell in
// direction k is F_k(x_f) and that of the fluid neighbour in opp(k) is
// F_opp(x_s) (or feq(rho0,U0) when the neighbour is a block-edge FLUID cell).
// One CTA, FP64 sums in a fixed order.
// ----------------------------------------------------------------------------
struct DragLink {
  int32_t cell_s, cell_f;
  int32_t k, fluid_edge;
};
struct DragParams {
  const DragLink *links;
  int n, pad_;
  const void *F;  // buffer read by the last block step of the drag block
  long long plane;
  double feqc[9];
  double *out;  // Fx, Fy
};

template <int P>
__global__ void __launch_bounds__(1024) k_drag(const __grid_constant__ DragParams p) {
  using S = typename Prec<P>::S;
  const S *F = (const S *)p.F;
  double fx = 0, fy = 0;
  for (int t = threadIdx.x; t < p.n; t += blockDim.x) {
    const DragLink L = p.links[t];
    const int k = L.k;
    int kd = 0;
    double ek = 0, ekd = 0, eky = 0, ekdy = 0;
#pragma unroll
    for (int q = 0; q < 9; q++)
      if (q == k) { kd = opp(q); ek = ex(q); eky = ey(q); ekd = ex(opp(q)); ekdy = ey(opp(q)); }
    const double fs = (double)ld_f<P>(F, (long long)k * p.plane + L.cell_f, k);
    const double ff = L.fluid_edge ? p.feqc[kd] : (double)ld_f<P>(F, (long long)kd * p.plane + L.cell_s, kd);
    fx += fs * ek - ff * ekd;
    fy += fs * eky - ff * ekdy;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_down_sync(0xffffffffu, fx, o);
    fy += __shfl_down_sync(0xffffffffu, fy, o);
  }
  __shared__ double sx[32], sy[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sx[w] = fx; sy[w] = fy; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ax = 0, ay = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) { ax += sx[q]; ay += sy[q]; }
    p.out[0] = ax;
    p.out[1] = ay;
  }
}

// ----------------------------------------------------------------------------
// Relative L2 change of u (lbm/error_L2.h:3-91) over every cell of every
// block, weighted 1/m per block; u_prev <- u.  Each CTA writes an FP64 partial
// pair to scratch; the last CTA to finish (ticket counter) sums the partials
// in CTA order and resets the ticket, so the result is deterministic.
// ----------------------------------------------------------------------------
struct L2Blk {
  long long cell0;
  int nx, pitch;
  double inv_m;
};
struct L2Params {
  const L2Blk *blocks;
  const IfBlk *blk;
  int nblk, pad_;
  long long total;
  double2 *partial;       // gridDim.x entries
  unsigned int *ticket;   // zero before the first launch; reset by the last CTA
  double *out;            // sum |u-up|^2 / m, sum |u|^2 / m
};

template <int P>
__global__ void __launch_bounds__(256) k_error_l2(const __grid_constant__ L2Params p) {
  using R = typename Prec<P>::R;
  double s1 = 0, s2 = 0;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < p.total;
       g += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = p.nblk - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.blocks[mid].cell0 <= g) lo = mid; else hi = mid - 1;
    }
    const L2Blk &b = p.blocks[lo];
    const IfBlk &B = p.blk[lo];
    const int local = int(g - b.cell0);
    const int j = local / b.nx, i = local - j * b.nx;
    const long long c = (long long)j * b.pitch + i;
    const double ux = ((const R *)B.ux)[c], uy = ((const R *)B.uy)[c];
    const double upx = ((const R *)B.upx)[c], upy = ((const R *)B.upy)[c];
    s1 += ((ux - upx) * (ux - upx) + (uy - upy) * (uy - upy)) * b.inv_m;
    s2 += (ux * ux + uy * uy) * b.inv_m;
    ((R *)B.upx)[c] = (R)ux;
    ((R *)B.upy)[c] = (R)uy;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  __shared__ double a1[8], a2[8];
  __shared__ bool last;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { a1[w] = s1; a2[w] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t1 = 0, t2 = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) { t1 += a1[q]; t2 += a2[q]; }
    p.partial[blockIdx.x] = make_double2(t1, t2);
    __threadfence();
    const unsigned int done = atomicAdd(p.ticket, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t1 = 0, t2 = 0;
    for (unsigned int q = 0; q < gridDim.x; q++) {
      const double2 v = __ldcg(&p.partial[q]);
      t1 += v.x;
      t2 += v.y;
    }
    p.out[0] = t1;
    p.out[1] = t2;
    *p.ticket = 0u;
  }
}

// ----------------------------------------------------------------------------
// Utility kernels: fill, finite check, field conversion.
// ----------------------------------------------------------------------------
template <typename T>
__global__ void k_fill(T *p, long long n, T v) {
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x)
    p[g] = v;
}

template <int P>
__global__ void k_fill_planes(typename Prec<P>::S *F, long long plane, double f0, double f1, double f2, double f3,
                              double f4, double f5, double f6, double f7, double f8) {
  const double fv[9] = {f0, f1, f2, f3, f4, f5, f6, f7, f8};
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < 9 * plane;
       g += (long long)gridDim.x * blockDim.x) {
    const int k = int(g / plane);
    st_f<P>(F, g, k, (typename Prec<P>::R)fv[k]);
  }
}

template <int P>
__global__ void k_count_nonfinite(const typename Prec<P>::S *F, long long plane, const uint8_t *flags, int nx,
                                  int ny, int pitch, unsigned long long *count) {
  unsigned long long bad = 0;
  const long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int j = int(g / nx), i = int(g - (long long)j * nx);
    const long long c = (long long)j * pitch + i;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const double v = (double)ld_f<P>(F, k * plane + c, k);
      if (!isfinite(v)) bad++;
    }
  }
  if (bad) atomicAdd(count, bad);
}

// pitched device planes <-> dense FP64 staging buffer
template <int P>
__global__ void k_planes_to_f64(const typename Prec<P>::S *F, long long plane, int nx, int ny, int pitch, double *out) {
  const long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < 9 * n; g += (long long)gridDim.x * blockDim.x) {
    const int k = int(g / n);
    const long long r = g - k * n;
    const int j = int(r / nx), i = int(r - (long long)j * nx);
    out[g] = (double)ld_f<P>(F, k * plane + (long long)j * pitch + i, k);
  }
}
template <int P>
__global__ void k_f64_to_planes(typename Prec<P>::S *F, long long plane, int nx, int ny, int pitch, const double *in) {
  const long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < 9 * n; g += (long long)gridDim.x * blockDim.x) {
    const int k = int(g / n);
    const long long r = g - k * n;
    const int j = int(r / nx), i = int(r - (long long)j * nx);
    st_f<P>(F, k * plane + (long long)j * pitch + i, k, (typename Prec<P>::R)in[g]);
  }
}
template <typename R>
__global__ void k_field_to_f64(const R *M, int nx, int ny, int pitch, double *out) {
  const long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int j = int(g / nx), i = int(g - (long long)j * nx);
    out[g] = (double)M[(long long)j * pitch + i];
  }
}
template <typename R>
__global__ void k_f64_to_field(R *M, int nx, int ny, int pitch, const double *in) {
  const long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int j = int(g / nx), i = int(g - (long long)j * nx);
    M[(long long)j * pitch + i] = (R)in[g];
  }
}

}  // namespace dev
}  // namespace mblbm
