// kernels.cuh - sm_100a kernels of the multi-block D2Q9 BGK step.
//
// Storage precisions (template parameter P):
//   MB_PREC_F64  : double storage, double arithmetic (the reference's precision)
//   MB_PREC_F32  : float storage of h = f - w_k, float arithmetic in the
//                  shifted variables (rho = 1 + sum h)
//   MB_PREC_F16S : half storage of h = f - w_k, float arithmetic as above
//   MB_PREC_F32U : float storage of f itself, float arithmetic
//   MB_PREC_F16C : 16-bit storage of h = f - w_k in the format h16c below
//                  (3 exponent and 12 fraction bits), float arithmetic
// Distributions live in structure-of-arrays planes: element (k, cell) of a
// block is F[k*plane + j*pitch + i] with pitch a multiple of 128 bytes.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/mblbm.h"

namespace mblbm {
namespace dev {

// D2Q9 lattice (lbm/lbm.h:43-45); folded into immediates by unrolled loops
__host__ __device__ constexpr int ex(int k) { return k == 1 || k == 5 || k == 8 ? 1 : (k == 3 || k == 6 || k == 7 ? -1 : 0); }
__host__ __device__ constexpr int ey(int k) { return k == 2 || k == 5 || k == 6 ? 1 : (k == 4 || k == 7 || k == 8 ? -1 : 0); }
__host__ __device__ constexpr int opp(int k) { return k == 0 ? 0 : (k <= 4 ? ((k + 1) & 3) + 1 : ((k - 3) & 3) + 5); }
__host__ __device__ constexpr int slip(int k) { return k == 2 ? 4 : k == 4 ? 2 : k == 5 ? 8 : k == 8 ? 5 : k == 6 ? 7 : k == 7 ? 6 : k; }
__host__ __device__ constexpr double wd(int k) { return k == 0 ? 4. / 9 : (k <= 4 ? 1. / 9 : 1. / 36); }

// Stored word of MB_PREC_F16C: sign, a 3-bit exponent E and a 12-bit fraction
// M.  E = 1..7 holds +-2^(E-10) (1 + M/4096), magnitudes in [2^-9, 2^-2);
// E = 0 holds +-2^-9 M/4096 (spacing 2^-21).  Against IEEE binary16 the
// shifted distributions |h| < 1/4 keep two more fraction bits: the spacing
// is 1/4 of binary16's at every |h| >= 2^-9 and at most 1/2 of it below.
// Conversion rounds to nearest (ties to even); magnitudes of 1/4 and above,
// Inf and NaN saturate to the largest code 0x7fff (with their sign), which
// mb_check_finite counts as bad.
struct __align__(2) h16c { unsigned short x; };
struct __align__(4) h16c2 { unsigned int x; };  // two codes, the lower one first in memory

template <int P> struct Prec;
template <> struct Prec<MB_PREC_F64> { using S = double; using R = double; static constexpr bool shifted = false; };
template <> struct Prec<MB_PREC_F32> { using S = float; using R = float; static constexpr bool shifted = true; };
template <> struct Prec<MB_PREC_F16S> { using S = __half; using R = float; static constexpr bool shifted = true; };
template <> struct Prec<MB_PREC_F32U> { using S = float; using R = float; static constexpr bool shifted = false; };
template <> struct Prec<MB_PREC_F16C> { using S = h16c; using R = float; static constexpr bool shifted = true; };

template <int P> __device__ __forceinline__ typename Prec<P>::R wk(int k) { return (typename Prec<P>::R)wd(k); }

// The shift of the shifted precisions: the stored word of direction k is
// h_k = f_k - s_k, with s = feq(rho_s, U_s) for constants rho_s, U_s (s = w:
// rho_s = 1, U_s = 0; s = feq(rho0, U0): the free stream).  The collision
// works on h directly: rho = rho_s + sum h, rho u = J_s + sum e h (J_s =
// rho_s U_s), and feq_k - s_k = w_k (d + 3 e.J_h + rho (4.5 (e.u)^2 - 1.5 u^2))
// + c_k with d = sum h, J_h = sum e h and c_k = w_k (rho_s + 3 e_k.J_s) - s_k,
// which depends on the direction pair only (zero for s = w).
struct Sh9 { float s[9]; };
struct Shift {
  Sh9 v;              // s_k
  float c[5];         // c_k for k = 0, the pairs (1,3), (2,4), (5,7) and (8,6)
  float rhos, jx, jy; // rho_s, J_s
  float q2, qd, qx;   // rho_s |U_s|^2, rho_s (Usx^2 - Usy^2), rho_s Usx Usy (MRT)
  int sym;            // s_k = s_opp(k) = s_slip(k): walls move stored words unchanged
  int sr;             // h16c: the collision rounds its outputs to the stored grid stochastically
};

// stored word <-> arithmetic type
__device__ __forceinline__ float to_r(__half h) { return __half2float(h); }
__device__ __forceinline__ float to_r(float v) { return v; }
__device__ __forceinline__ double to_r(double v) { return v; }
template <typename S> __device__ __forceinline__ S from_r(float v);
template <> __device__ __forceinline__ __half from_r<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ float from_r<float>(float v) { return v; }
template <typename S> __device__ __forceinline__ S from_r(double v) { return (S)v; }

// h16c codec.  Decode: the code shifted into an FP32 bit pattern (E into the
// exponent field, M into the top fraction bits; E = 0 lands on FP32
// subnormals, which keep the same linear spacing), scaled by 2^117.
__device__ __forceinline__ float h16c_decode(unsigned int u) {
  const unsigned int bits = ((u & 0x7fffu) << 11) | ((u & 0x8000u) << 16);
  return __uint_as_float(bits) * 0x1p117f;
}
// Encode: scale by 2^-117 (exact for |v| >= 2^-9; below, the product is
// rounded to the FP32 subnormal grid 2^-149, 2^-11 of the code's spacing
// there, so the result is the nearest code up to that much), then round the
// 11 dropped fraction bits to nearest even with an integer add (the carry
// moves into the exponent across binade and subnormal boundaries alike),
// saturating.
__device__ __forceinline__ unsigned int h16c_encode(float v) {
  const unsigned int b = __float_as_uint(v * 0x1p-117f);
  const unsigned int mag = b & 0x7fffffffu;
  unsigned int r = mag >= 0x7f800000u ? 0x7fffu : (mag + 0x3ffu + ((mag >> 11) & 1u)) >> 11;
  r = r < 0x7fffu ? r : 0x7fffu;
  return r | ((b >> 16) & 0x8000u);
}
__device__ __forceinline__ float to_r(h16c h) { return h16c_decode(h.x); }
// Random word of a cell for stochastic rounding: a hash of the cell's
// identity (block index and position) and of three of its inputs, whose low
// bits change whenever the state of the cell or its neighbours does; so the
// dither is the same in every kernel variant and execution mode.  Two
// multiply-xorshift rounds mix it.
__device__ __forceinline__ unsigned int sr_seed(unsigned int key, const float *f) {
  unsigned int h = key * 0x9E3779B1u + __float_as_uint(f[0]);
  h = (h ^ (h >> 15)) * 0x2C1B3C6Du;
  h += __float_as_uint(f[5]) ^ __float_as_uint(f[7]);
  h = (h ^ (h >> 12)) * 0x297A2D39u;
  return h ^ (h >> 15);
}
// odd multipliers that spread a cell's random word over its outputs
__host__ __device__ constexpr unsigned int sr_mul(int q) {
  return q == 0 ? 0x9E3779B1u : q == 1 ? 0x85EBCA77u : q == 2 ? 0xC2B2AE3Du : q == 3 ? 0x27D4EB2Fu
       : q == 4 ? 0x165667B1u : q == 5 ? 0xD3A2646Du : q == 6 ? 0xFD7046C5u : q == 7 ? 0xB55A4F09u : 0x2C1B3C6Du;
}
// v rounded to one of its two neighbouring h16c values, the upper one with
// probability (v - lower) / (upper - lower): the 11 dropped fraction bits get
// the 11 low bits of r added before truncation.  Returns the code's value.
__device__ __forceinline__ float h16c_round_sr(float v, unsigned int r) {
  const unsigned int b = __float_as_uint(v * 0x1p-117f);
  const unsigned int mag = b & 0x7fffffffu;
  unsigned int c = mag >= 0x7f800000u ? 0x7fffu : (mag + (r & 0x7ffu)) >> 11;
  c = c < 0x7fffu ? c : 0x7fffu;
  return h16c_decode(c | ((b >> 16) & 0x8000u));
}
template <> __device__ __forceinline__ h16c from_r<h16c>(float v) { return h16c{(unsigned short)h16c_encode(v)}; }
template <> __device__ __forceinline__ h16c from_r<h16c>(double v) { return from_r<h16c>((float)v); }

// value of distribution k from its stored form (shifted forms store f - w_k)
template <int P>
__device__ __forceinline__ typename Prec<P>::R ld_f(const typename Prec<P>::S *p, long long idx, int k, const Sh9 &sh) {
  if constexpr (Prec<P>::shifted) return to_r(p[idx]) + sh.s[k];
  else return p[idx];
}
template <int P>
__device__ __forceinline__ void st_f(typename Prec<P>::S *p, long long idx, int k, typename Prec<P>::R v,
                                     const Sh9 &sh) {
  if constexpr (Prec<P>::shifted) p[idx] = from_r<typename Prec<P>::S>(v - sh.s[k]);
  else p[idx] = v;
}
// the stored word of f_k = x given in FP64 (an equilibrium, a stale value)
template <int P>
__device__ __forceinline__ typename Prec<P>::S stored_of(double x, int k, const Sh9 &sh) {
  if constexpr (Prec<P>::shifted) return from_r<typename Prec<P>::S>((float)(x - (double)sh.s[k]));
  else return (typename Prec<P>::S)x;
}
// the stored word of f_k when f_k equals f_j of a stored word v (a wall
// returning another direction's value): v itself when s_k = s_j
template <int P>
__device__ __forceinline__ typename Prec<P>::S moved(typename Prec<P>::S v, int j, int k, const Shift &sh) {
  if constexpr (Prec<P>::shifted) {
    if (sh.sym) return v;
    return from_r<typename Prec<P>::S>(to_r(v) + (sh.v.s[j] - sh.v.s[k]));
  } else {
    return v;
  }
}

// Global loads and stores with an optional evict-first cache hint (.cs):
// the coarse level streams several hundred MB per step and, hinted, leaves
// the fine levels' buffers resident in L2.
template <bool EF, typename T> __device__ __forceinline__ T ld_ef(const T *p) {
  if constexpr (EF) {
    if constexpr (std::is_same<T, h16c>::value) {
      return h16c{__ldcs((const unsigned short *)p)};
    } else if constexpr (std::is_same<T, h16c2>::value) {
      return h16c2{__ldcs((const unsigned int *)p)};
    } else {
      return __ldcs(p);
    }
  } else {
    return *p;
  }
}
template <bool EF, typename T> __device__ __forceinline__ void st_ef(T *p, T v) {
  if constexpr (EF) {
    if constexpr (std::is_same<T, h16c>::value) __stcs((unsigned short *)p, v.x);
    else if constexpr (std::is_same<T, h16c2>::value) __stcs((unsigned int *)p, v.x);
    else __stcs(p, v);
  } else {
    *p = v;
  }
}

// Programmatic dependent launch: a kernel lets the next one in the graph be
// scheduled as soon as every CTA has started (pdl_trigger), and waits for its
// own producers to finish and flush (pdl_wait) before it reads their output.
// Both are no-ops when the launch has no programmatic dependency.
__device__ __forceinline__ void pdl_trigger() { cudaTriggerProgrammaticLaunchCompletion(); }
__device__ __forceinline__ void pdl_wait() { cudaGridDependencySynchronize(); }

// temporal_interpolation (multi/FH/assit_multi.h:213-247) of one direction
// from the three ring slots s0, s1, s2 of a fine point: one expression for
// the record kernel and the spline's fused form, so both round alike
template <typename R>
__device__ __forceinline__ R temporal3(R a, R b, R c, R s0, R s1, R s2) {
  return a * s0 - b * s1 + c * s2;
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
constexpr uint8_t FL_CCPULL = 64;  // C_BOUNDARY target of a same-level copy run beside the block step
constexpr uint8_t FL_TSKIP = 128;  // fine edge cell a spline writes for the next substep (StbParams::tskip)

struct StbBlk {
  const void *Fin;
  void *Fout;
  void *rho, *ux, *uy;
  const uint8_t *flags;
  int nx, ny, pitch, gid;  // gid: the block's index in its context
  long long plane;
  long long cell0;  // first linear cell index of this block in the launch (per-cell kernel)
  double rv_tau;
  long long wt0;    // first warp tile of this block in the launch (quad kernel)
  int tiles_x, row0;  // quad kernel: tiles of 128 cells per row; first row of the region (quad and row kernels)
  // range kernel: this block's cells of the region are CTAs cta0.. of the
  // launch, 256 consecutive cells (row-major over the region) per CTA
  int cta0, rcells;   // first CTA; cells of the region
  int rw, rcol0;      // region width and first column (first row: row0)
  float rinv_w;       // 1 / rw, for the row of a cell index
  // pair kernel: pairs of cells (i, i + 1), i - rcol0 even; ppr pairs per
  // row, CTAs pcta0.. of 256 consecutive pairs
  int pcta0, npairs;
  int ppr;
  float pinv;         // 1 / ppr
  // bulk-copy kernel (interior region): items tb0.. of 256 cells of one row,
  // tb_tiles per row (tiles start at column 0, multiples of 256)
  long long tb0;
  int tb_tiles, pad3_;
  int pad2_;
  double dt;          // 1 / m: time step of the block in coarse units (body-force term)
};
// a cell's identity for the stochastic rounding of h16c: block index and cell
__device__ __forceinline__ unsigned int cell_key(const StbBlk &B, int i, int j) {
  return (unsigned int)B.gid * 0x01000193u + (unsigned int)(j * B.nx + i);
}

// One same-level copy run beside the block step (k_cc_pull).
struct CcEntry {
  int tblk, sblk;  // global block ids
  int tcell;       // target cell, j * pitch + i
  int si, sj;      // source cell
  int pad_;
};

// Collision and boundary options (the options kernel k_block_step_x only).
struct StbOptions {
  int coll;         // MB_COLL_BGK or MB_COLL_MRT
  int has_force;    // body force non-zero
  double mrt_s[3];  // s_e, s_eps, s_q; <= 0: the block's 1/tau
  double force[2];  // forcex, forcey of every cell
};

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

// An f_c point (f_c_boundary_transfer, multi/FH/assit_multi.h:273-314) done
// beside the block step that updates its fine cell (k_fc_pull): block gid's
// cell `cell` (flagged FL_FCSRC) gives coarse cell dcell of block dblk, F in
// buffer dbuf, feq + para (f - feq) of its new values, and its rho/u.
struct StbFc {
  int gid, cell, dblk, dcell;
  int bits, dbuf;  // bits: 4 write F, 8 write rho/u
  double para;
};
constexpr uint8_t FL_FCSRC = 16;  // FLUID: fine point of an f_c line (on SOLID cells the bit marks a half-way wall)
// A cell k_fc_pull updates: block gid, (i, j), and its f_c points fc[e0, e1).
struct FcCell {
  int gid, i, j, e0, e1, pad_;
};

struct StbParams {
  int nblk;
  int macro_all;     // write rho/u of every FLUID cell (else only CF_MACRO cells)
  int write_macros;  // 0: never write rho/u (kernel timing only)
  int region;        // 0: all cells, 1: distance >= 2 from the block edge, 2: distance <= 1
  int evict_first;   // stream the blocks' buffers with evict-first cache hints
  int ccpull;        // skip cells flagged FL_CCPULL: k_cc_pull writes them
  int a0;            // global index of b[0]
  const CcEntry *cc_list;  // k_cc_pull: the copies of the launch
  int cc_n, pad_cc;
  long long tb_items;      // bulk-copy kernel: items of the launch
  unsigned int *err_host;  // error word (mapped host memory) of bounded waits
  long long total;   // cells in the launch (per-cell kernel) or warp tiles (quad kernel)
  long long rctas;   // CTAs of a range-kernel launch
  long long pctas;   // CTAs of a pair-kernel launch
  double feqc[9];    // feq(rho0, U0): block-edge FLUID cells and stale f of edge solids
  double rho0, u0x, u0y;
  StbOptions opt;
  int tskip;         // leave cells flagged FL_TSKIP alone: a spline writes their next values
  int fcskip;        // leave FLUID cells flagged FL_FCSRC alone: k_fc_pull updates them
  int fc_n;          // k_fc_pull: f_c points (fc, sorted by cell), targets in the block table fcblk
  int fc_cells;      // k_fc_pull: the FL_FCSRC cells it updates (fccell)
  int pad_fc;
  const StbFc *fc;
  const FcCell *fccell;
  const IfBlk *fcblk;
  Shift sh;          // shift of the stored words (shifted precisions)
  StbBlk b[STB_MAX_BLOCKS];
};

// BGK relaxation of a cell in FP32 arithmetic with the equilibria of
// opposite directions paired: for e_k u = +-a,
//   g_k = w_k (base + rh (3 e_k u + 4.5 (e_k u)^2 - 1.5 u^2))
//       = w_k (E +- O),  E = base + rh (4.5 a^2 - 1.5 u^2),  O = 3 rh a,
// with base = rho (plain storage) or rho - 1 (shifted storage, where g_k is
// feq_k - w_k).  Same scheme as feq (lbm/assit_func.h:2-9), fewer operations.
template <bool SHIFTED>
__device__ __forceinline__ void collide_f32(const float *f, float rv, float *out, float *m, const Shift &sh) {
  const float sum = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  const float rh = SHIFTED ? sh.rhos + sum : sum;
  const float base = sum;  // rho - rho_s when shifted, rho otherwise
  const float inv = __frcp_rn(rh);
  const float jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8], jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
  const float ux = (SHIFTED ? jx + sh.jx : jx) * inv;
  const float uy = (SHIFTED ? jy + sh.jy : jy) * inv;
  m[0] = rh;
  m[1] = ux;
  m[2] = uy;
  const float u15 = 1.5f * (ux * ux + uy * uy);
  const float w0 = 4.0f / 9.0f, w1 = 1.0f / 9.0f, w5 = 1.0f / 36.0f;
  const float g0 = w0 * (base - rh * u15) + (SHIFTED ? sh.c[0] : 0.0f);
  out[0] = f[0] + rv * (g0 - f[0]);
  // the odd part 3 w e.(rho u) of a pair, from J_h when shifted (J_s cancels
  // against the shift's own odd part)
  auto pair = [&](float a, float o, float w, float cq, int kp, int km) {
    const float e = w * (base + rh * (4.5f * a * a - u15)) + cq;
    out[kp] = f[kp] + rv * ((e + o) - f[kp]);
    out[km] = f[km] + rv * ((e - o) - f[km]);
  };
  if (SHIFTED) {
    pair(ux, w1 * (3.0f * jx), w1, sh.c[1], 1, 3);
    pair(uy, w1 * (3.0f * jy), w1, sh.c[2], 2, 4);
    pair(ux + uy, w5 * (3.0f * (jx + jy)), w5, sh.c[3], 5, 7);
    pair(ux - uy, w5 * (3.0f * (jx - jy)), w5, sh.c[4], 8, 6);
  } else {
    const float rh3 = 3.0f * rh;
    pair(ux, w1 * (rh3 * ux), w1, 0.0f, 1, 3);
    pair(uy, w1 * (rh3 * uy), w1, 0.0f, 2, 4);
    pair(ux + uy, w5 * (rh3 * (ux + uy)), w5, 0.0f, 5, 7);
    pair(ux - uy, w5 * (rh3 * (ux - uy)), w5, 0.0f, 8, 6);
  }
}

// FLUID interior cell: Macros (lbm/assit_func.h:23-31) and BGK (stb3 :103-111,
// zero forcing term) on pulled values f (f itself, or h = f - w when shifted).
// Writes the new distributions to out and rho/u to m.  FP64 evaluates the
// reference's expressions as written; FP32 arithmetic uses collide_f32.
template <int P>
__device__ __forceinline__ void stb_collide(const typename Prec<P>::R *f, typename Prec<P>::R rv,
                                            typename Prec<P>::R *out, typename Prec<P>::R *m, const Shift &sh,
                                            unsigned int key = 0u) {
  using R = typename Prec<P>::R;
  if constexpr (sizeof(R) == 4) {
    collide_f32<Prec<P>::shifted>(f, rv, out, m, sh);
    // stochastic rounding: each output is rounded here to a value of the
    // stored type, which the store then encodes exactly
    if constexpr (P == MB_PREC_F16C) {
      if (sh.sr) {
        const unsigned int h = sr_seed(key, f);
#pragma unroll
        for (int k = 0; k < 9; k++) out[k] = h16c_round_sr(out[k], (h * sr_mul(k)) >> 21);
      }
    }
    if constexpr (P == MB_PREC_F16S) {
      if (sh.sr) {  // the hardware's stochastic rounding to FP16, two values per instruction
        const unsigned int h = sr_seed(key, f);
#pragma unroll
        for (int q = 0; q < 5; q++) {
          unsigned int r = h * sr_mul(q);
          r ^= r >> 16;
          unsigned int d;
          asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(out[2 * q]), "f"(q < 4 ? out[2 * q + 1] : 0.0f), "r"(r));
          out[2 * q] = __half2float(__ushort_as_half((unsigned short)(d >> 16)));
          if (q < 4) out[2 * q + 1] = __half2float(__ushort_as_half((unsigned short)(d & 0xffffu)));
        }
      }
    }
  } else {
    R rh = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    R ux = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    R uy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
    ux = ux / rh;
    uy = uy / rh;
    m[0] = rh;
    m[1] = ux;
    m[2] = uy;
#pragma unroll
    for (int k = 0; k < 9; k++) out[k] = f[k] - (f[k] - feq<R>(k, rh, ux, uy)) * rv;
  }
}

// Pulled values of cell (i, j): F_k at x - e_k, or the cell's own F_k where
// x - e_k lies outside the block (those values are never used).  They do
// not depend on the cell's flag byte, so the pulls and the flag load share
// one memory round trip.
template <int P, bool EF>
__device__ __forceinline__ void stb_pull(const StbBlk &B, int i, int j, typename Prec<P>::S *raw) {
  using S = typename Prec<P>::S;
  const long long c = (long long)j * B.pitch + i;
  // plain pointers: inside the persistent executor these buffers are written
  // by earlier nodes of the same launch, so no non-coherent (read-only) loads
  const S *Fin = (const S *)B.Fin;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const bool inb = (ex(k) != 1 || i > 0) && (ex(k) != -1 || i < B.nx - 1) && (ey(k) != 1 || j > 0) &&
                     (ey(k) != -1 || j < B.ny - 1);
    const long long off = inb ? ((long long)ey(k) * B.pitch + ex(k)) : 0;
    raw[k] = ld_ef<EF>(Fin + (k * B.plane + c - off));
  }
}

// The f_c points fc[e0, e1) of a fine cell, from its new values out[] and its
// rho/u m[] (f_c_boundary_transfer, multi/FH/assit_multi.h:273-314): what the
// record kernel computes from the same values read back through the stored
// type.
template <int P>
__device__ __forceinline__ void stb_fc_points(const StbParams &p, int e0, int e1, const typename Prec<P>::R *out,
                                              const typename Prec<P>::R *m) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  for (int q = e0; q < e1; q++) {
    const StbFc &e = p.fc[q];
    const IfBlk &D = p.fcblk[e.dblk];
    const R rh = m[0], ux = m[1], uy = m[2];
    if (e.bits & 8) {
      ((R *)D.rho)[e.dcell] = rh;
      ((R *)D.ux)[e.dcell] = ux;
      ((R *)D.uy)[e.dcell] = uy;
    }
    if (e.bits & 4) {
      S *Fd = (S *)D.F[e.dbuf];
      const R para = (R)e.para;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        R ft;  // the stored word read back, as ld_f does
        if constexpr (Prec<P>::shifted) ft = to_r(from_r<S>(out[k])) + p.sh.v.s[k];
        else ft = to_r(from_r<S>(out[k]));
        const R fe = feq<R>(k, rh, ux, uy);
        st_f<P>(Fd, k * D.plane + e.dcell, k, fe + para * (ft - fe), p.sh.v);
      }
    }
  }
}

// The block step of cell (i, j) of block B (stb_finish below) with its new
// values stored at cell cd of block D: a same-level copy target's values.
// cc: the values are a c_c_boundary_transfer copy (multi/FH/assit_multi.h:38-44),
// which also carries rho/u whatever the source's type.
template <int P, bool EF>
__device__ __forceinline__ void stb_finish_at(const StbParams &p, const StbBlk &B, int i, int j,
                                              const typename Prec<P>::S *raw, uint8_t fl, const StbBlk &D,
                                              long long cd, bool cc) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  const long long c = (long long)j * B.pitch + i;
  S *Fout = (S *)D.Fout;
  const long long plane = D.plane;
  const int type = fl & 3;
  const bool wm = cc || (p.write_macros && (p.macro_all || (fl & 8)));

  if (type == 0) {  // FLUID
    if (fl & 4) {   // block edge: equilibrium at rho0, U0 (stb2 :47-57), collide keeps it
#pragma unroll
      for (int k = 0; k < 9; k++) {
        if constexpr (Prec<P>::shifted) st_ef<EF>(Fout + k * plane + cd, from_r<S>((R)p.feqc[k] - p.sh.v.s[k]));
        else st_ef<EF>(Fout + k * plane + cd, (S)p.feqc[k]);
      }
      if (wm) {
        st_ef<EF>((R *)D.rho + cd, (R)p.rho0);
        st_ef<EF>((R *)D.ux + cd, (R)p.u0x);
        st_ef<EF>((R *)D.uy + cd, (R)p.u0y);
      }
      return;
    }
    R f[9];  // interior FLUID cell: every pull is inside the block
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = to_r(raw[k]);
    R out[9], m[3];
    stb_collide<P>(f, (R)B.rv_tau, out, m, p.sh, cell_key(B, i, j));
    if (wm) {
      st_ef<EF>((R *)D.rho + cd, m[0]);
      st_ef<EF>((R *)D.ux + cd, m[1]);
      st_ef<EF>((R *)D.uy + cd, m[2]);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) st_ef<EF>(Fout + k * plane + cd, from_r<S>(out[k]));
    return;
  }
  if (cc) {  // rho/u of a solid or C_BOUNDARY source: its current values
    st_ef<EF>((R *)D.rho + cd, ((const R *)B.rho)[c]);
    st_ef<EF>((R *)D.ux + cd, ((const R *)B.ux)[c]);
    st_ef<EF>((R *)D.uy + cd, ((const R *)B.uy)[c]);
  }
  if (type == 1) {  // SOLID_SBB: pull (stale f = feq(rho0,U0) off-block), then on-node bounce-back
    S fr[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const int id = i - ex(k), jd = j - ey(k);
      fr[k] = (id >= 0 && id < B.nx && jd >= 0 && jd < B.ny) ? raw[k] : stored_of<P>(p.feqc[k], k, p.sh.v);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) st_ef<EF>(Fout + k * plane + cd, moved<P>(fr[opp(k)], opp(k), k, p.sh));
    return;
  }
  // C_BOUNDARY and row padding: untouched by the step, carried to the new buffer
  const S *Fin = (const S *)B.Fin;
#pragma unroll
  for (int k = 0; k < 9; k++) st_ef<EF>(Fout + k * plane + cd, ld_ef<EF>(Fin + k * B.plane + c));
}

// One cell of the block step, evolution_area_stb1/2/3
// (multi/FH/evolution_block.h:3-119), from its pulled values and flag byte.
template <int P, bool EF>
__device__ __forceinline__ void stb_finish(const StbParams &p, const StbBlk &B, int i, int j,
                                           const typename Prec<P>::S *raw, uint8_t fl) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  const long long c = (long long)j * B.pitch + i;
  S *Fout = (S *)B.Fout;
  const long long plane = B.plane;
  const int type = fl & 3;
  const bool wm = p.write_macros && (p.macro_all || (fl & 8));

  if (type == 0) {  // FLUID
    if (p.fcskip && (fl & FL_FCSRC)) return;  // k_fc_pull updates it beside this step
    if (fl & 4) {   // block edge: equilibrium at rho0, U0 (stb2 :47-57), collide keeps it
#pragma unroll
      for (int k = 0; k < 9; k++) {
        if constexpr (Prec<P>::shifted) st_ef<EF>(Fout + k * plane + c, from_r<S>((R)p.feqc[k] - p.sh.v.s[k]));
        else st_ef<EF>(Fout + k * plane + c, (S)p.feqc[k]);
      }
      if (wm) {
        st_ef<EF>((R *)B.rho + c, (R)p.rho0);
        st_ef<EF>((R *)B.ux + c, (R)p.u0x);
        st_ef<EF>((R *)B.uy + c, (R)p.u0y);
      }
      return;
    }
    R f[9];  // interior FLUID cell: every pull is inside the block
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = to_r(raw[k]);
    R out[9], m[3];
    stb_collide<P>(f, (R)B.rv_tau, out, m, p.sh, cell_key(B, i, j));
    if (wm) {
      st_ef<EF>((R *)B.rho + c, m[0]);
      st_ef<EF>((R *)B.ux + c, m[1]);
      st_ef<EF>((R *)B.uy + c, m[2]);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) st_ef<EF>(Fout + k * plane + c, from_r<S>(out[k]));
    return;
  }
  if (type == 1) {  // SOLID_SBB: pull (stale f = feq(rho0,U0) off-block), then on-node bounce-back
    S fr[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const int id = i - ex(k), jd = j - ey(k);
      fr[k] = (id >= 0 && id < B.nx && jd >= 0 && jd < B.ny) ? raw[k] : stored_of<P>(p.feqc[k], k, p.sh.v);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) st_ef<EF>(Fout + k * plane + c, moved<P>(fr[opp(k)], opp(k), k, p.sh));
    return;
  }
  // C_BOUNDARY and row padding: untouched by the step, carried to the new
  // buffer; a same-level copy target (FL_CCPULL) is k_cc_pull's
  if (p.ccpull && (fl & FL_CCPULL)) return;
  if (p.tskip && (fl & FL_TSKIP)) return;
  const S *Fin = (const S *)B.Fin;
#pragma unroll
  for (int k = 0; k < 9; k++) st_ef<EF>(Fout + k * plane + c, ld_ef<EF>(Fin + k * plane + c));
}


// Same-level copies (c_c_boundary_transfer, multi/FH/assit_multi.h:2-46) of a
// level whose sources are FLUID cells, run beside the level's block step
// instead of after it: each thread computes what its source cell gets in this
// step from the source block's input buffer (the block step's own code) and
// stores it, rho/u included, at the target.  The block step skips the
// targets (FL_CCPULL).  Chains of copies are resolved on the host.
template <int P>
__global__ void __launch_bounds__(128) k_cc_pull(const __grid_constant__ StbParams p) {
  pdl_trigger();
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.cc_n) return;
  const CcEntry e = p.cc_list[t];
  const StbBlk &B = p.b[e.sblk - p.a0], &D = p.b[e.tblk - p.a0];
  typename Prec<P>::S raw[9];
  stb_pull<P, false>(B, e.si, e.sj, raw);
  stb_finish_at<P, false>(p, B, e.si, e.sj, raw, B.flags[(long long)e.sj * B.pitch + e.si], D, e.tcell, true);
}



// Pulled values of a cell at least one cell from the block edge: every
// neighbour is inside the block (constant offsets).
template <int P, bool EF>
__device__ __forceinline__ void stb_pull_in(const StbBlk &B, long long c, typename Prec<P>::S *raw) {
  const typename Prec<P>::S *Fin = (const typename Prec<P>::S *)B.Fin;
#pragma unroll
  for (int k = 0; k < 9; k++) raw[k] = ld_ef<EF>(Fin + (k * B.plane + c - ((long long)ey(k) * B.pitch + ex(k))));
}

template <int P, bool EF>
__device__ __forceinline__ void stb_cell_h(const StbParams &p, const StbBlk &B, int i, int j) {
  typename Prec<P>::S raw[9];
  const long long c = (long long)j * B.pitch + i;
  if (i > 0 && i < B.nx - 1 && j > 0 && j < B.ny - 1) {
    stb_pull_in<P, EF>(B, c, raw);  // issued together with the flag load
    stb_finish<P, EF>(p, B, i, j, raw, B.flags[c]);
  } else {
    stb_pull<P, EF>(B, i, j, raw);
    stb_finish<P, EF>(p, B, i, j, raw, B.flags[c]);
  }
}

template <int P>
__device__ __forceinline__ void stb_cell(const StbParams &p, const StbBlk &B, int i, int j) {
  stb_cell_h<P, false>(p, B, i, j);
}

// The FL_FCSRC cells of a fine level's block step, updated beside it (the
// step leaves them alone: StbParams::fcskip) by the step's own per-cell
// code, then their f_c points from the values read back: what reads the
// coarse cells of those points waits for this small launch instead of the
// whole fine step.  One thread per cell.
template <int P>
__global__ void __launch_bounds__(128) k_fc_pull(const __grid_constant__ StbParams p) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  pdl_trigger();
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.fc_cells) return;
  const FcCell e = p.fccell[t];
  const StbBlk &B = p.b[e.gid - p.a0];
  stb_cell_h<P, false>(p, B, e.i, e.j);  // the step's own code (this launch's fcskip is 0)
  // its points read the cell back, as the record kernel does
  const long long c = (long long)e.j * B.pitch + e.i;
  const S *Fo = (const S *)B.Fout;
  R out[9], m[3];
#pragma unroll
  for (int k = 0; k < 9; k++) out[k] = to_r(Fo[k * B.plane + c]);
  m[0] = ((const R *)B.rho)[c];
  m[1] = ((const R *)B.ux)[c];
  m[2] = ((const R *)B.uy)[c];
  stb_fc_points<P>(p, e.e0, e.e1, out, m);
}

// Cell g (0 <= g < p.total) of a block-step launch: its block t and its
// (i, j) in the launch's region.
__device__ __forceinline__ void stb_locate(const StbParams &p, long long g, int &t, int &i, int &j) {
  t = 0;
#pragma unroll 1
  while (t + 1 < p.nblk && g >= p.b[t + 1].cell0) t++;
  const StbBlk &B = p.b[t];
  const int local = int(g - B.cell0);
  if (p.region == 1) {  // interior rectangle [2, nx-3] x [2, ny-3]
    const int w = B.nx - 4;
    j = 2 + local / w;
    i = 2 + (local - (j - 2) * w);
  } else if (p.region == 2 && B.nx > 4 && B.ny > 4) {  // rows 0,1,ny-2,ny-1, then columns 0,1,nx-2,nx-1
    if (local < 4 * B.nx) {
      const int r = local / B.nx;
      j = r < 2 ? r : B.ny - 4 + r;
      i = local - r * B.nx;
    } else {
      const int l2 = local - 4 * B.nx, h = B.ny - 4;
      const int q = l2 / h;
      i = q < 2 ? q : B.nx - 4 + q;
      j = 2 + (l2 - q * h);
    }
  } else {
    j = local / B.nx;
    i = local - j * B.nx;
  }
}

// Cell g of a block-step launch.
template <int P>
__device__ __forceinline__ void stb_at(const StbParams &p, long long g) {
  int t, i, j;
  stb_locate(p, g, t, i, j);
  if (p.evict_first) stb_cell_h<P, true>(p, p.b[t], i, j);
  else stb_cell_h<P, false>(p, p.b[t], i, j);
}

// Cells g0 and g1 of a block-step launch, with the loads of both in flight
// together.
template <int P, bool EF>
__device__ __forceinline__ void stb_at2_h(const StbParams &p, long long g0, long long g1) {
  using S = typename Prec<P>::S;
  int t0, i0, j0, t1, i1, j1;
  stb_locate(p, g0, t0, i0, j0);
  stb_locate(p, g1, t1, i1, j1);
  const StbBlk &B0 = p.b[t0], &B1 = p.b[t1];
  S r0[9], r1[9];
  const long long c0 = (long long)j0 * B0.pitch + i0, c1 = (long long)j1 * B1.pitch + i1;
  if (i0 > 0 && i0 < B0.nx - 1 && j0 > 0 && j0 < B0.ny - 1) stb_pull_in<P, EF>(B0, c0, r0);
  else stb_pull<P, EF>(B0, i0, j0, r0);
  if (i1 > 0 && i1 < B1.nx - 1 && j1 > 0 && j1 < B1.ny - 1) stb_pull_in<P, EF>(B1, c1, r1);
  else stb_pull<P, EF>(B1, i1, j1, r1);
  const uint8_t f0 = B0.flags[(long long)j0 * B0.pitch + i0], f1 = B1.flags[(long long)j1 * B1.pitch + i1];
  stb_finish<P, EF>(p, B0, i0, j0, r0, f0);
  stb_finish<P, EF>(p, B1, i1, j1, r1, f1);
}

// CPT = 1: one cell per thread (grid-stride: a capped grid leaves CTA slots
// on every SM for kernels that run beside it).  CPT = 2: a CTA owns chunks
// of 512 cells and a thread cells tid and tid + 256 of a chunk.
template <int P, int CPT>
__global__ void __launch_bounds__(256, CPT == 1 ? (P == MB_PREC_F64 ? 4 : 8) : (P == MB_PREC_F64 ? 2 : 4))
    k_block_step(const __grid_constant__ StbParams p) {
  pdl_trigger();
  pdl_wait();
  if constexpr (CPT == 1) {
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < p.total;
         g += (long long)gridDim.x * blockDim.x)
      stb_at<P>(p, g);
  } else {
    for (long long base = (long long)blockIdx.x * 512; base < p.total; base += (long long)gridDim.x * 512) {
      const long long g0 = base + threadIdx.x, g1 = g0 + 256;
      if (g1 < p.total) {
        if (p.evict_first) stb_at2_h<P, true>(p, g0, g1);
        else stb_at2_h<P, false>(p, g0, g1);
      } else if (g0 < p.total) {
        stb_at<P>(p, g0);
      }
    }
  }
}

// ----------------------------------------------------------------------------
// Options kernel: the block step with the collision and boundary options the
// reference declares but never uses.  Used for every block step of a context
// once any option is on; the other block-step kernels assume BGK, no force
// and only SOLID_SBB walls.
//  - body force: the term of stb3 (multi/FH/evolution_block.h:99-108) with
//    forcex/forcey one value everywhere, on every FLUID cell (block-edge
//    cells too, where stb3 collides the imposed equilibrium);
//  - MRT: F = f - M^-1 S (M f - meq) + dt Force_k with M_gpu (lbm/lbm.h:53-63),
//    M^-1 = M^T diag(1/|row|^2) (InvM_gpu, lbm/lbm.h:64-75, exactly), meq of
//    Meq (lbm/assit_func.h:10-22, A = 1, B = -3), S = diag(0, s_e, s_eps, 0,
//    s_q, 0, s_q, 1/tau, 1/tau);
//  - MB_SOLID_SLIP: on-node wall returning F_k = f_slip(k) (slip_gpu,
//    lbm/lbm.h:51) where SOLID_SBB returns f_opp(k);
//  - MB_SOLID_HBB: a FLUID cell whose upstream neighbour x - e_k is an HBB
//    cell takes f_k(x) = F_opp(k)(x), its own value of the previous step; HBB
//    cells keep their distributions.
// ----------------------------------------------------------------------------
constexpr uint8_t FL_HBB = 16, FL_SLIP = 32;  // FL_CCPULL = 64 is defined with the block step

// M_gpu entries (lbm/lbm.h:53-63) and squared row norms
__host__ __device__ constexpr int mrt_m(int q, int k) {
  return q == 0 ? 1
       : q == 1 ? (k == 0 ? -4 : k <= 4 ? -1 : 2)
       : q == 2 ? (k == 0 ? 4 : k <= 4 ? -2 : 1)
       : q == 3 ? ex(k)
       : q == 4 ? (k == 0 ? 0 : k <= 4 ? -2 * ex(k) : ex(k))
       : q == 5 ? ey(k)
       : q == 6 ? (k == 0 ? 0 : k <= 4 ? -2 * ey(k) : ey(k))
       : q == 7 ? (k == 0 ? 0 : k <= 4 ? ex(k) * ex(k) - ey(k) * ey(k) : 0)
       : (k <= 4 ? 0 : ex(k) * ey(k));
}
__host__ __device__ constexpr double mrt_norm(int q) {
  return q == 0 ? 9 : q == 1 || q == 2 ? 36 : q == 3 || q == 5 ? 6 : q == 4 || q == 6 ? 12 : 4;
}

// MRT relaxation of a FLUID cell.  f holds f (or h = f - w when shifted);
// writes the post-collision values (same variable) and rho/u to m.
template <int P>
__device__ __forceinline__ void mrt_collide(const typename Prec<P>::R *f, typename Prec<P>::R rv,
                                            const StbOptions &o, typename Prec<P>::R *out,
                                            typename Prec<P>::R *m, const Shift &sh) {
  using R = typename Prec<P>::R;
  // Macros (lbm/assit_func.h:23-31)
  R rh = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  const R base = rh;  // rho - rho_s when shifted
  if constexpr (Prec<P>::shifted) rh = (R)sh.rhos + rh;
  R ux = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
  R uy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
  if constexpr (Prec<P>::shifted) {
    ux += (R)sh.jx;
    uy += (R)sh.jy;
  }
  ux = ux / rh;
  uy = uy / rh;
  m[0] = rh;
  m[1] = ux;
  m[2] = uy;
  R mo[9];
#pragma unroll
  for (int q = 0; q < 9; q++) {
    R a = (R)0;
#pragma unroll
    for (int k = 0; k < 9; k++)
      if (mrt_m(q, k) != 0) a += (R)mrt_m(q, k) * f[k];
    mo[q] = a;
  }
  const R uv = ux * ux + uy * uy;
  R meq[9];
  if constexpr (Prec<P>::shifted) {  // Meq minus the moments of s = feq(rho_s, U_s)
    meq[0] = base;
    meq[1] = (R)-2 * base + (R)3 * (rh * uv - (R)sh.q2);
    meq[2] = base - (R)3 * (rh * uv - (R)sh.q2);
    meq[3] = rh * ux - (R)sh.jx;
    meq[5] = rh * uy - (R)sh.jy;
    meq[7] = rh * (ux * ux - uy * uy) - (R)sh.qd;
    meq[8] = rh * (ux * uy) - (R)sh.qx;
  } else {
    meq[0] = rh;
    meq[1] = rh * ((R)-2.0 + (R)3.0 * uv);
    meq[2] = rh * ((R)1.0 - (R)3.0 * uv);
    meq[3] = rh * ux;
    meq[5] = rh * uy;
    meq[7] = rh * (ux * ux - uy * uy);
    meq[8] = rh * (ux * uy);
  }
  meq[4] = -meq[3];
  meq[6] = -meq[5];
  const R se = o.mrt_s[0] > 0 ? (R)o.mrt_s[0] : rv;
  const R sp = o.mrt_s[1] > 0 ? (R)o.mrt_s[1] : rv;
  const R sq = o.mrt_s[2] > 0 ? (R)o.mrt_s[2] : rv;
  R dm[9];
  dm[0] = dm[3] = dm[5] = (R)0;
  dm[1] = se * (mo[1] - meq[1]) / (R)mrt_norm(1);
  dm[2] = sp * (mo[2] - meq[2]) / (R)mrt_norm(2);
  dm[4] = sq * (mo[4] - meq[4]) / (R)mrt_norm(4);
  dm[6] = sq * (mo[6] - meq[6]) / (R)mrt_norm(6);
  dm[7] = rv * (mo[7] - meq[7]) / (R)mrt_norm(7);
  dm[8] = rv * (mo[8] - meq[8]) / (R)mrt_norm(8);
#pragma unroll
  for (int k = 0; k < 9; k++) {
    R r = (R)0;
#pragma unroll
    for (int q = 0; q < 9; q++)
      if (mrt_m(q, k) != 0 && q != 0 && q != 3 && q != 5) r += (R)mrt_m(q, k) * dm[q];
    out[k] = f[k] - r;
  }
}

// body-force term of stb3 (evolution_block.h:102-107) for direction k
template <typename R>
__device__ __forceinline__ R force_k(int k, R ux, R uy, R fx, R fy, R rv) {
  const R eu = (R)ex(k) * ux + (R)ey(k) * uy;
  const R vx = (R)3.0 * ((R)ex(k) - ux) + (R)9.0 * eu * (R)ex(k);
  const R vy = (R)3.0 * ((R)ey(k) - uy) + (R)9.0 * eu * (R)ey(k);
  return ((R)1.0 - (R)0.5 * rv) * (R)wd(k) * (vx * fx + vy * fy);
}

template <int P>
__device__ __forceinline__ void stbx_cell(const StbParams &p, const StbBlk &B, int i, int j) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  const long long c = (long long)j * B.pitch + i;
  const uint8_t fl = B.flags[c];
  const int type = fl & 3;
  const S *Fin = (const S *)B.Fin;
  S *Fout = (S *)B.Fout;
  const long long plane = B.plane;
  const R rv = (R)B.rv_tau, dt = (R)B.dt;
  const R fx = (R)p.opt.force[0], fy = (R)p.opt.force[1];
  if (type == 0) {
    const bool wm = p.write_macros && (p.macro_all || (fl & 8));
    if (fl & 4) {  // block edge: the imposed equilibrium, collided (identity) plus the force term
#pragma unroll
      for (int k = 0; k < 9; k++) {
        R v = (R)p.feqc[k];
        if (p.opt.has_force) v += dt * force_k<R>(k, (R)p.u0x, (R)p.u0y, fx, fy, rv);
        if constexpr (Prec<P>::shifted) v -= (R)p.sh.v.s[k];
        Fout[k * plane + c] = from_r<S>(v);
      }
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
      const long long n = c - ((long long)ey(k) * B.pitch + ex(k));
      const bool hbb = (B.flags[n] & (3 | FL_HBB)) == (1 | FL_HBB);
      f[k] = to_r(hbb ? moved<P>(Fin[opp(k) * plane + c], opp(k), k, p.sh) : Fin[k * plane + n]);
    }
    R out[9], m[3];
    if (p.opt.coll == MB_COLL_MRT) mrt_collide<P>(f, rv, p.opt, out, m, p.sh);
    else stb_collide<P>(f, rv, out, m, p.sh, cell_key(B, i, j));
    if (p.opt.has_force) {
#pragma unroll
      for (int k = 0; k < 9; k++) out[k] += dt * force_k<R>(k, m[1], m[2], fx, fy, rv);
    }
    if (wm) {
      ((R *)B.rho)[c] = m[0];
      ((R *)B.ux)[c] = m[1];
      ((R *)B.uy)[c] = m[2];
    }
#pragma unroll
    for (int k = 0; k < 9; k++) Fout[k * plane + c] = from_r<S>(out[k]);
    return;
  }
  if (type == 1 && (fl & FL_SLIP)) {  // pull as SOLID_SBB, return the slip partner
    S raw[9];
    stb_pull<P, false>(B, i, j, raw);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const int id = i - ex(k), jd = j - ey(k);
      if (!(id >= 0 && id < B.nx && jd >= 0 && jd < B.ny)) raw[k] = stored_of<P>(p.feqc[k], k, p.sh.v);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) Fout[k * plane + c] = moved<P>(raw[slip(k)], slip(k), k, p.sh);
    return;
  }
  if (type == 1 && !(fl & FL_HBB)) {  // SOLID_SBB
    S raw[9];
    stb_pull<P, false>(B, i, j, raw);
    stb_finish<P, false>(p, B, i, j, raw, fl);
    return;
  }
  // HBB walls, C_BOUNDARY and row padding keep their distributions
#pragma unroll
  for (int k = 0; k < 9; k++) Fout[k * plane + c] = Fin[k * plane + c];
}

template <int P>
__global__ void __launch_bounds__(256) k_block_step_x(const __grid_constant__ StbParams p) {
  pdl_trigger();
  pdl_wait();
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < p.total;
       g += (long long)gridDim.x * blockDim.x) {
    int t, i, j;
    stb_locate(p, g, t, i, j);
    stbx_cell<P>(p, p.b[t], i, j);
  }
}

// The block step on row tiles: a CTA owns 256 consecutive cells of one row
// of one block (its block, row and first column are uniform over the CTA),
// a thread one cell.  Offsets are 32-bit (the host uses this kernel only
// when 9 planes of every block fit in 2^31 elements).  Interior FLUID cells
// take a short path; every other cell runs the general stb_finish.
// cells on the block edge and cells that are not interior FLUID: the general
// path, out of line so that its registers do not burden the common path
template <int P, bool EF>
__device__ __noinline__ void stb_cell_slow(const StbParams &p, const StbBlk &B, int i, int j) {
  stb_cell_h<P, EF>(p, B, i, j);
}

template <int P, bool EF, bool INTERIOR>
__device__ __forceinline__ void stb_cell_rows(const StbParams &p, const StbBlk &B, int i, int j) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  if (INTERIOR || (i > 0 && i < B.nx - 1 && j > 0 && j < B.ny - 1)) {
    const int c = j * B.pitch + i;
    const int plane = (int)B.plane;
    const S *Fin = (const S *)B.Fin;
    S raw[9];
#pragma unroll
    for (int k = 0; k < 9; k++) raw[k] = ld_ef<EF>(Fin + (k * plane + c - (ey(k) * B.pitch + ex(k))));
    const uint8_t fl = B.flags[c];
    if ((fl & (7 | FL_FCSRC)) == 0) {  // FLUID away from the block edge, no f_c point
      R f[9];
#pragma unroll
      for (int k = 0; k < 9; k++) f[k] = to_r(raw[k]);
      R out[9], m[3];
      stb_collide<P>(f, (R)B.rv_tau, out, m, p.sh, cell_key(B, i, j));
      if (p.write_macros && (p.macro_all || (fl & 8))) {
        st_ef<EF>((R *)B.rho + c, m[0]);
        st_ef<EF>((R *)B.ux + c, m[1]);
        st_ef<EF>((R *)B.uy + c, m[2]);
      }
      S *Fout = (S *)B.Fout;
#pragma unroll
      for (int k = 0; k < 9; k++) st_ef<EF>(Fout + (k * plane + c), from_r<S>(out[k]));
      return;
    }
  }
  stb_cell_slow<P, EF>(p, B, i, j);
}

// The block step on cell ranges: a CTA owns 256 consecutive cells (row-major
// over the region) of one block, so the block's parameters are uniform over
// the CTA; the row comes from a float reciprocal of the region width with
// one integer correction.  Offsets are 32-bit (the host uses this kernel only
// when 9 planes of every block fit in 2^31 elements).
template <int P, bool INTERIOR>
__global__ void __launch_bounds__(256, P == MB_PREC_F64 ? 4 : 6) k_block_step_r(const __grid_constant__ StbParams p) {
  pdl_trigger();
  pdl_wait();
  const int cta = blockIdx.x;
  int t = 0;
#pragma unroll 1
  while (t + 1 < p.nblk && cta >= p.b[t + 1].cta0) t++;
  const StbBlk &B = p.b[t];
  const int local = (cta - B.cta0) * 256 + (int)threadIdx.x;
  if (local >= B.rcells) return;
  int r = __float2int_rz((float)local * B.rinv_w);
  if (r * B.rw > local) r--;
  else if ((r + 1) * B.rw <= local) r++;
  const int j = B.row0 + r;
  const int i = B.rcol0 + (local - r * B.rw);
  if (p.evict_first) stb_cell_rows<P, true, INTERIOR>(p, B, i, j);
  else stb_cell_rows<P, false, INTERIOR>(p, B, i, j);
}

// ----------------------------------------------------------------------------
// The block step on cell pairs: a thread steps cells (i, j) and (i + 1, j),
// i even, so one address serves both cells of a plane: the three planes with
// e_x = 0 and all nine stores move both values in one aligned vector access,
// the six others in two scalar loads at neighbouring addresses.  A CTA owns
// 256 consecutive pairs (row-major over the region) of one block.  Offsets
// are 32-bit (the host uses this kernel only when 9 planes of every block fit
// in 2^31 elements).  Pairs of interior FLUID cells take the short path;
// every other cell runs the general stb_finish.
// ----------------------------------------------------------------------------
template <typename S> struct Vec2;
template <> struct Vec2<float> { using T = float2; };
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<__half> { using T = __half2; };
template <> struct Vec2<h16c> { using T = h16c2; };
__device__ __forceinline__ void unpack2(float2 v, float &a, float &b) { a = v.x; b = v.y; }
__device__ __forceinline__ void unpack2(double2 v, double &a, double &b) { a = v.x; b = v.y; }
__device__ __forceinline__ void unpack2(__half2 v, __half &a, __half &b) { a = __low2half(v); b = __high2half(v); }
__device__ __forceinline__ float2 pack2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 pack2(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ __half2 pack2(__half a, __half b) { return __halves2half2(a, b); }
__device__ __forceinline__ void unpack2(h16c2 v, h16c &a, h16c &b) {
  a.x = (unsigned short)(v.x & 0xffffu);
  b.x = (unsigned short)(v.x >> 16);
}
__device__ __forceinline__ h16c2 pack2(h16c a, h16c b) { return h16c2{(unsigned int)a.x | ((unsigned int)b.x << 16)}; }

template <int P, bool EF, bool INTERIOR>
__device__ __forceinline__ void stb_pair(const StbParams &p, const StbBlk &B, int i, int j, bool two) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  using V = typename Vec2<S>::T;
  if (two && (INTERIOR || (i > 0 && i + 1 < B.nx - 1 && j > 0 && j < B.ny - 1))) {
    const int c = j * B.pitch + i;  // even: pitch and i are even
    const int plane = (int)B.plane;
    const S *Fin = (const S *)B.Fin;
    S a[9], b[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const int o = k * plane + c - (ey(k) * B.pitch + ex(k));
      if (ex(k) == 0) unpack2(ld_ef<EF>((const V *)(Fin + o)), a[k], b[k]);
      else { a[k] = ld_ef<EF>(Fin + o); b[k] = ld_ef<EF>(Fin + o + 1); }
    }
    const unsigned short fl2 = *(const unsigned short *)(B.flags + c);
    const uint8_t fa = uint8_t(fl2 & 0xff), fb = uint8_t(fl2 >> 8);
    if (((fa | fb) & (7 | FL_FCSRC)) == 0) {  // both FLUID away from the block edge, no f_c point
      R f[9], oa[9], ob[9], ma[3], mb[3];
#pragma unroll
      for (int k = 0; k < 9; k++) f[k] = to_r(a[k]);
      stb_collide<P>(f, (R)B.rv_tau, oa, ma, p.sh, cell_key(B, i, j));
#pragma unroll
      for (int k = 0; k < 9; k++) f[k] = to_r(b[k]);
      stb_collide<P>(f, (R)B.rv_tau, ob, mb, p.sh, cell_key(B, i + 1, j));
      if (p.write_macros) {
        const bool wa = p.macro_all || (fa & 8), wb = p.macro_all || (fb & 8);
        R *rho = (R *)B.rho + c, *ux = (R *)B.ux + c, *uy = (R *)B.uy + c;
        if (wa && wb) {
          using VR = typename Vec2<R>::T;
          st_ef<EF>((VR *)rho, pack2(ma[0], mb[0]));
          st_ef<EF>((VR *)ux, pack2(ma[1], mb[1]));
          st_ef<EF>((VR *)uy, pack2(ma[2], mb[2]));
        } else {
          if (wa) { st_ef<EF>(rho, ma[0]); st_ef<EF>(ux, ma[1]); st_ef<EF>(uy, ma[2]); }
          if (wb) { st_ef<EF>(rho + 1, mb[0]); st_ef<EF>(ux + 1, mb[1]); st_ef<EF>(uy + 1, mb[2]); }
        }
      }
      S *Fout = (S *)B.Fout;
#pragma unroll
      for (int k = 0; k < 9; k++) st_ef<EF>((V *)(Fout + (k * plane + c)), pack2(from_r<S>(oa[k]), from_r<S>(ob[k])));
      return;
    }
  }
  stb_cell_slow<P, EF>(p, B, i, j);
  if (two) stb_cell_slow<P, EF>(p, B, i + 1, j);
}

// CTA `cta` of a cell-pair launch: 256 consecutive pairs of one block's region.
template <int P, bool INTERIOR>
__device__ __forceinline__ void stb_pair_cta(const StbParams &p, int cta) {
  int t = 0;
#pragma unroll 1
  while (t + 1 < p.nblk && cta >= p.b[t + 1].pcta0) t++;
  const StbBlk &B = p.b[t];
  const int local = (cta - B.pcta0) * 256 + (int)threadIdx.x;
  if (local >= B.npairs) return;
  int r = __float2int_rz((float)local * B.pinv);
  if (r * B.ppr > local) r--;
  else if ((r + 1) * B.ppr <= local) r++;
  const int q = local - r * B.ppr;
  const int j = B.row0 + r;
  const int i = B.rcol0 + 2 * q;
  const bool two = 2 * q + 1 < B.rw;
  if (p.evict_first) stb_pair<P, true, INTERIOR>(p, B, i, j, two);
  else stb_pair<P, false, INTERIOR>(p, B, i, j, two);
}

template <int P, bool INTERIOR>
__global__ void __launch_bounds__(256, P == MB_PREC_F64 ? 2 : 5) k_block_step_p(const __grid_constant__ StbParams p) {
  pdl_trigger();
  pdl_wait();
  stb_pair_cta<P, INTERIOR>(p, blockIdx.x);
}

// ----------------------------------------------------------------------------
// The block step of split levels' interiors with bulk asynchronous copies:
// a persistent CTA (8 consumer warps and one producer warp) walks items of
// 256 output cells of one row (row-major over the interiors of its blocks,
// items round-robin over the CTAs).  For an item the producer's elected lane
// brings the nine input row segments (plane k at row j - e_y(k), columns
// x0 - A .. x0 + 256 + A, A = 16 bytes of stored words, clamped to the row)
// and the row's flag bytes into a shared-memory stage with cp.async.bulk
// (TMA without a tensor map) completing on the stage's mbarrier; consumers
// pull their cell's values from the stage, collide and store to global
// memory, then release the stage.  STAGES stages keep that many items' loads
// in flight per CTA without holding registers.  Cells that are not interior
// FLUID cells take the general per-cell path from global memory.
// Every mbarrier wait is bounded: a wait that runs out sets the error word
// (mb_sync and the other synchronising calls then return MB_ERR_TIMEOUT) and
// the CTA stops after waiting, again bounded, for the copies it issued.
// ----------------------------------------------------------------------------
constexpr int TB_TW = 256;                   // output cells per item
constexpr int TB_THREADS = 288;              // 8 consumer warps + the producer warp
constexpr unsigned TB_SPIN_LIMIT = 1u << 22; // bounded waits: about a second with the sleeps
template <typename S> struct TbCfg {
  static constexpr int A = 16 / (int)sizeof(S);      // halo, rounded up to 16 bytes
  static constexpr int SEG = TB_TW + 2 * A;          // stored words per row segment
  static constexpr int SEG_BYTES = SEG * (int)sizeof(S);
  static constexpr int FLAG_BYTES = TB_TW + 32;      // flag bytes x0 - 16 .. x0 + 256 + 16
  static constexpr int STAGE_BYTES = 9 * SEG_BYTES + FLAG_BYTES;
  // two CTAs per SM leave room for a spline CTA's 96 KB (mb_set_cta_spread)
  static constexpr int STAGES = sizeof(S) == 2 ? 12 : (sizeof(S) == 4 ? 6 : 4);
  static constexpr int SMEM = STAGES * STAGE_BYTES + 2 * STAGES * 8;
};
static_assert(TbCfg<__half>::SEG_BYTES % 16 == 0 && TbCfg<float>::SEG_BYTES % 16 == 0 &&
                  TbCfg<double>::SEG_BYTES % 16 == 0 && TbCfg<float>::FLAG_BYTES % 16 == 0,
              "bulk copies need 16-byte sizes and offsets");

__device__ __forceinline__ void tb_mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void tb_mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tb_mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"((unsigned)__cvta_generic_to_shared(bar)) : "memory");
}
// bounded wait for the phase of the given parity to complete; false when it ran out
__device__ __forceinline__ bool tb_mbar_wait(uint64_t *bar, unsigned parity) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  for (unsigned n = 0; n < TB_SPIN_LIMIT; n++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (n > 4096) __nanosleep(128);
  }
  return false;
}
__device__ __forceinline__ void tb_bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          (unsigned)__cvta_generic_to_shared(dst)),
      "l"(src), "r"(bytes), "r"((unsigned)__cvta_generic_to_shared(bar))
      : "memory");
}

// item n of a launch: block t, row j, first column x0 of the tile
__device__ __forceinline__ void tb_locate(const StbParams &p, long long it, int &t, int &j, int &x0) {
  t = 0;
#pragma unroll 1
  while (t + 1 < p.nblk && it >= p.b[t + 1].tb0) t++;
  const StbBlk &B = p.b[t];
  const int local = int(it - B.tb0);
  const int r = local / B.tb_tiles;
  j = 2 + r;
  x0 = (local - r * B.tb_tiles) * TB_TW;
}

template <int P>
__global__ void __launch_bounds__(TB_THREADS, 1) k_block_step_tb(const __grid_constant__ StbParams p) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  using C = TbCfg<S>;
  extern __shared__ __align__(128) unsigned char tb_smem[];
  uint64_t *full = (uint64_t *)(tb_smem + C::STAGES * C::STAGE_BYTES);
  uint64_t *empty = full + C::STAGES;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < C::STAGES; s++) {
      tb_mbar_init(&full[s], 1);   // the producer's expect_tx arrival (+ the bytes)
      tb_mbar_init(&empty[s], 8);  // one arrival per consumer warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  pdl_trigger();
  pdl_wait();
  const long long items = p.tb_items;
  if (warp == 8) {  // producer
    if (lane != 0) return;
    long long n = 0;
    bool ok = true;
    for (long long it = blockIdx.x; it < items; it += gridDim.x, n++) {
      const int s = int(n % C::STAGES);
      const unsigned ph = unsigned((n / C::STAGES) & 1);
      if (n >= C::STAGES && !tb_mbar_wait(&empty[s], ph ^ 1u)) { ok = false; break; }
      int t, j, x0;
      tb_locate(p, it, t, j, x0);
      const StbBlk &B = p.b[t];
      unsigned char *st = tb_smem + (size_t)s * C::STAGE_BYTES;
      const S *Fin = (const S *)B.Fin;
      const int lo = max(x0 - C::A, 0), hi = min(x0 + TB_TW + C::A, B.pitch);
      const int flo = max(x0 - 16, 0), fhi = min(x0 + TB_TW + 16, B.pitch);
      const unsigned seg = unsigned(hi - lo) * (unsigned)sizeof(S), fseg = unsigned(fhi - flo);
      tb_mbar_expect_tx(&full[s], 9u * seg + fseg);
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const S *src = Fin + (long long)k * B.plane + (long long)(j - ey(k)) * B.pitch + lo;
        tb_bulk_load(st + k * C::SEG_BYTES + (lo - (x0 - C::A)) * (int)sizeof(S), src, seg, &full[s]);
      }
      tb_bulk_load(st + 9 * C::SEG_BYTES + (flo - (x0 - 16)), B.flags + (long long)j * B.pitch + flo, fseg, &full[s]);
    }
    // every issued stage completes before the CTA may end
    const long long issued = n;
    for (long long q = (issued > C::STAGES ? issued - C::STAGES : 0); q < issued; q++)
      if (!tb_mbar_wait(&full[q % C::STAGES], unsigned((q / C::STAGES) & 1))) ok = false;
    if (!ok && p.err_host) atomicOr(p.err_host, 2u);
    return;
  }
  // consumers
  long long n = 0;
  for (long long it = blockIdx.x; it < items; it += gridDim.x, n++) {
    const int s = int(n % C::STAGES);
    const unsigned ph = unsigned((n / C::STAGES) & 1);
    if (!tb_mbar_wait(&full[s], ph)) {
      if (lane == 0 && p.err_host) atomicOr(p.err_host, 2u);
      break;
    }
    int t, j, x0;
    tb_locate(p, it, t, j, x0);
    const StbBlk &B = p.b[t];
    const unsigned char *st = tb_smem + (size_t)s * C::STAGE_BYTES;
    const int i = x0 + tid;
    if (i >= 2 && i <= B.nx - 3) {
      const uint8_t fl = st[9 * C::SEG_BYTES + 16 + tid];
      if ((fl & (7 | FL_FCSRC)) == 0) {
        R f[9];
#pragma unroll
        for (int k = 0; k < 9; k++) f[k] = to_r(((const S *)(st + k * C::SEG_BYTES))[tid + C::A - ex(k)]);
        R out[9], m[3];
        stb_collide<P>(f, (R)B.rv_tau, out, m, p.sh, cell_key(B, i, j));
        const long long c = (long long)j * B.pitch + i;
        if (p.write_macros && (p.macro_all || (fl & 8))) {
          ((R *)B.rho)[c] = m[0];
          ((R *)B.ux)[c] = m[1];
          ((R *)B.uy)[c] = m[2];
        }
        S *Fout = (S *)B.Fout;
#pragma unroll
        for (int k = 0; k < 9; k++) Fout[k * B.plane + c] = from_r<S>(out[k]);
      } else {
        stb_cell_slow<P, false>(p, B, i, j);
      }
    }
    __syncwarp();
    if (lane == 0) tb_mbar_arrive(&empty[s]);
  }
}

// Four consecutive cells of a row in the stored form, as arithmetic values
// (for shifted precisions these are h = f - w); quads start at i % 4 == 0.
// EF: evict-first cache hints.
template <bool EF> __device__ __forceinline__ void ld_quad(const float *p, float *v) {
  const float4 x = ld_ef<EF>((const float4 *)p);
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
template <bool EF> __device__ __forceinline__ void st_quad(float *p, const float *v) {
  st_ef<EF>((float4 *)p, make_float4(v[0], v[1], v[2], v[3]));
}
template <bool EF> __device__ __forceinline__ void ld_quad(const double *p, double *v) {
  const double2 a = ld_ef<EF>((const double2 *)p), b = ld_ef<EF>((const double2 *)(p + 2));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
template <bool EF> __device__ __forceinline__ void st_quad(double *p, const double *v) {
  st_ef<EF>((double2 *)p, make_double2(v[0], v[1]));
  st_ef<EF>((double2 *)(p + 2), make_double2(v[2], v[3]));
}
template <bool EF> __device__ __forceinline__ void ld_quad(const __half *p, float *v) {
  const uint2 u = ld_ef<EF>((const uint2 *)p);
  const float2 a = __half22float2(*(const __half2 *)&u.x), b = __half22float2(*(const __half2 *)&u.y);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
template <bool EF> __device__ __forceinline__ void ld_quad(const h16c *p, float *v) {
  const uint2 u = ld_ef<EF>((const uint2 *)p);
  v[0] = h16c_decode(u.x & 0xffffu); v[1] = h16c_decode(u.x >> 16);
  v[2] = h16c_decode(u.y & 0xffffu); v[3] = h16c_decode(u.y >> 16);
}
template <bool EF> __device__ __forceinline__ void st_quad(h16c *p, const float *v) {
  uint2 u;
  u.x = h16c_encode(v[0]) | (h16c_encode(v[1]) << 16);
  u.y = h16c_encode(v[2]) | (h16c_encode(v[3]) << 16);
  st_ef<EF>((uint2 *)p, u);
}
template <bool EF> __device__ __forceinline__ void st_quad(__half *p, const float *v) {
  const __half2 a = __floats2half2_rn(v[0], v[1]), b = __floats2half2_rn(v[2], v[3]);
  uint2 u;
  u.x = *(const uint32_t *)&a;
  u.y = *(const uint32_t *)&b;
  st_ef<EF>((uint2 *)p, u);
}

// The block step on quads: a warp owns 128 consecutive cells of one row and
// each lane four of them, moved with one vector load and store per
// direction.  The +-1 shift of the pulled column comes from the neighbouring
// lane (shuffle) and, at the two ends of the warp's span, from one scalar
// load.  Quads that are all FLUID interior cells of the region take this
// path; any other quad (block-edge rows and columns, solids, region borders,
// row ends) runs the per-cell stb_cell for its cells.
template <int P, bool EF>
__device__ __forceinline__ void stb_quad_body(const StbParams &p, long long wt, int lane) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  int t = 0;
#pragma unroll 1
  while (t + 1 < p.nblk && wt >= p.b[t + 1].wt0) t++;
  const StbBlk &B = p.b[t];
  const int local = int(wt - B.wt0);
  const int rr = local / B.tiles_x;
  const int j = B.row0 + rr;
  const int i0 = (local - rr * B.tiles_x) * 128 + 4 * lane;
  const int clo = p.region == 1 ? 2 : 0, chi = p.region == 1 ? B.nx - 3 : B.nx - 1;
  if (j == 0 || j == B.ny - 1) {  // no row on one side: per-cell path for the whole warp
    for (int q = 0; q < 4; q++) {
      const int i = i0 + q;
      if (i >= clo && i <= chi) stb_cell_h<P, EF>(p, B, i, j);
    }
    return;
  }
  const bool inrow = i0 < B.pitch;
  const long long rowc = (long long)j * B.pitch;
  const uint32_t fl4 = inrow ? *(const uint32_t *)(B.flags + rowc + i0) : 0x03030303u;
  const bool fast = inrow && (fl4 & 0x17171717u) == 0u && i0 >= clo && i0 + 3 <= chi;  // FLUID, off the edge, no f_c point
  const S *Fin = (const S *)B.Fin;
  // issue every load before any shuffle consumes one: nine quads and, for the
  // six directions with a column shift, the cell just outside the warp's span
  // (lane 0 for e_x = +1, lane 31 for e_x = -1)
  R f[9][4];
  R halo[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const S *rowp = Fin + k * B.plane + (long long)(j - ey(k)) * B.pitch;
    f[k][0] = f[k][1] = f[k][2] = f[k][3] = (R)0;
    if (inrow) ld_quad<EF>(rowp + i0, f[k]);
    halo[k] = (R)0;
    if (ex(k) == 1 && lane == 0 && inrow && i0 > 0) halo[k] = to_r(ld_ef<EF>(rowp + i0 - 1));
    if (ex(k) == -1 && lane == 31 && i0 + 4 < B.pitch) halo[k] = to_r(ld_ef<EF>(rowp + i0 + 4));
  }
#pragma unroll
  for (int k = 0; k < 9; k++) {
    if (ex(k) == 1) {  // cells i0..i0+3 pull from i0-1..i0+2
      R pw = __shfl_up_sync(0xffffffffu, f[k][3], 1);
      if (lane == 0) pw = halo[k];
      f[k][3] = f[k][2]; f[k][2] = f[k][1]; f[k][1] = f[k][0]; f[k][0] = pw;
    } else if (ex(k) == -1) {  // pull from i0+1..i0+4
      R nw = __shfl_down_sync(0xffffffffu, f[k][0], 1);
      if (lane == 31) nw = halo[k];
      f[k][0] = f[k][1]; f[k][1] = f[k][2]; f[k][2] = f[k][3]; f[k][3] = nw;
    }
  }
  if (fast) {
    const R rv = (R)B.rv_tau;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      R fc[9], o[9], m[3];
#pragma unroll
      for (int k = 0; k < 9; k++) fc[k] = f[k][q];
      stb_collide<P>(fc, rv, o, m, p.sh, cell_key(B, i0 + q, j));
#pragma unroll
      for (int k = 0; k < 9; k++) f[k][q] = o[k];
      if (p.write_macros && (p.macro_all || ((fl4 >> (8 * q)) & 8u))) {
        st_ef<EF>((R *)B.rho + rowc + i0 + q, m[0]);
        st_ef<EF>((R *)B.ux + rowc + i0 + q, m[1]);
        st_ef<EF>((R *)B.uy + rowc + i0 + q, m[2]);
      }
    }
    S *Fout = (S *)B.Fout;
#pragma unroll
    for (int k = 0; k < 9; k++) st_quad<EF>(Fout + k * B.plane + rowc + i0, f[k]);
  } else {
    for (int q = 0; q < 4; q++) {
      const int i = i0 + q;
      if (i < B.nx && i >= clo && i <= chi) stb_cell_h<P, EF>(p, B, i, j);
    }
  }
}

template <int P>
__global__ void __launch_bounds__(256) k_block_step_q(const __grid_constant__ StbParams p) {
  pdl_trigger();
  const long long wt = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wt >= p.total) return;  // warp-uniform
  pdl_wait();
  if (p.evict_first) stb_quad_body<P, true>(p, wt, lane);
  else stb_quad_body<P, false>(p, wt, lane);
}

// Two 16-bit stored words packed in one 32-bit word (the lower cell in the
// low half), as arithmetic values, and back.  The collision has already
// rounded its outputs to values of the stored type (stochastic rounding), so
// packing them rounds nothing further.
__device__ __forceinline__ void unpack_h2(unsigned int w, float &lo, float &hi, const __half *) {
  const float2 v = __half22float2(*(const __half2 *)&w);
  lo = v.x;
  hi = v.y;
}
__device__ __forceinline__ void unpack_h2(unsigned int w, float &lo, float &hi, const h16c *) {
  lo = h16c_decode(w & 0xffffu);
  hi = h16c_decode(w >> 16);
}
__device__ __forceinline__ unsigned int pack_h2(float lo, float hi, const __half *) {
  const __half2 v = __floats2half2_rn(lo, hi);
  return *(const unsigned int *)&v;
}
__device__ __forceinline__ unsigned int pack_h2(float lo, float hi, const h16c *) {
  return h16c_encode(lo) | (h16c_encode(hi) << 16);
}
template <bool EF> __device__ __forceinline__ uint4 ld_oct(const void *p) {
  if constexpr (EF) return __ldcs((const uint4 *)p);
  else return *(const uint4 *)p;
}
template <bool EF> __device__ __forceinline__ void st_oct(void *p, uint4 v) {
  if constexpr (EF) __stcs((uint4 *)p, v);
  else *(uint4 *)p = v;
}

// The block step on octets, for the 16-bit stored forms: a warp owns 256
// consecutive cells of one row and each lane eight of them, moved with one
// 16-byte load and store per direction (four packed pairs of words).  The
// +-1 shift of the pulled column is a byte permutation of neighbouring
// pairs, with the word beyond the lane's octet from the neighbouring lane
// (shuffle) or, at the two ends of the warp's span, from one scalar load.
// Each pair of cells is unpacked, collided cell by cell with the per-cell
// code (same values and the same stochastic rounding as every other
// variant) and packed back in place.  Octets that are not all FLUID
// interior cells of the region run the per-cell stb_cell_h for their cells.
template <int P, bool EF>
__device__ __forceinline__ void stb_oct_body(const StbParams &p, long long wt, int lane) {
  using S = typename Prec<P>::S;
  static_assert(sizeof(S) == 2, "octets are for the 16-bit stored forms");
  int t = 0;
#pragma unroll 1
  while (t + 1 < p.nblk && wt >= p.b[t + 1].wt0) t++;
  const StbBlk &B = p.b[t];
  const int local = int(wt - B.wt0);
  const int rr = local / B.tiles_x;
  const int j = B.row0 + rr;
  const int i0 = (local - rr * B.tiles_x) * 256 + 8 * lane;
  const int clo = p.region == 1 ? 2 : 0, chi = p.region == 1 ? B.nx - 3 : B.nx - 1;
  if (j == 0 || j == B.ny - 1) {  // no row on one side: per-cell path for the whole warp
    for (int q = 0; q < 8; q++) {
      const int i = i0 + q;
      if (i >= clo && i <= chi) stb_cell_h<P, EF>(p, B, i, j);
    }
    return;
  }
  // the pitch is a multiple of 64 words, so every row and octet start is
  // 16-byte aligned; a lane past the row's pitch loads nothing
  const bool inrow = i0 < B.pitch;
  const long long rowc = (long long)j * B.pitch;
  uint2 fl8 = make_uint2(0x03030303u, 0x03030303u);
  if (inrow) fl8 = *(const uint2 *)(B.flags + rowc + i0);
  const bool fast = inrow && ((fl8.x | fl8.y) & 0x17171717u) == 0u && i0 >= clo && i0 + 7 <= chi;
  const S *Fin = (const S *)B.Fin;
  // every load before any shuffle consumes one: nine octets and, for the six
  // directions with a column shift, the word just outside the warp's span
  uint4 w[9];
  unsigned int halo[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const S *rowp = Fin + k * B.plane + (long long)(j - ey(k)) * B.pitch;
    w[k] = make_uint4(0u, 0u, 0u, 0u);
    if (inrow) w[k] = ld_oct<EF>(rowp + i0);
    halo[k] = 0u;
    if (ex(k) == 1 && lane == 0 && inrow && i0 > 0)
      halo[k] = (unsigned int)(*(const unsigned short *)(rowp + i0 - 1)) << 16;
    if (ex(k) == -1 && lane == 31 && i0 + 8 < B.pitch) halo[k] = *(const unsigned short *)(rowp + i0 + 8);
  }
#pragma unroll
  for (int k = 0; k < 9; k++) {
    if (ex(k) == 1) {  // cells i0..i0+7 pull from i0-1..i0+6: the high word of the previous pair leads
      unsigned int pw = __shfl_up_sync(0xffffffffu, w[k].w, 1);
      if (lane == 0) pw = halo[k];
      w[k].w = __byte_perm(w[k].z, w[k].w, 0x5432);
      w[k].z = __byte_perm(w[k].y, w[k].z, 0x5432);
      w[k].y = __byte_perm(w[k].x, w[k].y, 0x5432);
      w[k].x = __byte_perm(pw, w[k].x, 0x5432);
    } else if (ex(k) == -1) {  // pull from i0+1..i0+8: the low word of the next pair trails
      unsigned int nw = __shfl_down_sync(0xffffffffu, w[k].x, 1);
      if (lane == 31) nw = halo[k];
      w[k].x = __byte_perm(w[k].x, w[k].y, 0x5432);
      w[k].y = __byte_perm(w[k].y, w[k].z, 0x5432);
      w[k].z = __byte_perm(w[k].z, w[k].w, 0x5432);
      w[k].w = __byte_perm(w[k].w, nw, 0x5432);
    }
  }
  if (fast) {
    const float rv = (float)B.rv_tau;
    const bool wm = p.write_macros != 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float fa[9], fb[9], oa[9], ob[9], ma[3], mb[3];
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const unsigned int v = q == 0 ? w[k].x : q == 1 ? w[k].y : q == 2 ? w[k].z : w[k].w;
        unpack_h2(v, fa[k], fb[k], (const S *)nullptr);
      }
      const int ia = i0 + 2 * q;
      stb_collide<P>(fa, rv, oa, ma, p.sh, cell_key(B, ia, j));
      stb_collide<P>(fb, rv, ob, mb, p.sh, cell_key(B, ia + 1, j));
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const unsigned int v = pack_h2(oa[k], ob[k], (const S *)nullptr);
        if (q == 0) w[k].x = v;
        else if (q == 1) w[k].y = v;
        else if (q == 2) w[k].z = v;
        else w[k].w = v;
      }
      if (wm) {
        const unsigned int fq = (q < 2 ? fl8.x : fl8.y) >> (16 * (q & 1));
        if (p.macro_all || (fq & 8u)) {
          st_ef<EF>((float *)B.rho + rowc + ia, ma[0]);
          st_ef<EF>((float *)B.ux + rowc + ia, ma[1]);
          st_ef<EF>((float *)B.uy + rowc + ia, ma[2]);
        }
        if (p.macro_all || ((fq >> 8) & 8u)) {
          st_ef<EF>((float *)B.rho + rowc + ia + 1, mb[0]);
          st_ef<EF>((float *)B.ux + rowc + ia + 1, mb[1]);
          st_ef<EF>((float *)B.uy + rowc + ia + 1, mb[2]);
        }
      }
    }
    S *Fout = (S *)B.Fout;
#pragma unroll
    for (int k = 0; k < 9; k++) st_oct<EF>(Fout + k * B.plane + rowc + i0, w[k]);
  } else {
    for (int q = 0; q < 8; q++) {
      const int i = i0 + q;
      if (i < B.nx && i >= clo && i <= chi) stb_cell_h<P, EF>(p, B, i, j);
    }
  }
}

// Octet kernel (16-bit stored forms): 8 warps per CTA, one warp tile of 256
// cells each (StbBlk::wt0 and tiles_x count 256-cell tiles for it).
template <int P>
__global__ void __launch_bounds__(256, 3) k_block_step_o(const __grid_constant__ StbParams p) {
  pdl_trigger();
  const long long wt = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wt >= p.total) return;  // warp-uniform
  pdl_wait();
  if constexpr (sizeof(typename Prec<P>::S) == 2) {
    if (p.evict_first) stb_oct_body<P, true>(p, wt, lane);
    else stb_oct_body<P, false>(p, wt, lane);
  }
}


// ----------------------------------------------------------------------------
// Interface point records: c_c_boundary_transfer, temporal_interpolation,
// c_f_boundary_transfer, f_c_boundary_transfer (multi/FH/assit_multi.h).
// ----------------------------------------------------------------------------
constexpr int REC_THREADS = 64;
// Per-block fields the record kernel touches, as launch parameters: a record's
// first access then depends on one load (the record), not on the block table.
constexpr int REC_MAX_BLOCKS = 40;
struct RecBlk {
  void *F[2];
  void *rho, *ux, *uy;
  long long plane;
  double tau;
  int m, pad_;
};


// One reference line op of a record launch.  Its points are affine in the
// point index ip: target cell dst0 + ip*dstride, source (cell or slot point)
// src0 + ip*sstride.  Points whose writes the plan dropped are marked in the
// per-point mask (bits 4: F, 8: rho/u); has_mask = 0 means all writes live.
constexpr int REC_MAX_OPS = 24;
struct RecOp {
  uint8_t type, dst_block, src_block, bits;  // bits: RB_* buffer bits and weight index
  uint8_t m0, m1, m2, has_mask;
  int32_t count, dst0, dstride, src0, sstride, mask_off;
};
struct RecOpsParams {
  int nops, total;
  int op_start[REC_MAX_OPS + 1];
  RecOp ops[REC_MAX_OPS];
  RecBlk b[REC_MAX_BLOCKS];
  void *slots;
  const uint8_t *mask;
  double tw[4][3];
  Sh9 sh;  // shift of the stored words
};
static_assert(sizeof(RecOpsParams) <= 4096, "record launch parameters must fit the 4 KB parameter space");

// Point t (0 <= t < p.total) of a record launch.
template <int P>
__device__ __forceinline__ void rec_point(const RecOpsParams &p, int t) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  int o = 0;
#pragma unroll 1
  while (o + 1 < p.nops && t >= p.op_start[o + 1]) o++;
  const RecOp &op = p.ops[o];
  const int ip = t - p.op_start[o];
  const long long dc = (long long)op.dst0 + (long long)ip * op.dstride;
  const long long sc = (long long)op.src0 + (long long)ip * op.sstride;
  // every source load is issued before the write mask is known: one memory
  // round trip per point
  const uint8_t *mp = op.has_mask ? p.mask + op.mask_off + ip : nullptr;
  const RecBlk &D = p.b[op.dst_block];
  S *Fd = (S *)D.F[(op.bits >> 1) & 1];
  if (op.type == 0) {  // same-level copy (assit_multi.h:2-46)
    const RecBlk &A = p.b[op.src_block];
    const S *Fs = (const S *)A.F[op.bits & 1];
    const R m0 = ((const R *)A.rho)[sc], m1 = ((const R *)A.ux)[sc], m2 = ((const R *)A.uy)[sc];
    S f[9];
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = Fs[k * A.plane + sc];
    const uint8_t live = mp ? *mp : op.bits;
    if (live & 8) {
      ((R *)D.rho)[dc] = m0;
      ((R *)D.ux)[dc] = m1;
      ((R *)D.uy)[dc] = m2;
    }
    if (live & 4) {
#pragma unroll
      for (int k = 0; k < 9; k++) Fd[k * D.plane + dc] = f[k];
    }
    return;
  }
  if (op.type == 1 || op.type == 2) {  // temporal interpolation (:213-247) / c_f (:249-271)
    const R *s = (const R *)p.slots + sc * 27;
    R v[9];
    if (op.type == 1) {
      const int wi = (op.bits >> 4) & 3;
      const R a = (R)p.tw[wi][0], b = (R)p.tw[wi][1], cc = (R)p.tw[wi][2];
#pragma unroll
      for (int k = 0; k < 9; k++) v[k] = temporal3<R>(a, b, cc, s[op.m0 * 9 + k], s[op.m1 * 9 + k], s[op.m2 * 9 + k]);
    } else {
#pragma unroll
      for (int k = 0; k < 9; k++) v[k] = s[op.m2 * 9 + k];
    }
    const uint8_t live = mp ? *mp : op.bits;
    if (live & 4) {
#pragma unroll
      for (int k = 0; k < 9; k++) st_f<P>(Fd, k * D.plane + dc, k, v[k], p.sh);
    }
    return;
  }
  // f_c (:273-314): coarse edge <- fine point, f_neq scaled by r (tau_c-1)/(tau_f-1)
  const RecBlk &Fb = p.b[op.src_block];
  const S *Fs = (const S *)Fb.F[op.bits & 1];
  const R rh = ((const R *)Fb.rho)[sc], ux = ((const R *)Fb.ux)[sc], uy = ((const R *)Fb.uy)[sc];
  R ft[9];
  if (op.type == 4) {  // the fine cell holds what a c_f stored from slot point sstride
    const R *sv = (const R *)p.slots + (long long)op.sstride * 27 + op.m2 * 9;
#pragma unroll
    for (int k = 0; k < 9; k++) {  // the stored form's rounding, as st_f then ld_f
      if constexpr (Prec<P>::shifted) ft[k] = to_r(from_r<S>(sv[k] - p.sh.s[k])) + p.sh.s[k];
      else ft[k] = to_r(from_r<S>(sv[k]));
    }
  } else {
#pragma unroll
    for (int k = 0; k < 9; k++) ft[k] = ld_f<P>(Fs, k * Fb.plane + sc, k, p.sh);
  }
  const uint8_t live = mp ? *mp : op.bits;
  if (live & 8) {
    ((R *)D.rho)[dc] = rh;
    ((R *)D.ux)[dc] = ux;
    ((R *)D.uy)[dc] = uy;
  }
  if (live & 4) {
    const R para = (R)((double)(Fb.m / D.m) * (D.tau - 1.0) / (Fb.tau - 1.0));
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const R fe = feq<R>(k, rh, ux, uy);
      st_f<P>(Fd, k * D.plane + dc, k, fe + para * (ft[k] - fe), p.sh);
    }
  }
}

template <int P>
__global__ void __launch_bounds__(REC_THREADS) k_records(const __grid_constant__ RecOpsParams p) {
  pdl_trigger();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.total) return;
  pdl_wait();
  rec_point<P>(p, t);
}

// ----------------------------------------------------------------------------
// Spatial interpolation: init_Spline3 + tridiagonal solve + calculate_Spline3_gpu
// (assit_multi.h:48-211) for one coarse-fine line per CTA.
// ----------------------------------------------------------------------------

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

// Spatial interpolation, one warp per segment of SPL_SEG intervals of a
// coarse-fine line.  The spline moments M solve the (0.5, 2, 0.5) system of
// init_tri_A (multi/init_multi.h:30-51; decoupled natural end rows) by the
// Thomas recurrences y_i = (d_i - l_i y_{i-1}) / den_i, x_i = y_i - c'_i x_{i+1}
// (c'_i and 1/den_i of the whole system come from a per-line table).  Both
// recurrences contract by 0.268 per row (2 - sqrt 3), so the moments a
// segment needs are computed on a window of SPL_HALO rows either side of it,
// started from zero: the truncation changes them by less than 0.268^HALO of
// the data (1e-16 in FP64, 1e-9 in FP32), i.e. they equal the whole-line solve
// to rounding.  Every segment is independent, so a line's gathers and solves
// spread over many SMs.
constexpr int SPL_SEG = 16;
constexpr int SPL_WARPS = 4;
template <typename R> struct SplHalo { static constexpr int v = 16; };
template <> struct SplHalo<double> { static constexpr int v = 28; };
template <typename R> __host__ __device__ constexpr int spl_win() { return SPL_SEG + 2 * SplHalo<R>::v + 4; }

// Everything a spline warp needs about its line, as launch parameters (no
// dependent loads before the gather).
constexpr int SPL_MAX_TASKS = 16;
struct SplTaskP {
  int Nc, Nf, r, slot0;
  int ci0, cj0, cdi, cdj;  // coarse source line: start and unit step
  int fi0, fj0, fdi, fdj;  // fine edge line
  int coef0, m0, mask_off, seg0;
  double para;
  const void *Fc;          // current F buffer of the coarse block
  const void *Mc[3];       // coarse rho, ux, uy
  void *Mf[3];             // fine rho, ux, uy
  long long cplane;
  int cpitch, fpitch;
  // fused temporal interpolation (tmp != 0): F of each fine edge point in
  // buffer Ft <- tw0 s[tm0] - tw1 s[tm1] + tw2 s[tm2] of its slots, where
  // mask[tmask_off + ip] is set
  int tmp, tmask_off;
  int tm[3];
  double tw[3];
  void *Ft;
  long long fplane;
};
struct SplParamsP {
  int ntask, nseg;
  SplTaskP t[SPL_MAX_TASKS];
  void *slots;
  const uint8_t *mask;
  const void *coef;  // per line: c'_i (Nc values) then 1/den_i (Nc values), at 2 * coef0
  Sh9 sh;            // shift of the stored words
};
static_assert(sizeof(SplParamsP) <= 4096, "spline launch parameters must fit the 4 KB parameter space");

// the 12 fields (rho, ux, uy, F0..F8) of coarse point ip
template <int P>
__device__ __forceinline__ void spl_gather_p(const SplTaskP &T, int ip, typename Prec<P>::R *v, const Sh9 &sh) {
  using R = typename Prec<P>::R;
  using S = typename Prec<P>::S;
  const long long c = (long long)(T.cj0 + ip * T.cdj) * T.cpitch + (T.ci0 + ip * T.cdi);
  v[0] = ((const R *)T.Mc[0])[c];
  v[1] = ((const R *)T.Mc[1])[c];
  v[2] = ((const R *)T.Mc[2])[c];
  const S *F = (const S *)T.Fc;
#pragma unroll
  for (int k = 0; k < 9; k++) v[3 + k] = ld_f<P>(F, k * T.cplane + c, k, sh);
}

// shared memory of one spline warp: the gathered fields, the forward sweep
// (then the moments) and the window's c' and 1/den
template <typename R> __host__ __device__ constexpr size_t spl_warp_smem() { return (size_t)26 * spl_win<R>() * sizeof(R); }
// ... and, for the spline launches (UNROLL), the slot values each lane's
// first fine point reads for a fused temporal interpolation (27 per lane)
template <typename R> __host__ __device__ constexpr size_t spl_warp_smem_pf() {
  return spl_warp_smem<R>() + (size_t)27 * 32 * sizeof(R);
}

// Asynchronous 4- or 8-byte copy from global to shared memory (cp.async,
// completes into shared memory without holding registers).
template <typename R> __device__ __forceinline__ void cp_async_val(R *dst, const R *src) {
  static_assert(sizeof(R) == 4 || sizeof(R) == 8, "cp.async value size");
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"((int)sizeof(R)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Segment sid (0 <= sid < p.nseg) of a spline launch, by one warp, with its
// window arrays at wsm (spl_warp_smem bytes, 16-byte aligned; with UNROLL,
// spl_warp_smem_pf bytes).
template <int P, bool UNROLL>
__device__ __forceinline__ void spl_segment(const SplParamsP &p, int sid, int lane, unsigned char *wsm) {
  using R = typename Prec<P>::R;
  constexpr int H = SplHalo<R>::v;
  constexpr int W = spl_win<R>();
  R(*sfw)[W] = (R(*)[W])wsm;                   // [12][W] gathered fields
  R(*sxw)[W] = sfw + 12;                        // [12][W] forward sweep, then the moments
  R(*scw)[W] = sxw + 12;                        // [2][W] c'_i and 1/den_i of the window
  int tk = 0;
#pragma unroll 1
  while (tk + 1 < p.ntask && sid >= p.t[tk + 1].seg0) tk++;
  const SplTaskP &T = p.t[tk];
  const int seg = sid - T.seg0;
  const int N = T.Nc;
  const R *cpt = (const R *)p.coef + 2LL * T.coef0;
  const R *ivd = cpt + N;

  // intervals I in [Ilo, Ihi] (fine point ip uses rows I-1 and I, I = ceil(ip/r), at least 1)
  const int Ilo = 1 + seg * SPL_SEG, Ihi = min(N - 1, (seg + 1) * SPL_SEG);
  const int w0 = max(0, Ilo - 1 - H), w1 = min(N - 1, Ihi + H);  // rows solved
  const int g0 = max(0, w0 - 1), g1 = min(N - 1, w1 + 1);        // rows gathered
  // fine points of the segment (evaluated below)
  const int ip0 = (seg == 0) ? 0 : T.r * (Ilo - 1) + 1;
  const int ip1 = min(T.Nf - 1, T.r * Ihi);
  R *slots = (R *)p.slots;
  // fused temporal interpolation: the slot values of the lane's first point
  // that this launch does not write (markers other than m0) are copied to
  // shared memory now, beside the gather, instead of read after the slot
  // stores (no other op of the launch writes them)
  R *pf = (R *)(wsm + spl_warp_smem<R>()) + lane * 27;
  const int ipf = ip0 + lane;
  const bool pre = UNROLL && T.tmp && ipf <= ip1;
  // the write masks of the lane's first point, loaded now as well (plan
  // data, constant during the launch)
  bool mk_first = true, tk_first = false;
  if (ipf <= ip1) {
    mk_first = T.mask_off < 0 || p.mask[T.mask_off + ipf];
    tk_first = T.tmp && p.mask[T.tmask_off + ipf];
  }
  if constexpr (UNROLL) {
    if (pre) {
      const R *s3 = slots + (long long)(T.slot0 + ipf) * 27;
#pragma unroll
      for (int q = 0; q < 3; q++)
        if (T.tm[q] != T.m0)
#pragma unroll
          for (int k = 0; k < 9; k++) cp_async_val<R>(pf + T.tm[q] * 9 + k, s3 + T.tm[q] * 9 + k);
    }
  }
  if constexpr (UNROLL) {
    // at most 3 x 32 rows (the window is below 96 rows): every load of the
    // gather in flight at once
    static_assert(spl_win<R>() + 2 <= 96, "gather window");
    R v[3][12], c0[3], c1[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const int i = g0 + lane + 32 * q;
      if (i <= g1) {
        spl_gather_p<P>(T, i, v[q], p.sh);
        c0[q] = cpt[i];
        c1[q] = ivd[i];
      }
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const int i = g0 + lane + 32 * q;
      if (i <= g1) {
#pragma unroll
        for (int f = 0; f < 12; f++) sfw[f][i - g0] = v[q][f];
        scw[0][i - g0] = c0[q];
        scw[1][i - g0] = c1[q];
      }
    }
  } else {
    for (int i = g0 + lane; i <= g1; i += 32) {
      R v[12];
      spl_gather_p<P>(T, i, v, p.sh);
#pragma unroll
      for (int f = 0; f < 12; f++) sfw[f][i - g0] = v[f];
      scw[0][i - g0] = cpt[i];
      scw[1][i - g0] = ivd[i];
    }
  }
  __syncwarp();
  if (lane < 12) {
    const int f = lane;
    const R *x = sfw[f] - g0;  // x[i] = field at row i
    R *y = sxw[f] - g0;
    const R *cp = scw[0] - g0, *iv = scw[1] - g0;
    // right-hand sides 6 f_i - 3 f_{i-1} - 3 f_{i+1}, zero at both ends (assit_multi.h:82-107)
    R yv = 0;
#pragma unroll 4
    for (int i = w0; i <= w1; i++) {
      const R d = (i == 0 || i == N - 1) ? (R)0 : ((R)6.0 * x[i] - (R)3.0 * x[i - 1] - (R)3.0 * x[i + 1]);
      const R l = (i <= 1 || i == N - 1) ? (R)0 : (R)0.5;
      yv = (d - l * yv) * iv[i];
      y[i] = yv;
    }
    R xv = 0;
#pragma unroll 4
    for (int i = w1; i >= w0; i--) {
      xv = y[i] - cp[i] * xv;
      y[i] = xv;
    }
  }
  __syncwarp();

  // evaluate the fine points of the segment (calculate_Spline3_gpu :136-185)
  const R para = (R)T.para;
  if constexpr (UNROLL) {
    if (pre) cp_async_wait_all();  // the lane's own copies
  }
  for (int ip = ip0 + lane; ip <= ip1; ip += 32) {
    const R xx = (R)ip / (R)T.r;
    int I = (int)ceil(xx);
    if (I == 0) I = 1;
    R out[12];
#pragma unroll
    for (int f = 0; f < 12; f++)
      out[f] = spline3_s<R>(xx, (R)(I - 1), (R)1.0, sfw[f][I - 1 - g0], sfw[f][I - g0],
                            sxw[f][I - 1 - g0], sxw[f][I - g0]);
    const long long fc = (long long)(T.fj0 + ip * T.fdj) * T.fpitch + (T.fi0 + ip * T.fdi);
    if (ip == ipf ? mk_first : (T.mask_off < 0 || p.mask[T.mask_off + ip])) {
      ((R *)T.Mf[0])[fc] = out[0];
      ((R *)T.Mf[1])[fc] = out[1];
      ((R *)T.Mf[2])[fc] = out[2];
    }
    R *sl = slots + ((long long)(T.slot0 + ip) * 3 + T.m0) * 9;
    R slv[9];  // the slot values this launch writes (marker m0)
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const R fe = feq<R>(k, out[0], out[1], out[2]);
      slv[k] = fe + para * (out[3 + k] - fe);
      sl[k] = slv[k];
    }
    if (ip == ipf ? tk_first : (T.tmp && p.mask[T.tmask_off + ip])) {  // the fused temporal interpolation of the slots
      // marker m0 from the values just computed, the others from the
      // prefetched copies (the lane's first point) or from global memory
      const R *s3 = (pre && ip == ipf) ? pf : slots + (long long)(T.slot0 + ip) * 27;
      const R a = (R)T.tw[0], b = (R)T.tw[1], cc = (R)T.tw[2];
      typename Prec<P>::S *Fd = (typename Prec<P>::S *)T.Ft;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const R s0 = T.tm[0] == T.m0 ? slv[k] : s3[T.tm[0] * 9 + k];
        const R s1 = T.tm[1] == T.m0 ? slv[k] : s3[T.tm[1] * 9 + k];
        const R s2 = T.tm[2] == T.m0 ? slv[k] : s3[T.tm[2] * 9 + k];
        st_f<P>(Fd, k * T.fplane + fc, k, temporal3<R>(a, b, cc, s0, s1, s2), p.sh);
      }
    }
  }
}

template <int P>
__global__ void __launch_bounds__(32 * SPL_WARPS) k_spline(const __grid_constant__ SplParamsP p) {
  using R = typename Prec<P>::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  pdl_trigger();
  const int sid = blockIdx.x * (int)(blockDim.x >> 5) + warp;  // blockDim: 1 to SPL_WARPS warps
  if (sid >= p.nseg) return;
  pdl_wait();
  spl_segment<P, true>(p, sid, lane, smem_raw + warp * spl_warp_smem_pf<R>());
}

// ----------------------------------------------------------------------------
// Batched launches: one launch runs the same plan node of many cases (the
// cases of a batch share the plan's structure, not their sizes).  Each case
// has its own parameter block in device memory and a contiguous range of
// CTAs (cta0[c] .. cta0[c+1]-1); a CTA finds its case, copies the case's
// parameter block into shared memory and runs the single-case code on its
// CTA index within that case.
// ----------------------------------------------------------------------------
struct BatchArgs {
  const unsigned char *params;  // ncases parameter blocks, pstride bytes apart (16-byte multiples)
  const int *cta0;              // first CTA of each case
  int ncases, pstride;
};

// the case of this CTA (uniform), and its parameter block copied to smem
__device__ __forceinline__ int batch_case(const BatchArgs &a, unsigned char *smem, int nbytes) {
  int lo = 0, hi = a.ncases - 1;
  const int b = (int)blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(a.cta0 + mid) <= b) lo = mid; else hi = mid - 1;
  }
  const int4 *src = (const int4 *)(a.params + (size_t)lo * a.pstride);
  for (int q = threadIdx.x; q < nbytes / 16; q += blockDim.x) ((int4 *)smem)[q] = __ldg(src + q);
  __syncthreads();
  return lo;
}

template <int P>
__global__ void __launch_bounds__(256, P == MB_PREC_F64 ? 4 : 8) kb_block_step(const __grid_constant__ BatchArgs a) {
  __shared__ __align__(16) unsigned char sp[(sizeof(StbParams) + 15) / 16 * 16];
  const int c = batch_case(a, sp, (int)sizeof(sp));
  const StbParams &p = *(const StbParams *)sp;
  const long long g = (long long)((int)blockIdx.x - __ldg(a.cta0 + c)) * 256 + threadIdx.x;
  if (g < p.total) stb_at<P>(p, g);
}

// Persistent form of kb_block_step: a grid of G CTAs (a few per SM, all
// resident), CTA b takes the tiles [T b / G, T (b + 1) / G) of the launch's
// T tiles of 256 cells (cases in order, cta0 holding each case's first
// tile), so the work is split evenly by cells and a CTA copies a case's
// parameter block only when its range enters that case.
template <int P>
__global__ void __launch_bounds__(256, P == MB_PREC_F64 ? 4 : 8) kb_block_step_ps(const __grid_constant__ BatchArgs a) {
  __shared__ __align__(16) unsigned char sp[(sizeof(StbParams) + 15) / 16 * 16];
  const StbParams &p = *(const StbParams *)sp;
  const long long T = __ldg(a.cta0 + a.ncases), G = gridDim.x;
  const int t0 = (int)(T * blockIdx.x / G), t1 = (int)(T * (blockIdx.x + 1) / G);
  int lo = 0, hi = a.ncases - 1;  // case of the first tile
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(a.cta0 + mid) <= t0) lo = mid; else hi = mid - 1;
  }
  int cur = -1;
#pragma unroll 1
  for (int t = t0; t < t1; t++) {
    while (lo + 1 < a.ncases && __ldg(a.cta0 + lo + 1) <= t) lo++;
    if (lo != cur) {
      __syncthreads();  // every thread is done with the previous case's parameters
      const int4 *src = (const int4 *)(a.params + (size_t)lo * a.pstride);
      for (int q = threadIdx.x; q < (int)sizeof(sp) / 16; q += blockDim.x) ((int4 *)sp)[q] = __ldg(src + q);
      __syncthreads();
      cur = lo;
    }
    const long long g = (long long)(t - __ldg(a.cta0 + lo)) * 256 + threadIdx.x;
    if (g < p.total) stb_at<P>(p, g);
  }
}

// Cell-pair form of kb_block_step: one CTA per CTA of the cell-pair kernel
// (256 pairs of one block's region), cases in order.
template <int P>
__global__ void __launch_bounds__(256, P == MB_PREC_F64 ? 2 : 5) kb_block_step_pt(const __grid_constant__ BatchArgs a) {
  __shared__ __align__(16) unsigned char sp[(sizeof(StbParams) + 15) / 16 * 16];
  const int c = batch_case(a, sp, (int)sizeof(sp));
  const StbParams &p = *(const StbParams *)sp;
  const int cta = (int)blockIdx.x - __ldg(a.cta0 + c);
  if (cta < p.pctas) stb_pair_cta<P, false>(p, cta);
}

// Cell-pair form of kb_block_step_ps: the tiles are the cell-pair kernel's
// CTAs (256 pairs of one block's region, cta0 holding each case's first),
// split evenly over a persistent grid.  Whole levels and interiors only (the
// pair code also serves an interior region).
template <int P>
__global__ void __launch_bounds__(256, P == MB_PREC_F64 ? 2 : 5) kb_block_step_pp(const __grid_constant__ BatchArgs a) {
  __shared__ __align__(16) unsigned char sp[(sizeof(StbParams) + 15) / 16 * 16];
  const StbParams &p = *(const StbParams *)sp;
  const long long T = __ldg(a.cta0 + a.ncases), G = gridDim.x;
  const int t0 = (int)(T * blockIdx.x / G), t1 = (int)(T * (blockIdx.x + 1) / G);
  int lo = 0, hi = a.ncases - 1;  // case of the first tile
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(a.cta0 + mid) <= t0) lo = mid; else hi = mid - 1;
  }
  int cur = -1;
#pragma unroll 1
  for (int t = t0; t < t1; t++) {
    while (lo + 1 < a.ncases && __ldg(a.cta0 + lo + 1) <= t) lo++;
    if (lo != cur) {
      __syncthreads();  // every thread is done with the previous case's parameters
      const int4 *src = (const int4 *)(a.params + (size_t)lo * a.pstride);
      for (int q = threadIdx.x; q < (int)sizeof(sp) / 16; q += blockDim.x) ((int4 *)sp)[q] = __ldg(src + q);
      __syncthreads();
      cur = lo;
    }
    const int cta = t - __ldg(a.cta0 + lo);
    if (cta < p.pctas) stb_pair_cta<P, false>(p, cta);
  }
}

template <int P>
__global__ void __launch_bounds__(REC_THREADS) kb_records(const __grid_constant__ BatchArgs a) {
  __shared__ __align__(16) unsigned char sp[(sizeof(RecOpsParams) + 15) / 16 * 16];
  const int c = batch_case(a, sp, (int)sizeof(sp));
  const RecOpsParams &p = *(const RecOpsParams *)sp;
  const int t = ((int)blockIdx.x - __ldg(a.cta0 + c)) * (int)blockDim.x + (int)threadIdx.x;
  if (t < p.total) rec_point<P>(p, t);
}

template <int P>
__global__ void __launch_bounds__(32 * SPL_WARPS) kb_spline(const __grid_constant__ BatchArgs a) {
  using R = typename Prec<P>::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PB = (sizeof(SplParamsP) + 15) / 16 * 16;
  const int c = batch_case(a, smem_raw, PB);
  const SplParamsP &p = *(const SplParamsP *)smem_raw;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sid = ((int)blockIdx.x - __ldg(a.cta0 + c)) * (int)(blockDim.x >> 5) + warp;
  if (sid < p.nseg) spl_segment<P, true>(p, sid, lane, smem_raw + PB + warp * spl_warp_smem_pf<R>());
}

// ----------------------------------------------------------------------------
// Persistent plan executor.  One launch runs every node of a compiled plan
// (block steps, record ops, spline lines of one or more coarse steps) with the
// plan's dependencies tracked on the device.  Each node is cut into work
// items; a node's successors become ready when its last item completes.
//
// A CTA is eight worker warps and one scheduler warp.  The scheduler claims
// items (atomic counter per node), stages the parameter block of the next
// item in one of two shared buffers while the workers execute the current
// one, and signals completion of each item after the workers are done with
// it.  Workers and scheduler hand items over through two named barriers
// (FULL: an item is staged; EMPTY: the workers finished one).
//
// Nodes [0, nurgent) are the latency-bound chain (every node but the
// interior of split levels), in plan order; nodes [nurgent, nnodes) the bulk
// interior block steps.  The scheduler takes the first ready urgent node of
// its scan window, else the first ready bulk node: bulk work fills the time
// the fine-level chain spends waiting on its own dependencies.  Items never
// wait, so the executor cannot deadlock; a scheduler that finds no ready
// work sleeps with backoff and gives up (error word set, all CTAs exit) after
// timeout_ns without work.
//
// Ordering: after the workers pass EMPTY, the scheduler fences and adds one
// to the node's done count; the scheduler that completes the last item
// fences, decrements each successor's pending count, fences and increments
// the generation word.  A scheduler rescans pending counts only after an
// acquire load shows a new generation (or its window moved), reads them with
// acquire loads, and publishes the claimed item through FULL before any
// worker reads the node's inputs.  All loads of distributions are plain
// (coherent) loads: buffers are written by earlier nodes of the same launch.
// ----------------------------------------------------------------------------
constexpr int PRG_WORKERS = 256;
constexpr int PRG_THREADS = PRG_WORKERS + 32;
constexpr int PRG_SCHED_WARP = PRG_WORKERS / 32;
constexpr int PRG_MAX_NODES = 1024;
constexpr int PRG_WIN = 16;  // scan window per class (urgent, bulk): one lane per node
constexpr int PRG_BAR_FULL = 1, PRG_BAR_EMPTY = 2;
enum : int { PK_STB = 0, PK_REC = 1, PK_SPL = 2, PK_NOP = 3 };

struct PrgNode {
  int kind;
  int items;       // work items
  long long units; // cells (STB), points (REC) or segments (SPL)
  int per_item;    // units per item
  int param_off;   // byte offset of the node's parameter block in the blob (16-byte aligned)
  int param_bytes; // multiple of 16
  int succ0, nsucc;
  int plan_index;  // index of the node in the compiled plan (for traces)
};
static_assert(sizeof(PrgNode) == 40, "PrgNode layout");

// One executed work item, when tracing is on: global-timer stamps of the
// start of its claim, of its hand-over to the workers and of the workers'
// completion.
struct PrgTraceRec {
  unsigned long long t_pick, t_start, t_end;
  int plan_node, item;
  int sm, cta;
  int launch, pad_;
};
static_assert(sizeof(PrgTraceRec) == 48, "PrgTraceRec layout");

struct PrgArgs {
  const PrgNode *nodes;
  const int *succ;
  const unsigned char *blob;
  unsigned int *claim, *done, *pending;  // per node; reset before every launch
  unsigned int *gen;                     // nodes completed so far; reset before every launch
  unsigned int *bulk_active;             // CTAs holding a bulk item; reset before every launch
  int bulk_limit;                        // claim bulk items only while bulk_active < bulk_limit (0: no limit)
  unsigned int *err;                     // device error word: nonzero stops every CTA
  unsigned int *host_err;                // mapped host word mirrored on error (may be null)
  int nnodes, nurgent;
  unsigned long long timeout_ns;
  PrgTraceRec *trace;                    // tracing kernel only
  unsigned int *trace_n;
  unsigned int trace_cap;
  int launch;
};

// shared memory of the executor: two parameter buffers, then SPL_WARPS
// spline windows
__host__ __device__ constexpr size_t prg_cmax(size_t x, size_t y) { return x > y ? x : y; }
__host__ __device__ constexpr size_t prg_pbuf() {
  return (prg_cmax(sizeof(StbParams), prg_cmax(sizeof(RecOpsParams), sizeof(SplParamsP))) + 15) / 16 * 16;
}
template <typename R> __host__ __device__ constexpr size_t prg_smem() {
  return 2 * prg_pbuf() + SPL_WARPS * spl_warp_smem<R>();
}

__device__ __forceinline__ unsigned long long prg_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned int prg_ld_acquire(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int prg_ld_relaxed(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ bool prg_bit(const unsigned int *m, int n) { return (m[n >> 5] >> (n & 31)) & 1u; }
__device__ __forceinline__ void prg_bar_sync(int id) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(PRG_THREADS) : "memory");
}
__device__ __forceinline__ void prg_bar_arrive(int id) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "n"(PRG_THREADS) : "memory");
}

// Scheduler-warp state (registers of every lane, kept uniform).
struct PrgSched {
  int lo_u, lo_b;          // first node of each class not known to be exhausted
  unsigned int gen_seen;   // generation of the last full readiness scan
  int scan_u, scan_b;      // window starts of that scan
};

// Scheduler warp: claim an item.  Returns node >= 0 (and item), -1 when
// every node is exhausted, -2 on error or timeout, -3 when nothing is ready
// and block is false.
__device__ __forceinline__ int prg_claim(const PrgArgs &a, unsigned int *s_exh, unsigned int *s_rdy, PrgSched &st,
                                         int &item, int lane, bool block) {
  unsigned long long t0 = 0;
  unsigned int back = 64;
#pragma unroll 1
  for (;;) {
    // skip the exhausted prefix of each class (one lane; the masks are shared)
    if (lane == 0) {
      while (st.lo_u < a.nurgent && prg_bit(s_exh, st.lo_u)) st.lo_u++;
      while (st.lo_b < a.nnodes && prg_bit(s_exh, st.lo_b)) st.lo_b++;
    }
    st.lo_u = __shfl_sync(0xffffffffu, st.lo_u, 0);
    st.lo_b = __shfl_sync(0xffffffffu, st.lo_b, 0);
    if (st.lo_u >= a.nurgent && st.lo_b >= a.nnodes) return -1;
    // pending counts change only when a node completes (new generation)
    unsigned int g = 0;
    if (lane == 0) g = prg_ld_acquire(a.gen);
    g = __shfl_sync(0xffffffffu, g, 0);
    const bool rescan = g != st.gen_seen || st.lo_u != st.scan_u || st.lo_b != st.scan_b;
    st.gen_seen = g;
    st.scan_u = st.lo_u;
    st.scan_b = st.lo_b;
    // bulk items only below the concurrency limit: latency-bound chain work
    // slows several-fold beside saturated memory
    bool bulk_ok = true;
    if (a.bulk_limit > 0) {
      if (lane == 0) bulk_ok = prg_ld_relaxed(a.bulk_active) < (unsigned int)a.bulk_limit;
      bulk_ok = __shfl_sync(0xffffffffu, bulk_ok, 0);
    }
    const int n = lane < PRG_WIN ? st.lo_u + lane : st.lo_b + (lane - PRG_WIN);
    const bool valid = lane < PRG_WIN ? n < a.nurgent : (bulk_ok && n < a.nnodes);
    bool cand = false;
    int items = 0;
    if (valid && !prg_bit(s_exh, n)) {
      items = __ldg(&a.nodes[n].items);
      if (prg_bit(s_rdy, n)) {
        cand = true;
      } else if (rescan && prg_ld_acquire(&a.pending[n]) == 0u) {
        atomicOr(&s_rdy[n >> 5], 1u << (n & 31));
        cand = true;
      }
    }
    unsigned int m = __ballot_sync(0xffffffffu, cand);
    while (m) {
      const int ld = __ffs(m) - 1;
      int c = 0;
      if (lane == ld) {
        c = (int)atomicAdd(&a.claim[n], 1u);
        if (c >= items) atomicOr(&s_exh[n >> 5], 1u << (n & 31));
        else if (n >= a.nurgent && a.bulk_limit > 0) atomicAdd(a.bulk_active, 1u);
      }
      const int got = __shfl_sync(0xffffffffu, (lane == ld && c < items) ? 1 : 0, ld);
      if (got) {
        item = __shfl_sync(0xffffffffu, c, ld);
        return __shfl_sync(0xffffffffu, n, ld);
      }
      m &= m - 1u;
    }
    __syncwarp();
    if (!block) return -3;
    // nothing to claim: stop on error, else wait (bounded)
    if (prg_ld_relaxed(a.err)) return -2;
    const unsigned long long now = prg_clock();
    if (t0 == 0) {
      t0 = now;
    } else if (now - t0 > a.timeout_ns) {
      if (lane == 0) {
        atomicCAS(a.err, 0u, 1u);
        if (a.host_err) *(volatile unsigned int *)a.host_err = 1u;
      }
      return -2;
    }
    __nanosleep(back);
    back = back < 2048u ? back * 2u : back;
  }
}

// Scheduler warp: one item finished by the workers (after EMPTY).
__device__ __forceinline__ void prg_complete(const PrgArgs &a, int node, int lane) {
  if (lane == 0) {
    if (node >= a.nurgent && a.bulk_limit > 0) atomicSub(a.bulk_active, 1u);
    __threadfence();
    const unsigned int old = atomicAdd(&a.done[node], 1u);
    if (old + 1u == (unsigned int)__ldg(&a.nodes[node].items)) {
      __threadfence();
      const int s0 = __ldg(&a.nodes[node].succ0), ns = __ldg(&a.nodes[node].nsucc);
      for (int q = 0; q < ns; q++) atomicSub(&a.pending[__ldg(&a.succ[s0 + q])], 1u);
      __threadfence();
      atomicAdd(a.gen, 1u);
    }
  }
  __syncwarp();
}

struct PrgSlot {
  int node, kind;
  int u0, u1;  // the item's units [u0, u1)
};

// The scheduler warp's loop (kept out of line: its registers do not count
// against the worker path).
template <bool TRACE>
__device__ __noinline__ void prg_scheduler(const PrgArgs &a, unsigned int *s_exh, unsigned int *s_rdy, PrgSlot *s_slot,
                                           unsigned char *smem_raw, int lane) {
  PrgSched st{0, a.nurgent, 0xffffffffu, -1, -1};
  int pnode0 = -1, pnode1 = -1;  // node whose parameters are in buffer 0 / 1
  unsigned long long tp0 = 0, tp1 = 0, ts0 = 0, ts1 = 0;  // tracing: claim start, hand-over
  int titem0 = 0, titem1 = 0;
  auto stage = [&](int b, int node, int item) {
    if (lane == 0) {
      s_slot[b].node = node;
      if (node >= 0) {
        const long long per = __ldg(&a.nodes[node].per_item), units = __ldg(&a.nodes[node].units);
        const long long u0 = (long long)item * per;
        s_slot[b].kind = __ldg(&a.nodes[node].kind);
        s_slot[b].u0 = (int)u0;
        s_slot[b].u1 = (int)(u0 + per < units ? u0 + per : units);
      }
    }
    if (node >= 0 && node != (b ? pnode1 : pnode0)) {
      const int4 *src = (const int4 *)(a.blob + __ldg(&a.nodes[node].param_off));
      int4 *dst = (int4 *)(smem_raw + b * prg_pbuf());
      const int nv = __ldg(&a.nodes[node].param_bytes) >> 4;
      for (int q = lane; q < nv; q += 32) dst[q] = __ldg(src + q);
      (b ? pnode1 : pnode0) = node;
    }
    if (TRACE) (b ? titem1 : titem0) = item;
    __syncwarp();
  };
  auto publish = [&](int b) {
    if (TRACE) (b ? ts1 : ts0) = prg_clock();
    prg_bar_arrive(PRG_BAR_FULL);
  };
  auto record = [&](int b, int node) {
    if (!TRACE || lane != 0) return;
    const unsigned int r = atomicAdd(a.trace_n, 1u);
    if (r < a.trace_cap) {
      unsigned int sm;
      asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
      PrgTraceRec &T = a.trace[r];
      T.t_pick = b ? tp1 : tp0;
      T.t_start = b ? ts1 : ts0;
      T.t_end = prg_clock();
      T.plan_node = __ldg(&a.nodes[node].plan_index);
      T.item = b ? titem1 : titem0;
      T.sm = (int)sm;
      T.cta = blockIdx.x;
      T.launch = a.launch;
      T.pad_ = 0;
    }
  };
  int b = 0, item = 0;
  if (TRACE) tp0 = prg_clock();
  int run = prg_claim(a, s_exh, s_rdy, st, item, lane, true);
  stage(b, run, item);
  publish(b);
  if (run < 0) return;
  b ^= 1;
#pragma unroll 1
  for (;;) {
    // stage the next item while the workers run the current one
    if (TRACE) (b ? tp1 : tp0) = prg_clock();
    int nxt = prg_claim(a, s_exh, s_rdy, st, item, lane, false);
    if (nxt >= 0) stage(b, nxt, item);
    prg_bar_sync(PRG_BAR_EMPTY);
    record(b ^ 1, run);
    if (nxt >= 0) {
      publish(b);
      prg_complete(a, run, lane);
    } else {
      prg_complete(a, run, lane);
      if (nxt == -3) {
        if (TRACE) (b ? tp1 : tp0) = prg_clock();
        nxt = prg_claim(a, s_exh, s_rdy, st, item, lane, true);
      }
      stage(b, nxt < 0 ? -1 : nxt, item);
      publish(b);
      if (nxt < 0) return;
    }
    run = nxt;
    b ^= 1;
  }
}

template <int P, bool TRACE>
__global__ void __launch_bounds__(PRG_THREADS, P == MB_PREC_F64 ? 2 : 5) k_program(const __grid_constant__ PrgArgs a) {
  using R = typename Prec<P>::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned int s_exh[PRG_MAX_NODES / 32], s_rdy[PRG_MAX_NODES / 32];
  __shared__ PrgSlot s_slot[2];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int q = tid; q < PRG_MAX_NODES / 32; q += PRG_THREADS) {
    s_exh[q] = 0u;
    s_rdy[q] = 0u;
  }
  __syncthreads();

  if (warp == PRG_SCHED_WARP) {
    prg_scheduler<TRACE>(a, s_exh, s_rdy, s_slot, smem_raw, lane);
    return;
  }

  // ---------------- worker warps ----------------
  int b = 0;
#pragma unroll 1
  for (;;) {
    prg_bar_sync(PRG_BAR_FULL);
    if (s_slot[b].node < 0) break;
    const int kind = s_slot[b].kind, u0 = s_slot[b].u0, u1 = s_slot[b].u1;
    const unsigned char *pb = smem_raw + b * prg_pbuf();
    if (kind == PK_STB) {
      const StbParams &p = *(const StbParams *)pb;
      for (int g = u0 + tid; g < u1; g += PRG_WORKERS) stb_at<P>(p, g);
    } else if (kind == PK_REC) {
      const RecOpsParams &p = *(const RecOpsParams *)pb;
      for (int g = u0 + tid; g < u1; g += PRG_WORKERS) rec_point<P>(p, g);
    } else if (kind == PK_SPL) {
      const SplParamsP &p = *(const SplParamsP *)pb;
      const int sid = u0 + warp;
      if (warp < SPL_WARPS && sid < u1)
        spl_segment<P, false>(p, sid, lane, smem_raw + 2 * prg_pbuf() + warp * spl_warp_smem<R>());
    }
    prg_bar_arrive(PRG_BAR_EMPTY);
    b ^= 1;
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
  int32_t k, fluid_edge;  // bit 0: cell_f on the block edge; bit 1: cell_s is a half-way wall
};
struct DragParams {
  const DragLink *links;
  int n, pad_;
  const void *F;  // buffer read by the last block step of the drag block
  long long plane;
  double feqc[9];
  double *out;  // Fx, Fy
  Sh9 sh;       // shift of the stored words
};

// one CTA of 256 threads: it finds a free slot among the bulk work's CTAs as
// soon as one of them retires (a 1024-thread CTA waits for four)
constexpr int DRAG_THREADS = 256;
template <int P>
__global__ void __launch_bounds__(DRAG_THREADS) k_drag(const __grid_constant__ DragParams p) {
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
    const double fs = (double)ld_f<P>(F, (long long)k * p.plane + L.cell_f, k, p.sh);
    // returning value: feq(rho0, U0) at a block-edge FLUID cell (bit 0), the
    // outgoing value itself at a half-way wall (bit 1), else the on-node
    // wall's F_opp
    const double ff = (L.fluid_edge & 1) ? p.feqc[kd]
                      : (L.fluid_edge & 2) ? fs
                                           : (double)ld_f<P>(F, (long long)kd * p.plane + L.cell_s, kd, p.sh);
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
// One rectangle of cells of the L2 change: columns i0.., rows j0.. of block
// blk.  error_L2 runs in two parts (the interiors of split levels, and every
// other cell), each over its own list of boxes.
constexpr int L2_MAX_BOXES = 4 * MB_MAX_AREA;
struct L2Blk {
  int blk, i0, j0;
  int nx, pitch;  // box width; the block's pitch
  double inv_m;
  int ny, rt0;    // box rows; first row tile (256 cells of one box row) of this box
  int rtiles_x;   // row tiles per box row
  int pad_;
};
struct L2Params {
  const L2Blk *blocks;
  const IfBlk *blk;
  int nblk, ntiles;       // boxes; row tiles over all boxes
  long long total;
  double2 *partial;       // gridDim.x entries
  unsigned int *ticket;   // zero before the first launch; reset by the last CTA
  double *out;            // sum |u-up|^2 / m, sum |u|^2 / m
};

// A CTA walks row tiles (256 consecutive cells of one row of one block, the
// block and row uniform over the CTA) with a fixed stride, L2_ILP tiles per
// iteration with all their loads in flight before any use, so every cell is
// summed by the same thread in the same order on every call.  The last CTA
// (ticket counter) adds the per-CTA partials with all its threads in a fixed
// order and resets the ticket.
constexpr int L2_ILP = 4;
template <int P>
__global__ void __launch_bounds__(256) k_error_l2(const __grid_constant__ L2Params p) {
  using R = typename Prec<P>::R;
  __shared__ int s_rt0[L2_MAX_BOXES];
  for (int q = threadIdx.x; q < p.nblk; q += blockDim.x) s_rt0[q] = p.blocks[q].rt0;
  __syncthreads();
  double s1 = 0, s2 = 0;
  const int stride = gridDim.x;
  for (int t0 = blockIdx.x; t0 < p.ntiles; t0 += L2_ILP * stride) {
    R ux[L2_ILP], uy[L2_ILP], upx[L2_ILP], upy[L2_ILP];
    R *px[L2_ILP], *py[L2_ILP];
    double w[L2_ILP];
#pragma unroll
    for (int u = 0; u < L2_ILP; u++) {
      const int t = t0 + u * stride;
      px[u] = nullptr;
      if (t >= p.ntiles) continue;
      int lo = 0, hi = p.nblk - 1;  // last box whose first tile is <= t
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_rt0[mid] <= t) lo = mid; else hi = mid - 1;
      }
      const L2Blk &b = p.blocks[lo];
      const IfBlk &B = p.blk[b.blk];
      const int lt = t - s_rt0[lo];
      const int j = lt / b.rtiles_x;
      const int i = (lt - j * b.rtiles_x) * 256 + (int)threadIdx.x;
      if (i >= b.nx) continue;
      const int c = (b.j0 + j) * b.pitch + b.i0 + i;
      ux[u] = ((const R *)B.ux)[c];
      uy[u] = ((const R *)B.uy)[c];
      upx[u] = ((const R *)B.upx)[c];
      upy[u] = ((const R *)B.upy)[c];
      px[u] = (R *)B.upx + c;
      py[u] = (R *)B.upy + c;
      w[u] = b.inv_m;
    }
#pragma unroll
    for (int u = 0; u < L2_ILP; u++) {
      if (!px[u]) continue;
      const double x = ux[u], y = uy[u], xp = upx[u], yp = upy[u];
      s1 += ((x - xp) * (x - xp) + (y - yp) * (y - yp)) * w[u];
      s2 += (x * x + y * y) * w[u];
      *px[u] = ux[u];
      *py[u] = uy[u];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  __shared__ double a1[8], a2[8];
  __shared__ bool last;
  const int w0 = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { a1[w0] = s1; a2[w0] = s2; }
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
  if (!last) return;
  __threadfence();
  // thread q adds partials q, q + 256, ... in order; then a fixed tree
  double t1 = 0, t2 = 0;
  for (unsigned int q = threadIdx.x; q < gridDim.x; q += blockDim.x) {
    const double2 v = __ldcg(&p.partial[q]);
    t1 += v.x;
    t2 += v.y;
  }
  __shared__ double r1[256], r2[256];
  r1[threadIdx.x] = t1;
  r2[threadIdx.x] = t2;
  __syncthreads();
  for (int sz = blockDim.x / 2; sz > 0; sz >>= 1) {
    if ((int)threadIdx.x < sz) {
      r1[threadIdx.x] += r1[threadIdx.x + sz];
      r2[threadIdx.x] += r2[threadIdx.x + sz];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    p.out[0] = r1[0];
    p.out[1] = r2[0];
    *p.ticket = 0u;
  }
}

// Ring slots of one coarse-fine line <- the fine edge F (init_Fstore,
// multi/init_multi.h:3-28): every slot of fine point ip holds F at that point.
template <int P>
__global__ void k_slots_from_edge(const typename Prec<P>::S *F, long long plane, int fi0, int fj0, int fdi, int fdj,
                                  int pitch, int Nf, typename Prec<P>::R *slots, int slot0, const Sh9 sh) {
  for (int ip = blockIdx.x * blockDim.x + threadIdx.x; ip < Nf; ip += gridDim.x * blockDim.x) {
    const long long cell = (long long)(fj0 + ip * fdj) * pitch + (fi0 + ip * fdi);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const typename Prec<P>::R v = ld_f<P>(F, k * plane + cell, k, sh);
      for (int q = 0; q < 3; q++) slots[((long long)(slot0 + ip) * 3 + q) * 9 + k] = v;
    }
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
                              double f4, double f5, double f6, double f7, double f8, const Sh9 sh) {
  const double fv[9] = {f0, f1, f2, f3, f4, f5, f6, f7, f8};
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < 9 * plane;
       g += (long long)gridDim.x * blockDim.x) {
    const int k = int(g / plane);
    st_f<P>(F, g, k, (typename Prec<P>::R)fv[k], sh);
  }
}

template <int P>
__global__ void k_count_nonfinite(const typename Prec<P>::S *F, long long plane, const uint8_t *flags, int nx,
                                  int ny, int pitch, unsigned long long *count, const Sh9 sh) {
  unsigned long long bad = 0;
  const long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int j = int(g / nx), i = int(g - (long long)j * nx);
    const long long c = (long long)j * pitch + i;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      if constexpr (std::is_same<typename Prec<P>::S, h16c>::value) {
        if ((F[k * plane + c].x & 0x7fffu) == 0x7fffu) bad++;  // saturated: out of range, Inf or NaN
      } else {
        const double v = (double)ld_f<P>(F, k * plane + c, k, sh);
        if (!isfinite(v)) bad++;
      }
    }
  }
  if (bad) atomicAdd(count, bad);
}

// pitched device planes <-> dense FP64 staging buffer
template <int P>
__global__ void k_planes_to_f64(const typename Prec<P>::S *F, long long plane, int nx, int ny, int pitch, double *out,
                                const Sh9 sh) {
  const long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < 9 * n; g += (long long)gridDim.x * blockDim.x) {
    const int k = int(g / n);
    const long long r = g - k * n;
    const int j = int(r / nx), i = int(r - (long long)j * nx);
    out[g] = (double)ld_f<P>(F, k * plane + (long long)j * pitch + i, k, sh);
  }
}
template <int P>
__global__ void k_f64_to_planes(typename Prec<P>::S *F, long long plane, int nx, int ny, int pitch, const double *in,
                                const Sh9 sh) {
  const long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < 9 * n; g += (long long)gridDim.x * blockDim.x) {
    const int k = int(g / n);
    const long long r = g - k * n;
    const int j = int(r / nx), i = int(r - (long long)j * nx);
    st_f<P>(F, k * plane + (long long)j * pitch + i, k, (typename Prec<P>::R)in[g], sh);
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
