// unet_umma.cuh - 3x3 convolutions of the surrogate U-Net as implicit GEMMs on
// the Blackwell tensor cores (tcgen05.mma, accumulators in tensor memory).
//
// GEMM view of one layer (stride 1, zero padding 1, NHWC BF16 activations):
//   Y[p][n] = sum over taps t = 0..8 and input channels c of
//             X[p shifted by tap t][c] * Wt[n][t][c]
// M = pixels, N = output channels, K = 9 x Cin.  A CTA owns a tile of 128
// pixels (R image rows x Cw columns, R * Cw = 128) and NT output channels.
// Pipeline per K step (one tap, CH input channels):
//   * one thread issues two TMA tile loads into a stage of shared memory:
//     the A tile as a 4-D box {CH channels, Cw columns, R rows, 1 image} of
//     the activation tensor at the tap's offset (the hardware fills the
//     out-of-image halo with zeros: the convolution's padding), and the B
//     tile as a 2-D box {CH, NT} of the weights [Cout][9 Cin];
//   * one thread issues CH/16 tcgen05.mma (M = 128, N = NT, K = 16, BF16
//     operands, FP32 accumulation in tensor memory) on the stage and
//     commits them to the stage's "empty" barrier, which frees the stage
//     for the next TMA load;
// after the last K step a commit to the "done" barrier releases the four
// warps, which read the accumulator rows of their 32 lanes from tensor
// memory (tcgen05.ld) and apply the epilogue: bias and ReLU into BF16
// (forward), or an FP32 store or accumulate (input gradient: the same
// kernel with the flipped, transposed weights).
// Both operands are K-major with the swizzle of their row length (CH = 16,
// 32, 64 channels: 32-, 64-, 128-byte swizzle), as the TMA writes them.
// Every wait on a barrier is bounded (about two seconds of global time);
// a wait that runs out sets the error word, and the CTA still releases its
// tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace umma {

constexpr int TM = 128;       // pixels per tile (MMA M)
constexpr int THREADS = 128;  // four warps
constexpr int STAGES = 4;
constexpr unsigned long long WAIT_NS = 2000000000ull;

struct ConvArgs {
  int H, W;            // image size of the layer
  int Cw, R;           // pixel tile: R rows x Cw columns
  int tiles_x, tiles_y;
  int Cin, NT;         // K = 9 Cin; N tile
  int relu, out_f32, accumulate;
  const float *bias;   // forward (BF16 output) only
  void *Y;             // output view: pixel p, channel n at Y[p * ycs + yco + n]
  int ycs, yco;
  int Cout;            // channels of the output tensor view written by this launch (n < Cout)
  unsigned int *err;   // set to 1 when a bounded wait ran out
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// bounded wait for the phase of the given parity; false when it ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  const unsigned a = smem_u32(bar);
  unsigned long long t0 = 0;
  for (unsigned n = 0;; n++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((n & 1023) == 1023) {
      const unsigned long long t = gtimer();
      if (t0 == 0) t0 = t;
      else if (t - t0 > WAIT_NS) return false;
      __nanosleep(64);
    }
  }
}

// TMA tile loads (this GPU's own global memory, no multicast)
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

// Shared-memory matrix descriptor of a K-major operand tile written by TMA
// with a 32/64/128-byte swizzle: rows of CH*2 bytes, 8-row groups SBO bytes
// apart; layout codes 6/4/2 (32B/64B/128B swizzle), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(unsigned saddr, unsigned sbo, unsigned layout) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1u << 16;                     // leading byte offset (unused by swizzled K-major tiles)
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;  // stride byte offset
  d |= (uint64_t)1u << 46;                     // version
  d |= (uint64_t)layout << 61;
  return d;
}
// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t instr_desc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 16 consecutive FP32 columns of this warp's 32 lanes (one row per thread)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  // the registers pass through the wait, so no use of them moves above it
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

template <int CH>
struct Cfg {
  static constexpr int A_BYTES = TM * CH * 2;
  static constexpr unsigned LAYOUT = CH == 64 ? 2u : (CH == 32 ? 4u : 6u);  // 128B / 64B / 32B swizzle
  static constexpr unsigned SBO = 8 * CH * 2;                                // 8 rows of CH channels
  __host__ __device__ static int b_bytes(int nt) { return nt * CH * 2; }
  static size_t smem(int nt) { return 1024 + (size_t)STAGES * (A_BYTES + b_bytes(nt)) + 256; }
};

template <int CH>
__global__ void __launch_bounds__(THREADS, 1)
    k_conv3x3_umma(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap wmap,
                   const __grid_constant__ ConvArgs a) {
  extern __shared__ __align__(1024) unsigned char dyn[];
  using C = Cfg<CH>;
  // stages start on a 1024-byte boundary (the 128-byte swizzle repeats every 8 rows of 128 bytes)
  unsigned char *base = (unsigned char *)(((uintptr_t)dyn + 1023) & ~(uintptr_t)1023);
  const int BB = C::b_bytes(a.NT);
  unsigned char *sA = base;
  unsigned char *sB = base + STAGES * C::A_BYTES;
  uint64_t *full = (uint64_t *)(sB + STAGES * BB);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tslot = (uint32_t *)(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ncols = a.NT <= 32 ? 32 : (a.NT <= 64 ? 64 : (a.NT <= 128 ? 128 : 256));

  if (warp == 0) {  // tensor memory for the NT x 128 FP32 accumulator
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  // this CTA's pixel tile and channel tile
  int t = blockIdx.x;
  const int tx = t % a.tiles_x;
  t /= a.tiles_x;
  const int ty = t % a.tiles_y;
  const int img = t / a.tiles_y;
  const int x0 = tx * a.Cw, y0 = ty * a.R;
  const int n0 = blockIdx.y * a.NT;
  const int kc = a.Cin / CH;  // K steps per tap
  const int KIT = 9 * kc;
  bool ok = true;

  if (warp == 0 && lane == 0) {  // TMA producer
    const unsigned bytes = (unsigned)(C::A_BYTES + BB);
    for (int it = 0; it < KIT && ok; it++) {
      const int s = it % STAGES;
      if (it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1)) { ok = false; break; }
      const int tap = it / kc, c0 = (it - tap * kc) * CH;
      const int dy = tap / 3 - 1, dx = tap % 3 - 1;
      mbar_expect_tx(&full[s], bytes);
      tma_load_4d(sA + s * C::A_BYTES, &xmap, c0, x0 + dx, y0 + dy, img, &full[s]);
      tma_load_2d(sB + s * BB, &wmap, tap * a.Cin + c0, n0, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    const uint32_t idesc = instr_desc(a.NT);
    for (int it = 0; it < KIT && ok; it++) {
      const int s = it % STAGES;
      if (!mbar_wait(&full[s], (it / STAGES) & 1)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned aa = smem_u32(sA + s * C::A_BYTES), ba = smem_u32(sB + s * BB);
#pragma unroll
      for (int k = 0; k < CH / 16; k++) {  // K = 16 per MMA: 32 bytes further along each row
        const uint64_t da = smem_desc(aa + k * 32, C::SBO, C::LAYOUT);
        const uint64_t db = smem_desc(ba + k * 32, C::SBO, C::LAYOUT);
        mma_f16(tmem, da, db, idesc, (it > 0 || k > 0) ? 1u : 0u);
      }
      mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
    }
    mma_commit(done);  // completes when every MMA issued above has
  }
  if (!ok) atomicExch(a.err, 1u);

  // epilogue: every warp waits for the accumulator, then reads its 32 rows
  __syncwarp();
  const bool acc_ready = mbar_wait(done, 0);
  if (!acc_ready) atomicExch(a.err, 1u);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (acc_ready) {
    const int m = warp * 32 + lane;  // pixel of this thread within the tile
    const int y = y0 + m / a.Cw, x = x0 + m % a.Cw;
    const long long p = ((long long)img * a.H + y) * a.W + x;
    const bool valid = y < a.H && x < a.W;
    for (int c = 0; c < a.NT; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      const int n = n0 + c;
      if (!valid || n >= a.Cout) continue;
      if (a.out_f32) {
        float *yp = (float *)a.Y + p * a.ycs + a.yco + n;
#pragma unroll
        for (int q = 0; q < 16; q += 4) {
          float4 o = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
          if (a.accumulate) {
            const float4 old = *(const float4 *)(yp + q);
            o.x += old.x;
            o.y += old.y;
            o.z += old.z;
            o.w += old.w;
          }
          *(float4 *)(yp + q) = o;
        }
      } else {
        __nv_bfloat16 *yp = (__nv_bfloat16 *)a.Y + p * a.ycs + a.yco + n;
        uint32_t packed[8];
#pragma unroll
        for (int q = 0; q < 16; q += 2) {
          float v0 = v[q] + a.bias[n + q], v1 = v[q + 1] + a.bias[n + q + 1];
          if (a.relu) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
          packed[q / 2] = *(const uint32_t *)&h;
        }
        *(uint4 *)yp = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        *(uint4 *)(yp + 8) = make_uint4(packed[4], packed[5], packed[6], packed[7]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

// ---------------------------------------------------------------------------
// Weight gradient: dW[co][t][ci] += sum over pixels p of dY[p][co] * X[p + off_t][ci]
// as a GEMM with M = 128 output channels (co), N = NT input channels (ci),
// K = pixels.  Both operands keep the channels contiguous in memory, so both
// are MN-major tiles: a stage holds 64 pixels (a box of R rows x Cw columns
// of one image) of 64-channel chunks, each chunk 64 rows (pixels) of 128
// bytes with the 128-byte swizzle, chunks 8 KB apart (the descriptor's
// leading byte offset), 8-row groups 1 KB apart (its stride byte offset).
// A CTA reduces one tap over a contiguous run of pixel boxes and adds its
// 128 x NT partial sums to dW with FP32 atomics.  Channels beyond Cout read
// as zeros (the TMA fills them) and are not written.
// ---------------------------------------------------------------------------
constexpr int WG_KP = 64;  // pixels per stage
struct WgradArgs {
  int H, W, Cw, R;       // image size; pixel box Cw columns x R rows (64 pixels)
  int bx, by;            // boxes per row block, per image
  int nboxes;            // boxes of the whole batch
  int boxes_per_cta;     // split-K: boxes of one CTA
  int Cin, Cout, NT;     // NT: input channels of this launch's tiles (a multiple of 64)
  float *dW;             // [Cout][9][Cin]
  unsigned int *err;
};

__host__ __device__ constexpr uint32_t instr_desc_mn(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(TM >> 4) << 24);
}
__device__ __forceinline__ uint64_t smem_desc_mn(unsigned saddr) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)(8192u >> 4) << 16;  // leading byte offset: next 64-channel chunk
  d |= (uint64_t)(1024u >> 4) << 32;  // stride byte offset: next 8 pixels
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;            // 128-byte swizzle
  return d;
}
inline size_t wgrad_smem(int nt) { return 1024 + (size_t)STAGES * (2 * 8192 + (size_t)(nt / 64) * 8192) + 256; }

__global__ void __launch_bounds__(THREADS, 1)
    k_wgrad_umma(const __grid_constant__ CUtensorMap gmap, const __grid_constant__ CUtensorMap xmap,
                 const __grid_constant__ WgradArgs a) {
  extern __shared__ __align__(1024) unsigned char dyn[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dyn + 1023) & ~(uintptr_t)1023);
  const int nch = a.NT / 64;
  const int ABYTES = 2 * 8192, BBYTES = nch * 8192;
  unsigned char *sA = base;
  unsigned char *sB = base + STAGES * ABYTES;
  uint64_t *full = (uint64_t *)(sB + STAGES * BBYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tslot = (uint32_t *)(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ncols = a.NT <= 64 ? 64 : (a.NT <= 128 ? 128 : 256);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  const int co0 = blockIdx.y * TM;
  const int tap = blockIdx.z % 9, ci0 = (blockIdx.z / 9) * a.NT;
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;
  const int b0 = blockIdx.x * a.boxes_per_cta;
  const int b1 = min(a.nboxes, b0 + a.boxes_per_cta);
  const int KIT = b1 - b0;
  bool ok = true;
  if (warp == 0 && lane == 0) {  // TMA producer
    const unsigned bytes = (unsigned)(ABYTES + BBYTES);
    for (int it = 0; it < KIT && ok; it++) {
      const int s = it % STAGES;
      if (it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1)) { ok = false; break; }
      int b = b0 + it;
      const int bxi = b % a.bx;
      b /= a.bx;
      const int byi = b % a.by, img = b / a.by;
      const int x0 = bxi * a.Cw, y0 = byi * a.R;
      mbar_expect_tx(&full[s], bytes);
      tma_load_4d(sA + s * ABYTES, &gmap, co0, x0, y0, img, &full[s]);
      tma_load_4d(sA + s * ABYTES + 8192, &gmap, co0 + 64, x0, y0, img, &full[s]);
      for (int c = 0; c < nch; c++)
        tma_load_4d(sB + s * BBYTES + c * 8192, &xmap, ci0 + 64 * c, x0 + dx, y0 + dy, img, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    const uint32_t idesc = instr_desc_mn(a.NT);
    for (int it = 0; it < KIT && ok; it++) {
      const int s = it % STAGES;
      if (!mbar_wait(&full[s], (it / STAGES) & 1)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned aa = smem_u32(sA + s * ABYTES), ba = smem_u32(sB + s * BBYTES);
#pragma unroll
      for (int k = 0; k < WG_KP / 16; k++)  // 16 pixels per MMA: 16 rows of 128 bytes further
        mma_f16(tmem, smem_desc_mn(aa + k * 2048), smem_desc_mn(ba + k * 2048), idesc, (it > 0 || k > 0) ? 1u : 0u);
      mma_commit(&empty[s]);
    }
    mma_commit(done);
  }
  if (!ok) atomicExch(a.err, 1u);
  __syncwarp();
  const bool acc_ready = KIT > 0 && mbar_wait(done, 0);
  if (KIT > 0 && !acc_ready) atomicExch(a.err, 1u);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (acc_ready) {
    const int co = co0 + warp * 32 + lane;  // row of this thread
    for (int c = 0; c < a.NT; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      if (co >= a.Cout) continue;
      float *d = a.dW + ((long long)co * 9 + tap) * a.Cin + ci0 + c;
#pragma unroll
      for (int q = 0; q < 16; q++)
        if (ci0 + c + q < a.Cin) atomicAdd(d + q, v[q]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

}  // namespace umma
