// l2_noalloc.cu - relative L2 change of a velocity field that allocates nothing.
//
// mb_error_L2 reduces into scratch that mb_create allocated.  Some callers
// cannot allocate device memory at all: a host application that owns the
// whole device through its own memory pool (a cudaMalloc outside the pool
// fails or breaks its accounting), or a time-stepping loop that must not
// synchronise the device (cudaMalloc and cudaFree do; the reference allocates
// and frees a buffer in every spline call).  mb_error_L2_noalloc serves them:
// the caller passes its own device arrays and a device output, and the
// per-CTA partial sums live in one fixed array in this file.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds it (MB_L2_NOALLOC_MAX_CTAS + 32 eight-byte words, about 19 KB)
// until the process exits.  Host code cannot use its name as a device
// address: the first call on each device looks the address up with
// cudaGetSymbolAddress, with that device current, and keeps it.  Make that
// first call before any stream capture.  All calls share the array and it
// keeps the last call's contents, so each call clears its counter first;
// calls that overlap on the GPU (two streams at once) race on it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/mblbm.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// words [0, 2*MAX_CTAS): partial sums of CTA b at 2b, 2b+1 (as doubles);
// word 2*MAX_CTAS: the finished-CTA counter
constexpr int kWords = 2 * MB_L2_NOALLOC_MAX_CTAS + 32;

struct SegParams {
  const double *ux[MB_L2_NOALLOC_MAX_SEGMENTS];
  const double *uy[MB_L2_NOALLOC_MAX_SEGMENTS];
  double *upx[MB_L2_NOALLOC_MAX_SEGMENTS];
  double *upy[MB_L2_NOALLOC_MAX_SEGMENTS];
  long long start[MB_L2_NOALLOC_MAX_SEGMENTS + 1];  // prefix of segment lengths
  double weight[MB_L2_NOALLOC_MAX_SEGMENTS];
  int nseg, pad_;
  unsigned long long *scratch;  // device address of g_l2_noalloc_scratch
  double *out;
};

}  // namespace

static __device__ __align__(256) unsigned long long g_l2_noalloc_scratch[kWords];

namespace {

// Same sums as error_L2_area + error_L2 (lbm/error_L2.h:3-91): every cell of
// every segment, weighted, u_prev <- u; one FP64 partial per CTA, summed in
// CTA order by the last CTA to finish.
__global__ void __launch_bounds__(kThreads) k_error_l2_static(const __grid_constant__ SegParams p) {
  double *part = reinterpret_cast<double *>(p.scratch);
  unsigned int *ticket = reinterpret_cast<unsigned int *>(p.scratch + 2 * MB_L2_NOALLOC_MAX_CTAS);
  const long long total = p.start[p.nseg];
  double s1 = 0, s2 = 0;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = p.nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.start[mid] <= g) lo = mid;
      else hi = mid - 1;
    }
    const long long c = g - p.start[lo];
    const double ux = p.ux[lo][c], uy = p.uy[lo][c], upx = p.upx[lo][c], upy = p.upy[lo][c];
    s1 += ((ux - upx) * (ux - upx) + (uy - upy) * (uy - upy)) * p.weight[lo];
    s2 += (ux * ux + uy * uy) * p.weight[lo];
    p.upx[lo][c] = ux;
    p.upy[lo][c] = uy;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  __shared__ double a1[kThreads / 32], a2[kThreads / 32];
  __shared__ bool last;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    a1[w] = s1;
    a2[w] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t1 = 0, t2 = 0;
    for (int q = 0; q < kThreads / 32; q++) {
      t1 += a1[q];
      t2 += a2[q];
    }
    part[2 * blockIdx.x] = t1;
    part[2 * blockIdx.x + 1] = t2;
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t1 = 0, t2 = 0;
    for (unsigned int q = 0; q < gridDim.x; q++) {
      t1 += __ldcg(&part[2 * q]);
      t2 += __ldcg(&part[2 * q + 1]);
    }
    p.out[0] = t1;
    p.out[1] = t2;
    p.out[2] = sqrt(t1) / sqrt(t2);
    *ticket = 0u;
  }
}

std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once.
int scratch_address(unsigned long long **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MB_ERR_NODEVICE;
  if (dev < 0 || dev >= kMaxDevices) return MB_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_l2_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "mblbm: cudaGetSymbolAddress(g_l2_noalloc_scratch) failed: %s\n", cudaGetErrorString(e));
      return MB_ERR_CUDA;
    }
    g_addr[dev] = p;
  }
  *out = static_cast<unsigned long long *>(g_addr[dev]);
  return MB_OK;
}

}  // namespace

extern "C" int mb_error_L2_noalloc(const mb_l2_segment *segs, int nseg, double *d_out, mb_stream stream) {
  if (!segs || !d_out || nseg < 1) return MB_ERR_INVALID;
  if (nseg > MB_L2_NOALLOC_MAX_SEGMENTS) {
    std::fprintf(stderr, "mblbm: mb_error_L2_noalloc takes at most %d segments (got %d)\n",
                 MB_L2_NOALLOC_MAX_SEGMENTS, nseg);
    return MB_ERR_UNSUPPORTED;
  }
  SegParams p{};
  long long total = 0;
  for (int s = 0; s < nseg; s++) {
    const mb_l2_segment &g = segs[s];
    if (g.n < 0 || (g.n > 0 && (!g.ux || !g.uy || !g.upx || !g.upy))) return MB_ERR_INVALID;
    p.ux[s] = g.ux;
    p.uy[s] = g.uy;
    p.upx[s] = g.upx;
    p.upy[s] = g.upy;
    p.weight[s] = g.weight;
    p.start[s] = total;
    total += g.n;
    if (total > MB_L2_NOALLOC_MAX_CELLS) {
      std::fprintf(stderr, "mblbm: mb_error_L2_noalloc takes at most %lld cells\n", (long long)MB_L2_NOALLOC_MAX_CELLS);
      return MB_ERR_UNSUPPORTED;
    }
  }
  p.start[nseg] = total;
  p.nseg = nseg;
  p.out = d_out;
  int e = scratch_address(&p.scratch);
  if (e) return e;
  cudaStream_t s = (cudaStream_t)stream;
  // the counter must start at zero whatever an earlier call left behind
  if (cudaMemsetAsync(p.scratch + 2 * MB_L2_NOALLOC_MAX_CTAS, 0, sizeof(unsigned int), s) != cudaSuccess)
    return MB_ERR_CUDA;
  long long blocks = (total + kThreads - 1) / kThreads;
  if (blocks < 1) blocks = 1;
  if (blocks > MB_L2_NOALLOC_MAX_CTAS) blocks = MB_L2_NOALLOC_MAX_CTAS;
  void *args[] = {&p};
  if (cudaLaunchKernel((const void *)k_error_l2_static, dim3((unsigned)blocks), dim3(kThreads), args, 0, s) !=
      cudaSuccess)
    return MB_ERR_CUDA;
  return MB_OK;
}
