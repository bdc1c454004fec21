// mblbm.cu - device context, plan execution (direct or CUDA graph) and the C ABI.
//
// Replaces main() of zhangya9741/Multi-block-LBM-GPU (Multi-block-LBM.cu:19-230)
// as a library: allocation, initialisation, the coarse time step of
// evolution() and the per-step diagnostics, each behind an extern "C" entry
// point that returns a status code and enqueues work on the caller's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mblbm.h"
#include "kernels.cuh"
#include "mblbm_internal.h"

using namespace mblbm;
using namespace mblbm::dev;

#define MB_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      std::fprintf(stderr, "mblbm: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_),    \
                   __FILE__, __LINE__);                                                        \
      return MB_ERR_CUDA;                                                                      \
    }                                                                                          \
  } while (0)

namespace {

size_t prec_bytes(int prec) {
  return prec == MB_PREC_F64 ? 8 : ((prec == MB_PREC_F16S || prec == MB_PREC_F16C) ? 2 : 4);
}
size_t real_bytes(int prec) { return prec == MB_PREC_F64 ? 8 : 4; }
bool prec_shifted(int prec) { return prec == MB_PREC_F32 || prec == MB_PREC_F16S || prec == MB_PREC_F16C; }
// FP32 storage and the h16c form subtract the free stream's equilibrium (the
// stored words are then small wherever the flow is near the free stream;
// measured on developed shedding: FP32 Cd 9e-6 from FP64 against 2.5e-4 with
// f - w, h16c -0.62 % against -1.05 %); IEEE FP16 keeps f - w (its f - feq
// form loses 5 % of Cd there)
int default_shift(int prec) {
  return (prec == MB_PREC_F32 || prec == MB_PREC_F16C) ? MB_SHIFT_FEQ0 : MB_SHIFT_W;
}

// One part of error_L2 (interiors of split levels, or every other cell) as
// boxes in device memory.
struct L2Part {
  L2Blk *d = nullptr;
  int nbox = 0, ntiles = 0, grid = 0;
};

struct DevPlanNode {
  NodeKind kind;
  bool background = false;  // bandwidth-bound bulk work: lowest scheduling priority
  bool slack = false;       // off the estimated critical path: one priority step below the chain
  // launch
  void *func = nullptr;
  dim3 grid, block;
  size_t smem = 0;
  // parameter blocks (one of them used)
  StbParams stb;
  RecOpsParams rec;
  SplParamsP spl;
  L2Params l2;
  DragParams drag;
  void *args[1];
  std::vector<int> deps;
};

// One executor launch: its arguments, the claim | done | pending state and
// the state's values at launch (copied over it before every launch), grid and
// dynamic shared memory.
struct PrgLaunch {
  PrgArgs prg{};
  unsigned int *state = nullptr;
  const unsigned int *init = nullptr;
  size_t state_bytes = 0;
  int grid = 0;
  size_t smem = 0;
};

struct CompiledPlan {
  std::vector<PlanNode> nodes;
  std::vector<DevPlanNode> dn;
  std::vector<void *> dev_allocs;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  SchedState end;
  long long kernels = 0;
  double *d_diag_res = nullptr;  // diagnostic plans: Fx, Fy and the two L2 sums of every part, per coarse step
  int diag_steps = 0;
  // persistent executor: the whole plan (graph mode 3), or the chain
  // segments of a hybrid graph (mode 4)
  bool prg_built = false;
  PrgLaunch prgm;
  std::vector<PrgLaunch> segs;
  ~CompiledPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void *p : dev_allocs) cudaFree(p);
  }
};

}  // namespace

struct mb_ctx {
  int prec = MB_PREC_F32;
  int device = 0;
  mb_geometry geo{};
  int nblk = 0;
  std::vector<BlockLayout> bl;
  std::vector<std::vector<uint8_t>> hflags;
  // device state
  std::vector<IfBlk> blk;  // host mirror of the device block table
  IfBlk *d_blk = nullptr;
  std::vector<void *> allocs;
  void *d_slots = nullptr;
  long long n_slot_points = 0;
  std::vector<SplLine> spl_lines;
  std::vector<int> spl_coef0;  // per line: offset of its c' / 1/den table (units of 2 values)
  void *d_spl_coef = nullptr;  // per line: c'_i and 1/den_i of the spline system
  // drag
  int drag_area = 0;
  int n_drag = 0;
  DragLink *d_links = nullptr;
  double *d_drag_out = nullptr;
  double *h_drag_out = nullptr;  // pinned
  // L2
  // error_L2 in two parts (interiors of split levels, the rest), per split mask
  std::map<unsigned, std::array<L2Part, L2_NPARTS>> l2parts;
  double2 *d_l2_partial[L2_NPARTS] = {};  // per part: parts may run concurrently
  unsigned int *d_l2_ticket[L2_NPARTS] = {};
  double *d_l2_out = nullptr;
  double *h_l2_out = nullptr;  // pinned
  int l2_grid = 0;
  int l2_tiles = 0;
  // mb_step_diag: per-step Fx, Fy and the two L2 sums (device, pinned host)
  double *d_diag = nullptr;
  double *h_diag = nullptr;
  size_t diag_cap = 0;
  long long total_cells = 0;
  // misc scratch
  unsigned long long *d_count = nullptr;
  double *d_stage = nullptr;
  size_t stage_elems = 0;
  double feqc[9]{};
  // collision and boundary options (k_block_step_x)
  StbOptions opt{};
  long long n_alt_walls = 0;  // HBB and slip cells over all blocks
  // same-level copies fused into block steps
  std::vector<CcLevel> cc;
  std::vector<CcEntry *> d_cclist;  // per level: the copies of fusable levels (k_cc_pull)
  int fuse_cc = 1;
  int fuse_tmp = 0;  // splines do the next temporal interpolation of their line (mb_set_fusion bit 1)
  // ... in place, beside the fine level's substep (mb_set_fusion bit 2; on:
  // 103.1 against 104.3 us per step in FP32 on config 2, 93.3 against 93.8 in
  // FP16 storage, 18 launches per coarse step against 20)
  int fuse_early = 1;
  // f_c points beside the fine level's last block step (mb_set_fusion bit 3)
  // and record launches split by what they wait for (bit 4): both measured
  // within run-to-run noise of the defaults on config 2, so off
  int fuse_fc = 0;
  int split_waits = 0;
  unsigned early_levels = 0;  // levels whose temporal edge cells carry CF_TSKIP
  // scheduler
  SchedState state;
  bool inited = false;
  int use_graph = 1;
  int period = 1;
  long long split_cells = 1000000;
  long long stream_cells = 2000000;
  unsigned split_mask = 0;            // nonzero: the levels to split (bit per level), overriding split_cells
  int bulk_levels = 0;                // 1: whole-level block steps that stream with hints are bulk (low priority) work   // block steps over >= this many cells use evict-first cache hints (0: never)
  int stb_variant[MB_MAX_LEVEL] = {0};  // 0: one cell per thread, 1: quads (k_block_step_q)
  int bulk_ctas_per_sm = 0;             // >0: cap interior (bulk) block-step grids at this many CTAs per SM
  int tb_ctas_per_sm = 2;               // persistent CTAs per SM of the bulk-copy block step (variant 5)
  int num_sms = 148;
  // persistent executor
  unsigned int *d_prg_err = nullptr;    // device error word of k_program
  unsigned int *h_prg_err = nullptr;    // mapped pinned mirror, read after any synchronisation
  unsigned int *d_prg_err_host = nullptr;
  unsigned long long prg_timeout_ns = 2000000000ull;
  int prg_bulk_cells = 512;             // cells per item of bulk block-step nodes
  int prg_urgent_cells = 256;           // cells per item of the other block-step nodes
  int prg_periods = 2;                  // scheduler periods per executor launch
  int hyb_ctas_per_sm = 2;              // executor CTAs per SM of a hybrid graph's chain segments
  int plan_steps = 24;                  // coarse steps per replayed graph (rounded up to periods)
  int prg_bulk_limit = 0;               // CTAs allowed on bulk items at once (0: no limit)
  int rec_points = 32;                  // interface points per record CTA / executor item
  int spl_segs = 1;                     // spline segments per CTA / executor item
  // minimum dynamic shared memory per spline / record CTA: caps how many CTAs
  // of these latency-bound launches one SM takes, so that a launch that
  // starts while a block step still holds most SMs spreads over the SMs that
  // free up instead of piling onto the first ones
  int spl_cta_smem = 96 * 1024;
  int rec_cta_smem = 0;
  int bulk_cta_smem = 0;  // unused shared memory reserved by each bulk (interior) block-step CTA
  // the fine levels' F and rho/u and the interface slots, one allocation
  // (the range of the L2 access-policy window, mb_set_l2_persist)
  void *fine_arena = nullptr;
  size_t fine_bytes = 0;
  size_t l2_persist = 0;  // bytes of L2 set aside for it (0: none)
  int shift_mode = MB_SHIFT_W;  // stored words h = f - s: s = w, or feq(rho0, U0)
  Shift shift{};
  PrgTraceRec *d_trace = nullptr;       // executor trace (mb_set_program_trace)
  unsigned int *d_trace_n = nullptr;
  unsigned int trace_cap = 0;
  int prg_launches = 0;
  std::map<std::string, std::unique_ptr<CompiledPlan>> plans;
  long long kernels_last_call = 0;
  long long updates_per_step = 0;
};

namespace {

// The shift of a context's stored words and the collision's constants for it
// (kernels.cuh, Shift): s = w (rho_s = 1, U_s = 0) or s = feq(rho0, U0) of
// the configuration.  Precisions that store f itself get s = 0.
Shift make_shift(const mb_ctx *c, int mode) {
  Shift sh{};
  if (!prec_shifted(c->prec)) {
    sh.sym = 1;
    return sh;
  }
  const mb_config &cfg = c->geo.config;
  const double rs = mode == MB_SHIFT_FEQ0 ? cfg.rho0 : 1.0;
  const double ux = mode == MB_SHIFT_FEQ0 ? cfg.U0[0] : 0.0, uy = mode == MB_SHIFT_FEQ0 ? cfg.U0[1] : 0.0;
  const double uv = ux * ux + uy * uy;
  double sd[9];
  for (int k = 0; k < 9; k++) {
    const double eu = ex(k) * ux + ey(k) * uy;
    sd[k] = wd(k) * rs * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uv);
    sh.v.s[k] = (float)sd[k];
  }
  // c_k = w_k (rho_s + 3 e_k.J_s) - s_k = -w_k rho_s (4.5 (e_k.U_s)^2 - 1.5 |U_s|^2), per pair
  const int rep[5] = {0, 1, 2, 5, 8};
  for (int q = 0; q < 5; q++) {
    const int k = rep[q];
    const double eu = ex(k) * ux + ey(k) * uy;
    sh.c[q] = (float)(-wd(k) * rs * (4.5 * eu * eu - 1.5 * uv));
  }
  sh.rhos = (float)rs;
  sh.jx = (float)(rs * ux);
  sh.jy = (float)(rs * uy);
  sh.q2 = (float)(rs * uv);
  sh.qd = (float)(rs * (ux * ux - uy * uy));
  sh.qx = (float)(rs * ux * uy);
  sh.sym = 1;
  for (int k = 0; k < 9; k++)
    if (sh.v.s[k] != sh.v.s[opp(k)] || sh.v.s[k] != sh.v.s[slip(k)]) sh.sym = 0;
  return sh;
}

// Runs STMT with P bound to the runtime precision and S to its storage type.
#define MB_DISPATCH(prec, STMT)                                     \
  do {                                                              \
    if ((prec) == MB_PREC_F64) {                                    \
      constexpr int P = MB_PREC_F64;                                \
      using S = double;                                             \
      STMT;                                                         \
    } else if ((prec) == MB_PREC_F32) {                             \
      constexpr int P = MB_PREC_F32;                                \
      using S = float;                                              \
      STMT;                                                         \
    } else if ((prec) == MB_PREC_F32U) {                            \
      constexpr int P = MB_PREC_F32U;                               \
      using S = float;                                              \
      STMT;                                                         \
    } else if ((prec) == MB_PREC_F16C) {                            \
      constexpr int P = MB_PREC_F16C;                               \
      using S = h16c;                                               \
      STMT;                                                         \
    } else {                                                        \
      constexpr int P = MB_PREC_F16S;                               \
      using S = __half;                                             \
      STMT;                                                         \
    }                                                               \
  } while (0)

template <typename T>
int dalloc(mb_ctx *c, T **p, size_t n) {
  void *q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return MB_ERR_NOMEM;
  c->allocs.push_back(q);
  *p = (T *)q;
  return MB_OK;
}

// Links of the drag sum (fdrag_store, force_block.h:78-127), i-outer,
// j-inner, k: SOLID_SBB and SOLID_HBB cells of the drag block with a FLUID
// upstream neighbour (slip walls are left out).  Replaces any earlier list.
int upload_drag_links(mb_ctx *c) {
  const int a = c->drag_area;
  const BlockLayout &b = c->bl[a];
  const auto &fl = c->hflags[a];
  std::vector<DragLink> links;
  for (int i = 0; i < b.nx; i++)
    for (int j = 0; j < b.ny; j++) {
      const long long cs = (long long)j * b.pitch + i;
      if ((fl[cs] & 3) != CT_SOLID || (fl[cs] & CF_SLIP)) continue;
      for (int k = 0; k < 9; k++) {
        const int id = i - ex(k), jd = j - ey(k);
        if (id < 0 || id > b.nx - 1 || jd < 0 || jd > b.ny - 1) continue;
        const long long cf = (long long)jd * b.pitch + id;
        if ((fl[cf] & 3) != CT_FLUID) continue;
        const int32_t kind = ((fl[cf] & CF_EDGE) ? 1 : 0) | ((fl[cs] & CF_HBB) ? 2 : 0);
        links.push_back({(int32_t)cs, (int32_t)cf, k, kind});
      }
    }
  if (c->d_links) {
    auto it = std::find(c->allocs.begin(), c->allocs.end(), (void *)c->d_links);
    if (it != c->allocs.end()) c->allocs.erase(it);
    cudaFree(c->d_links);
    c->d_links = nullptr;
  }
  c->n_drag = (int)links.size();
  int e;
  if ((e = dalloc(c, &c->d_links, links.size()))) return e;
  if (!links.empty())
    MB_CUDA(cudaMemcpy(c->d_links, links.data(), links.size() * sizeof(DragLink), cudaMemcpyHostToDevice));
  return MB_OK;
}

// MB_* cell type code of a flag byte
int flag_code(uint8_t f) {
  const int t = f & 3;
  if (t == CT_FLUID) return MB_FLUID;
  if (t == CT_SOLID) return (f & CF_HBB) ? MB_SOLID_HBB : (f & CF_SLIP) ? MB_SOLID_SLIP : MB_SOLID_SBB;
  return MB_C_BOUNDARY;
}

int launch_grid(long long n, int threads) { return (int)std::min<long long>((n + threads - 1) / threads, 148LL * 64); }

// ---- templated dispatch over precision -------------------------------------
template <template <int> class K, typename... A>
void *kfunc(int prec) {
  if (prec == MB_PREC_F64) return K<MB_PREC_F64>::ptr();
  if (prec == MB_PREC_F32) return K<MB_PREC_F32>::ptr();
  if (prec == MB_PREC_F32U) return K<MB_PREC_F32U>::ptr();
  if (prec == MB_PREC_F16C) return K<MB_PREC_F16C>::ptr();
  return K<MB_PREC_F16S>::ptr();
}
template <int P> struct KStb { static void *ptr() { return (void *)k_block_step<P, 1>; } };
template <int P> struct KStb2 { static void *ptr() { return (void *)k_block_step<P, 2>; } };
template <int P> struct KStbR { static void *ptr() { return (void *)k_block_step_r<P, false>; } };
template <int P> struct KStbRI { static void *ptr() { return (void *)k_block_step_r<P, true>; } };
template <int P> struct KStbP { static void *ptr() { return (void *)k_block_step_p<P, false>; } };
template <int P> struct KStbPI { static void *ptr() { return (void *)k_block_step_p<P, true>; } };
template <int P> struct KStbQ { static void *ptr() { return (void *)k_block_step_q<P>; } };
template <int P> struct KStbO {
  static void *ptr() {
    if constexpr (sizeof(typename Prec<P>::S) == 2) return (void *)k_block_step_o<P>;
    else return nullptr;  // octets exist for the 16-bit stored forms only
  }
};
template <int P> struct KStbX { static void *ptr() { return (void *)k_block_step_x<P>; } };
template <int P> struct KCcp { static void *ptr() { return (void *)k_cc_pull<P>; } };
template <int P> struct KFcp { static void *ptr() { return (void *)k_fc_pull<P>; } };
template <int P> struct KStbTb { static void *ptr() { return (void *)k_block_step_tb<P>; } };
int tb_smem(int prec) {
  switch (prec) {
    case MB_PREC_F64: return TbCfg<double>::SMEM;
    case MB_PREC_F16S: return TbCfg<__half>::SMEM;
    case MB_PREC_F16C: return TbCfg<h16c>::SMEM;
    default: return TbCfg<float>::SMEM;
  }
}
template <int P> struct KRec { static void *ptr() { return (void *)k_records<P>; } };
template <int P> struct KSpl { static void *ptr() { return (void *)k_spline<P>; } };
template <int P> struct KDrag { static void *ptr() { return (void *)k_drag<P>; } };
template <int P> struct KL2 { static void *ptr() { return (void *)k_error_l2<P>; } };
template <int P> struct KPrg { static void *ptr() { return (void *)k_program<P, false>; } };
template <int P> struct KBStb { static void *ptr() { return (void *)kb_block_step<P>; } };
template <int P> struct KBStbPs { static void *ptr() { return (void *)kb_block_step_ps<P>; } };
template <int P> struct KBStbPp { static void *ptr() { return (void *)kb_block_step_pp<P>; } };
template <int P> struct KBStbPt { static void *ptr() { return (void *)kb_block_step_pt<P>; } };
template <int P> struct KBRec { static void *ptr() { return (void *)kb_records<P>; } };
template <int P> struct KBSpl { static void *ptr() { return (void *)kb_spline<P>; } };
template <int P> struct KPrgT { static void *ptr() { return (void *)k_program<P, true>; } };
size_t program_smem(int prec) { return prec == MB_PREC_F64 ? prg_smem<double>() : prg_smem<float>(); }

// dynamic shared memory of k_spline per warp: two 12 x window arrays and the
// window's c' and 1/den
constexpr int MB_CTA_SMEM_MAX = 200 * 1024;  // largest spread request (B200: 227 KB per CTA)

size_t spline_smem(int prec) {
  return prec == MB_PREC_F64 ? SPL_WARPS * spl_warp_smem_pf<double>() : SPL_WARPS * spl_warp_smem_pf<float>();
}

// ---- node lowering ------------------------------------------------------------
// cells of a block in a block-step region (see StbRegion)
long long region_cells(int nx, int ny, int region) {
  const long long all = (long long)nx * ny;
  const long long in = (nx > 4 && ny > 4) ? (long long)(nx - 4) * (ny - 4) : 0;
  return region == STB_INTERIOR ? in : (region == STB_RIM ? all - in : all);
}

bool stb_uses_quads(const mb_ctx *c, int level, int region);
int stb_tile(const mb_ctx *c, int level, int region);

// any collision or boundary option on: every block step runs k_block_step_x
bool options_on(const mb_ctx *c) { return c->opt.coll != MB_COLL_BGK || c->opt.has_force || c->n_alt_walls > 0; }

// Launch parameters of a block-step node.  total counts cells for the
// one-cell-per-thread kernel and warp tiles for the quad kernel (quads).
StbParams make_stb(mb_ctx *c, int a0, int a1, uint64_t parity, int macro_all, int write_macros, int region,
                   int tile, int ccpull) {
  const bool quads = tile > 0;
  StbParams p{};
  p.nblk = a1 - a0;
  p.a0 = a0;
  p.ccpull = ccpull;
  p.err_host = c->d_prg_err_host;
  p.macro_all = macro_all;
  p.write_macros = write_macros;
  p.region = region;
  for (int k = 0; k < 9; k++) p.feqc[k] = c->feqc[k];
  p.sh = c->shift;
  p.rho0 = c->geo.config.rho0;
  p.u0x = c->geo.config.U0[0];
  p.u0y = c->geo.config.U0[1];
  p.opt = c->opt;
  long long cell = 0, wt = 0, rt = 0, pt = 0, tb = 0, level_cells = 0;
  for (int a = a0; a < a1; a++) level_cells += region_cells(c->blk[a].nx, c->blk[a].ny, region);
  p.evict_first = c->stream_cells > 0 && level_cells >= c->stream_cells;
  for (int a = a0; a < a1; a++) {
    const IfBlk &B = c->blk[a];
    const int cur = (parity >> a) & 1;
    StbBlk &s = p.b[a - a0];
    s.Fin = B.F[cur];
    s.Fout = B.F[cur ^ 1];
    s.rho = B.rho;
    s.ux = B.ux;
    s.uy = B.uy;
    s.flags = B.flags;
    s.nx = B.nx;
    s.ny = B.ny;
    s.pitch = B.pitch;
    s.gid = a;
    s.plane = B.plane;
    s.cell0 = cell;
    s.rv_tau = c->geo.Areas[a].rv_tau;
    s.dt = 1.0 / c->geo.Areas[a].m;
    cell += region_cells(B.nx, B.ny, region);
    // quad and octet kernels: rows of the region in warp tiles of 128 (quads)
    // or 256 (octets) cells
    const int tw = tile > 0 ? tile : 128;
    s.tiles_x = (B.nx + tw - 1) / tw;
    s.row0 = region == STB_INTERIOR ? 2 : 0;
    const int nrows = region == STB_INTERIOR ? std::max(0, B.ny - 4) : B.ny;
    s.wt0 = wt;
    wt += (long long)s.tiles_x * nrows;
    // range kernel: CTAs of 256 consecutive cells of the region
    s.rcol0 = region == STB_INTERIOR ? 2 : 0;
    s.rw = std::max(0, region == STB_INTERIOR ? B.nx - 4 : B.nx);
    s.rcells = s.rw > 0 ? (int)std::min<long long>((long long)s.rw * nrows, 1LL << 30) : 0;
    s.rinv_w = s.rw > 0 ? 1.0f / (float)s.rw : 0.f;
    s.cta0 = (int)rt;
    rt += (s.rcells + 255) / 256;
    // pair kernel: CTAs of 256 consecutive pairs of the region
    s.ppr = (s.rw + 1) / 2;
    s.npairs = s.ppr > 0 ? (int)std::min<long long>((long long)s.ppr * nrows, 1LL << 30) : 0;
    s.pinv = s.ppr > 0 ? 1.0f / (float)s.ppr : 0.f;
    s.pcta0 = (int)pt;
    pt += (s.npairs + 255) / 256;
    // bulk-copy kernel: interior rows 2..ny-3 in tiles of 256 columns from column 0
    s.tb0 = tb;
    s.tb_tiles = (B.nx > 4 && B.ny > 4) ? (B.nx - 2 + TB_TW - 1) / TB_TW : 0;
    tb += (long long)s.tb_tiles * std::max(0, B.ny - 4);
  }
  p.tb_items = tb;
  p.rctas = rt;
  p.pctas = pt;
  p.total = quads ? wt : cell;
  return p;
}

// octet kernel: variant 6 on a level of a 16-bit stored form (others run 0)
bool stb_uses_octets(const mb_ctx *c, int level) { return c->stb_variant[level] == 6 && prec_bytes(c->prec) == 2; }

// the rim is always stepped one cell per thread
bool stb_uses_quads(const mb_ctx *c, int level, int region) {
  return region != STB_RIM && (c->stb_variant[level] == 1 || stb_uses_octets(c, level)) && c->use_graph != 3 &&
         !(c->use_graph == 4 && region != STB_INTERIOR) && !options_on(c);
}

// warp-tile width of a launch: 128 cells (quads), 256 (octets), 0 (others)
int stb_tile(const mb_ctx *c, int level, int region) {
  if (!stb_uses_quads(c, level, region)) return 0;
  return stb_uses_octets(c, level) ? 256 : 128;
}

bool background_capped(const mb_ctx *c, bool background) { return background && c->bulk_ctas_per_sm > 0; }

// the range kernel indexes 9 planes of a block with 32-bit offsets
bool rows_fit(const mb_ctx *c, const StbParams &p) {
  for (int t = 0; t < p.nblk; t++)
    if (9 * p.b[t].plane >= (1LL << 31) || (long long)p.b[t].ny * p.b[t].pitch >= (1LL << 31) ||
        p.b[t].rcells >= (1 << 24) || p.b[t].npairs >= (1 << 24))  // rows come from float products
      return false;
  (void)c;
  return p.rctas < (1LL << 31) && p.pctas < (1LL << 31);
}

// One-cell-per-thread block steps on the chain (not bulk work) run in CTAs
// of 128 threads: beside the bulk interior's CTAs an SM then fits seven of
// them (896 threads) where it fits three of 256 (768).  Measured on config 2:
// 100.7 against 101.7 us per step in FP32, 90.0 against 90.3 in FP16 storage.
constexpr int STB_CHAIN_THREADS = 128;

// kernel and grid of a block-step launch (variant 0: one cell per thread,
// 1: quads, 2: two cells per thread, 3: row tiles); background grids may be
// capped
void stb_launch_shape(const mb_ctx *c, int level, int region, bool background, const StbParams &p, void **func,
                      dim3 *grid) {
  if (options_on(c)) {
    *func = kfunc<KStbX>(c->prec);
    *grid = dim3((unsigned)std::max<long long>((p.total + 255) / 256, 0));
    return;
  }
  if (stb_uses_quads(c, level, region)) {  // the quad and octet grids are never capped
    *func = stb_uses_octets(c, level) ? kfunc<KStbO>(c->prec) : kfunc<KStbQ>(c->prec);
    *grid = dim3((unsigned)((p.total + 7) / 8));  // 8 warp tiles per CTA
    return;
  }
  if (c->stb_variant[level] == 5 && region == STB_INTERIOR && p.tb_items > 0) {
    *func = kfunc<KStbTb>(c->prec);
    const int per_sm = c->bulk_ctas_per_sm > 0 ? c->bulk_ctas_per_sm : c->tb_ctas_per_sm;
    *grid = dim3((unsigned)std::min<long long>(p.tb_items, (long long)c->num_sms * per_sm));
    return;
  }
  if (c->stb_variant[level] == 4 && region != STB_RIM && !background_capped(c, background) && rows_fit(c, p)) {
    *func = region == STB_INTERIOR ? kfunc<KStbPI>(c->prec) : kfunc<KStbP>(c->prec);
    *grid = dim3((unsigned)p.pctas);
    return;
  }
  if (c->stb_variant[level] == 3 && region != STB_RIM && !background_capped(c, background) && rows_fit(c, p)) {
    *func = region == STB_INTERIOR ? kfunc<KStbRI>(c->prec) : kfunc<KStbR>(c->prec);
    *grid = dim3((unsigned)p.rctas);
    return;
  }
  const bool two = c->stb_variant[level] == 2;
  *func = two ? kfunc<KStb2>(c->prec) : kfunc<KStb>(c->prec);
  const long long per = two ? 512 : (background ? 256 : STB_CHAIN_THREADS);
  long long ctas = (p.total + per - 1) / per;
  if (background && c->bulk_ctas_per_sm > 0) ctas = std::min<long long>(ctas, (long long)c->bulk_ctas_per_sm * c->num_sms);
  *grid = dim3((unsigned)std::max<long long>(ctas, 0));
}

// The boxes of both error_L2 parts for a split mask (bit per level): part 0
// the interiors (distance >= 2 from the block edge) of split levels, part 1
// their rims and every cell of the other levels, blocks in order.
int l2_parts(mb_ctx *c, unsigned mask, const L2Part **out) {
  auto it = c->l2parts.find(mask);
  if (it == c->l2parts.end()) {
    std::array<L2Part, L2_NPARTS> parts;
    const mb_layout &L = c->geo.layout;
    for (int q = 0; q < L2_NPARTS; q++) {
      std::vector<L2Blk> bx;
      long long tiles = 0;
      auto add = [&](int a, int i0, int j0, int w, int h) {
        if (w <= 0 || h <= 0) return;
        L2Blk b{};
        b.blk = a;
        b.i0 = i0;
        b.j0 = j0;
        b.nx = w;
        b.ny = h;
        b.pitch = c->bl[a].pitch;
        b.inv_m = 1.0 / c->geo.Areas[a].m;
        b.rtiles_x = (w + 255) / 256;
        b.rt0 = (int)tiles;
        tiles += (long long)b.rtiles_x * h;
        bx.push_back(b);
      };
      for (int l = 0; l < L.LEVEL; l++) {
        const bool sp = (mask >> l) & 1;
        if (q != 0 && q != 1 + l) continue;
        for (int a = L.ASP[l]; a < L.ASP[l + 1]; a++) {
          const int nx = c->bl[a].nx, ny = c->bl[a].ny;
          const bool inner = sp && nx > 4 && ny > 4;
          if (q == 0) {
            if (inner) add(a, 2, 2, nx - 4, ny - 4);
          } else if (inner) {
            add(a, 0, 0, nx, 2);
            add(a, 0, ny - 2, nx, 2);
            add(a, 0, 2, 2, ny - 4);
            add(a, nx - 2, 2, 2, ny - 4);
          } else {
            add(a, 0, 0, nx, ny);
          }
        }
      }
      if ((int)bx.size() > L2_MAX_BOXES || tiles > c->l2_tiles) return MB_ERR_UNSUPPORTED;
      L2Part &pt = parts[q];
      pt.nbox = (int)bx.size();
      pt.ntiles = (int)tiles;
      pt.grid = (int)std::min<long long>(tiles, c->l2_grid);
      if (!bx.empty()) {
        if (int e = dalloc(c, &pt.d, bx.size())) return e;
        MB_CUDA(cudaMemcpy(pt.d, bx.data(), bx.size() * sizeof(L2Blk), cudaMemcpyHostToDevice));
      }
    }
    it = c->l2parts.emplace(mask, parts).first;
  }
  *out = it->second.data();
  return MB_OK;
}

// CTAs of a part's launch: two per SM at most, so that the parts running
// beside the fine levels' chain (the interiors, and each level's part at the
// turn of a step) leave the chain's launches free slots (the same grid
// everywhere: the sums' order follows the grid)
int l2_grid_of(const mb_ctx *c, const L2Part *pt, int q) {
  (void)q;
  return std::min(pt[q].grid, 2 * c->num_sms);
}

L2Params l2_params(mb_ctx *c, const L2Part *pt, int q, double *out) {
  L2Params p{};
  p.blocks = pt[q].d;
  p.blk = c->d_blk;
  p.nblk = pt[q].nbox;
  p.ntiles = pt[q].ntiles;
  p.total = c->total_cells;
  p.partial = c->d_l2_partial[q];
  p.ticket = c->d_l2_ticket[q];
  p.out = out;
  return p;
}

// the levels the plans split into interior and rim nodes
unsigned current_split_levels(const mb_ctx *c) {
  PlanCompiler pc(c->geo, c->bl, c->hflags, c->spl_lines);
  pc.split_cells = c->split_cells;
  pc.split_mask = c->split_mask;
  return pc.split_levels();
}

int lower_plan(mb_ctx *c, CompiledPlan &cp) {
  cp.dn.resize(cp.nodes.size());
  for (const PlanNode &n : cp.nodes)
    if (n.kind == NK_DRAG || n.kind == NK_L2) cp.diag_steps = std::max(cp.diag_steps, n.level + 1);
  if (cp.diag_steps > 0) {  // zero: a part without cells adds nothing
    const size_t bytes = (size_t)cp.diag_steps * DIAG_STRIDE * sizeof(double);
    if (cudaMalloc(&cp.d_diag_res, bytes) != cudaSuccess) return MB_ERR_NOMEM;
    cp.dev_allocs.push_back(cp.d_diag_res);
    MB_CUDA(cudaMemset(cp.d_diag_res, 0, bytes));
  }
  for (size_t q = 0; q < cp.nodes.size(); q++) {
    const PlanNode &n = cp.nodes[q];
    DevPlanNode &d = cp.dn[q];
    d.kind = n.kind;
    d.deps = n.deps;
    if (n.kind == NK_STB) {
      d.stb = make_stb(c, n.a0, n.a1, n.parity, n.macro_all, 1, n.region, stb_tile(c, n.level, n.region), n.ccpull);
      d.stb.tskip = n.tskip;
      d.stb.fcskip = n.fcskip;
      // bulk: interiors of split levels, and whole levels streamed with
      // evict-first hints when bulk_levels is set
      d.background = (n.region == STB_INTERIOR) || (c->bulk_levels && n.region == STB_ALL && d.stb.evict_first);
      d.block = dim3(256);
      stb_launch_shape(c, n.level, n.region, d.background, d.stb, &d.func, &d.grid);
      if (d.func == kfunc<KStb>(c->prec) && !d.background) d.block = dim3(STB_CHAIN_THREADS);
      if (d.func == kfunc<KStbTb>(c->prec)) {
        d.block = dim3(TB_THREADS);
        d.smem = (size_t)tb_smem(c->prec);
      } else if (d.background && c->bulk_cta_smem > 0) {
        // shared memory the kernel does not use, reserved so that an SM holds
        // fewer bulk CTAs and keeps room for the chain's (mb_set_bulk_spread)
        d.smem = (size_t)c->bulk_cta_smem;
      }
      d.args[0] = &d.stb;
    } else if (n.kind == NK_L2) {
      const int part = n.part;
      const L2Part *pt = nullptr;
      if (int e = l2_parts(c, (unsigned)n.a0, &pt)) return e;
      d.l2 = l2_params(c, pt, part, cp.d_diag_res + DIAG_STRIDE * n.level + 2 + 2 * part);
      d.func = kfunc<KL2>(c->prec);
      d.block = dim3(256);
      d.grid = dim3((unsigned)l2_grid_of(c, pt, part));
      d.background = part == 0;  // beside the fine levels' chain: bulk work
      d.args[0] = &d.l2;
    } else if (n.kind == NK_DRAG) {
      const int a = c->drag_area;
      const IfBlk &B = c->blk[a];
      d.drag = DragParams{};
      d.drag.links = c->d_links;
      d.drag.n = c->n_drag;
      d.drag.F = B.F[((n.parity >> a) & 1) ^ 1];  // the buffer the block's last step read
      d.drag.plane = B.plane;
      for (int k = 0; k < 9; k++) d.drag.feqc[k] = c->feqc[k];
      d.drag.sh = c->shift.v;
      d.drag.out = cp.d_diag_res + DIAG_STRIDE * n.level;
      d.func = kfunc<KDrag>(c->prec);
      d.block = dim3(DRAG_THREADS);
      d.grid = dim3(1);
      d.args[0] = &d.drag;
    } else if (n.kind == NK_FCP) {
      // the CF_FCSRC cells of the step's blocks and their f_c points
      d.stb = make_stb(c, n.a0, n.a1, n.parity, n.macro_all, 1, STB_ALL, 0, 0);
      std::vector<StbFc> fc;
      for (const FcFuse &e : n.fc) {
        if (!(e.bits & (RB_WRITE_F | RB_WRITE_M))) continue;
        StbFc x{};
        x.gid = e.src_block;
        x.cell = e.src_cell;
        x.dblk = e.dst_block;
        x.dcell = e.dst_cell;
        x.bits = e.bits & (RB_WRITE_F | RB_WRITE_M);
        x.dbuf = e.dst_buf;
        x.para = e.para;
        fc.push_back(x);
      }
      std::stable_sort(fc.begin(), fc.end(), [](const StbFc &u, const StbFc &v) {
        return u.gid != v.gid ? u.gid < v.gid : u.cell < v.cell;
      });
      std::vector<FcCell> cells;
      size_t e = 0;
      for (int a = n.a0; a < n.a1; a++) {
        const BlockLayout &b = c->bl[a];
        for (int j = 0; j < b.ny; j++)
          for (int i = 0; i < b.nx; i++) {
            const long long cell = (long long)j * b.pitch + i;
            if ((c->hflags[a][(size_t)cell] & (3 | CF_FCSRC)) != (CT_FLUID | CF_FCSRC)) continue;
            FcCell fcl{};
            fcl.gid = a;
            fcl.i = i;
            fcl.j = j;
            while (e < fc.size() && (fc[e].gid < a || (fc[e].gid == a && fc[e].cell < cell))) e++;
            fcl.e0 = (int)e;
            while (e < fc.size() && fc[e].gid == a && fc[e].cell == cell) e++;
            fcl.e1 = (int)e;
            cells.push_back(fcl);
          }
      }
      const size_t b1 = fc.size() * sizeof(StbFc), b2 = cells.size() * sizeof(FcCell);
      unsigned char *dp = nullptr;
      if (cudaMalloc(&dp, std::max<size_t>(b1 + b2, 16)) != cudaSuccess) return MB_ERR_NOMEM;
      cp.dev_allocs.push_back(dp);
      if (b1) MB_CUDA(cudaMemcpy(dp, fc.data(), b1, cudaMemcpyHostToDevice));
      if (b2) MB_CUDA(cudaMemcpy(dp + b1, cells.data(), b2, cudaMemcpyHostToDevice));
      d.stb.fc = (const StbFc *)dp;
      d.stb.fc_n = (int)fc.size();
      d.stb.fccell = (const FcCell *)(dp + b1);
      d.stb.fc_cells = (int)cells.size();
      d.stb.fcblk = c->d_blk;
      d.func = kfunc<KFcp>(c->prec);
      d.block = dim3(128);
      d.grid = dim3((unsigned)((cells.size() + 127) / 128));
      d.args[0] = &d.stb;
    } else if (n.kind == NK_CCP) {
      d.stb = make_stb(c, n.a0, n.a1, n.parity, 0, 1, STB_ALL, 0, 0);
      d.stb.cc_list = c->d_cclist[n.level];
      d.stb.cc_n = (int)c->cc[n.level].links.size();
      d.func = kfunc<KCcp>(c->prec);
      d.block = dim3(128);
      d.grid = dim3((unsigned)((d.stb.cc_n + 127) / 128));
      d.args[0] = &d.stb;
    } else if (n.kind == NK_REC) {
      if ((int)n.ops.size() > REC_MAX_OPS) return MB_ERR_UNSUPPORTED;
      d.rec = RecOpsParams{};
      std::vector<uint8_t> mask;
      int total = 0;
      for (size_t o = 0; o < n.ops.size(); o++) {
        const int r0 = n.ops[o].first, cnt = n.ops[o].second;
        const Rec &a = n.recs[r0];
        RecOp &op = d.rec.ops[o];
        op.type = a.type;
        op.dst_block = a.dst_block;
        op.src_block = a.src_block;
        op.m0 = a.m0;
        op.m1 = a.m1;
        op.m2 = a.m2;
        op.count = cnt;
        op.dst0 = a.dst_cell;
        op.src0 = a.src;
        op.dstride = cnt > 1 ? n.recs[r0 + 1].dst_cell - a.dst_cell : 0;
        op.sstride = cnt > 1 ? n.recs[r0 + 1].src - a.src : 0;
        if (a.type == REC_FC_SLOT) {  // single point: sstride carries its slot point
          if (cnt != 1) return MB_ERR_INVALID;
          op.sstride = int32_t(a.m0 | (a.m1 << 8) | (a.pad << 16));
        }
        uint8_t full = 0, all_same = 1;
        const uint8_t buf_bits = uint8_t(a.bits & ~(RB_WRITE_F | RB_WRITE_M));
        for (int q = 0; q < cnt; q++) {
          const Rec &r = n.recs[r0 + q];
          // every op is a line: affine in the point index
          if (r.dst_cell != op.dst0 + q * op.dstride || r.src != op.src0 + q * op.sstride ||
              uint8_t(r.bits & ~(RB_WRITE_F | RB_WRITE_M)) != buf_bits)
            return MB_ERR_INVALID;
          full |= r.bits & (RB_WRITE_F | RB_WRITE_M);
          if ((r.bits & (RB_WRITE_F | RB_WRITE_M)) != (a.bits & (RB_WRITE_F | RB_WRITE_M))) all_same = 0;
        }
        op.bits = all_same ? a.bits : uint8_t(buf_bits | full);
        op.has_mask = all_same ? 0 : 1;
        op.mask_off = (int)mask.size();
        if (!all_same)
          for (int q = 0; q < cnt; q++) mask.push_back(uint8_t(n.recs[r0 + q].bits & (RB_WRITE_F | RB_WRITE_M)));
        d.rec.op_start[o] = total;
        total += cnt;
      }
      d.rec.nops = (int)n.ops.size();
      d.rec.op_start[n.ops.size()] = total;
      d.rec.total = total;
      uint8_t *dm = nullptr;
      if (cudaMalloc(&dm, std::max<size_t>(mask.size(), 1)) != cudaSuccess) return MB_ERR_NOMEM;
      cp.dev_allocs.push_back(dm);
      if (!mask.empty()) MB_CUDA(cudaMemcpy(dm, mask.data(), mask.size(), cudaMemcpyHostToDevice));
      d.rec.mask = dm;
      d.rec.slots = c->d_slots;
      d.rec.sh = c->shift.v;
      std::memcpy(d.rec.tw, n.tw, sizeof(n.tw));
      for (int a = 0; a < c->nblk; a++) {
        const IfBlk &B = c->blk[a];
        d.rec.b[a] = {{B.F[0], B.F[1]}, B.rho, B.ux, B.uy, B.plane, B.tau, B.m, 0};
      }
      d.func = kfunc<KRec>(c->prec);
      // small CTAs spread a launch's scattered accesses (one cache sector
      // per value on lines across rows) over many SMs' load/store units
      d.block = dim3(c->rec_points);
      d.grid = dim3((unsigned)((total + c->rec_points - 1) / c->rec_points));
      d.smem = (size_t)c->rec_cta_smem;
      d.args[0] = &d.rec;
    } else {
      if ((int)n.spl.size() > SPL_MAX_TASKS) return MB_ERR_UNSUPPORTED;
      d.spl = SplParamsP{};
      int nseg = 0;
      for (size_t t = 0; t < n.spl.size(); t++) {
        const SplLine &L = c->spl_lines[n.spl[t].line];
        const IfBlk &Cb = c->blk[L.coarse], &Fb = c->blk[L.fine];
        SplTaskP &T = d.spl.t[t];
        T.Nc = L.Nc; T.Nf = L.Nf; T.r = L.r; T.slot0 = L.slot0;
        T.ci0 = L.ci0; T.cj0 = L.cj0; T.cdi = L.cdi; T.cdj = L.cdj;
        T.fi0 = L.fi0; T.fj0 = L.fj0; T.fdi = L.fdi; T.fdj = L.fdj;
        T.coef0 = c->spl_coef0[n.spl[t].line];
        T.m0 = n.spl[t].m0;
        T.mask_off = n.spl[t].mask_off;
        T.seg0 = nseg;
        T.para = L.para;
        T.Fc = Cb.F[n.spl[t].src_buf];
        T.Mc[0] = Cb.rho; T.Mc[1] = Cb.ux; T.Mc[2] = Cb.uy;
        T.Mf[0] = Fb.rho; T.Mf[1] = Fb.ux; T.Mf[2] = Fb.uy;
        T.cplane = Cb.plane;
        T.cpitch = Cb.pitch;
        T.fpitch = Fb.pitch;
        T.tmp = n.spl[t].tmp;
        T.tmask_off = n.spl[t].tmask_off;
        for (int q = 0; q < 3; q++) {
          T.tm[q] = n.spl[t].tm[q];
          T.tw[q] = n.spl[t].tw[q];
        }
        T.Ft = n.spl[t].tmp ? Fb.F[n.spl[t].tbuf] : nullptr;
        T.fplane = Fb.plane;
        nseg += (L.Nc - 1 + SPL_SEG - 1) / SPL_SEG;
      }
      d.spl.ntask = (int)n.spl.size();
      d.spl.nseg = nseg;
      uint8_t *dm = nullptr;
      if (cudaMalloc(&dm, std::max<size_t>(n.spl_mask.size(), 1)) != cudaSuccess) return MB_ERR_NOMEM;
      cp.dev_allocs.push_back(dm);
      if (!n.spl_mask.empty()) MB_CUDA(cudaMemcpy(dm, n.spl_mask.data(), n.spl_mask.size(), cudaMemcpyHostToDevice));
      d.spl.mask = dm;
      d.spl.slots = c->d_slots;
      d.spl.coef = c->d_spl_coef;
      d.spl.sh = c->shift.v;
      d.func = kfunc<KSpl>(c->prec);
      d.block = dim3(32 * c->spl_segs);
      d.grid = dim3((unsigned)((nseg + c->spl_segs - 1) / c->spl_segs));
      d.smem = std::max(spline_smem(c->prec) / SPL_WARPS * c->spl_segs, (size_t)c->spl_cta_smem);
      d.args[0] = &d.spl;
    }
  }
  cp.kernels = 0;
  for (auto &d : cp.dn) cp.kernels += d.grid.x ? 1 : 0;
  return MB_OK;
}

int run_direct(CompiledPlan &cp, cudaStream_t s) {
  for (auto &d : cp.dn) {
    if (d.grid.x == 0) continue;
    MB_CUDA(cudaLaunchKernel(d.func, d.grid, d.block, d.args, d.smem, s));
  }
  return MB_OK;
}

// Interior nodes of split levels get the lowest priority and every other
// kernel the highest, one step less for nodes with slack: pending CTAs of the
// latency-bound fine-level chain are then dispatched ahead of the queued bulk
// CTAs as SMs free up, and a fine-level step that can wait (the first
// substep of a level, beside the coarser level's step) yields to the chain.
int set_priority(cudaGraphNode_t node, bool background, bool slack = false) {
  int least = 0, greatest = 0;
  MB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  cudaKernelNodeAttrValue v{};
  v.priority = background ? least : (slack && greatest < least ? greatest + 1 : greatest);
  MB_CUDA(cudaGraphKernelNodeSetAttribute(node, cudaKernelNodeAttributePriority, &v));
  return MB_OK;
}

// The access-policy window of the chain kernels: the fine levels' arena,
// hits persisting in the set-aside part of L2, in proportion to its size.
bool l2_window(const mb_ctx *c, cudaAccessPolicyWindow *w) {
  if (!c->l2_persist || !c->fine_arena) return false;
  int dev = 0, maxw = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, dev) != cudaSuccess || maxw <= 0)
    return false;
  w->base_ptr = c->fine_arena;
  w->num_bytes = std::min(c->fine_bytes, (size_t)maxw);
  w->hitRatio = (float)std::min(1.0, (double)c->l2_persist / (double)w->num_bytes);
  w->hitProp = cudaAccessPropertyPersisting;
  w->missProp = cudaAccessPropertyStreaming;
  return true;
}

// Marks the nodes whose start may slip by more than SLACK_US without
// lengthening the plan, by longest paths over a rough cost model of each
// launch (a fixed latency plus a term in its CTAs; bulk nodes cost nothing
// here, as they run beside the chain).
constexpr double SLACK_US = 3.0;
void mark_slack(CompiledPlan &cp) {
  const int nd = (int)cp.dn.size();
  std::vector<double> cost(nd, 0), head(nd, 0), tail(nd, 0);
  for (int q = 0; q < nd; q++) {
    const DevPlanNode &d = cp.dn[q];
    if (d.grid.x == 0 || d.background) continue;
    if (d.kind == NK_STB) cost[q] = 2.0 + d.grid.x / 200.0;
    else if (d.kind == NK_SPL) cost[q] = 4.0 + d.grid.x / 20.0;
    else if (d.kind == NK_REC) cost[q] = 3.0 + d.grid.x / 100.0;
    else cost[q] = 2.0;
  }
  for (int q = 0; q < nd; q++)  // nodes are in topological order
    for (int p : cp.dn[q].deps) head[q] = std::max(head[q], head[p] + cost[p]);
  for (int q = nd - 1; q >= 0; q--) tail[q] = std::max(tail[q], cost[q]);
  for (int q = nd - 1; q >= 0; q--)
    for (int p : cp.dn[q].deps) tail[p] = std::max(tail[p], cost[p] + tail[q]);
  double T = 0;
  for (int q = 0; q < nd; q++) T = std::max(T, head[q] + tail[q]);
  for (int q = 0; q < nd; q++) cp.dn[q].slack = T - (head[q] + tail[q]) > SLACK_US;
}

int build_graph(CompiledPlan &cp, bool pdl, const cudaAccessPolicyWindow *win = nullptr) {
  mark_slack(cp);
  MB_CUDA(cudaGraphCreate(&cp.graph, 0));
  std::vector<cudaGraphNode_t> gn(cp.dn.size(), nullptr);
  for (size_t q = 0; q < cp.dn.size(); q++) {
    DevPlanNode &d = cp.dn[q];
    std::vector<cudaGraphNode_t> deps;
    for (int p : d.deps)
      if (gn[p]) deps.push_back(gn[p]);
    if (d.grid.x == 0) {  // nothing to do, but later nodes may order through it
      MB_CUDA(cudaGraphAddEmptyNode(&gn[q], cp.graph, deps.data(), deps.size()));
      continue;
    }
    cudaKernelNodeParams kp{};
    kp.func = d.func;
    kp.gridDim = d.grid;
    kp.blockDim = d.block;
    kp.sharedMemBytes = (unsigned)d.smem;
    kp.kernelParams = d.args;
    kp.extra = nullptr;
    if (!pdl) {
      MB_CUDA(cudaGraphAddKernelNode(&gn[q], cp.graph, deps.data(), deps.size(), &kp));
      if (int e = set_priority(gn[q], d.background, d.slack)) return e;
      if (win && !d.background) {  // chain kernels keep the fine levels' lines in the set-aside L2
        cudaKernelNodeAttrValue v{};
        v.accessPolicyWindow = *win;
        MB_CUDA(cudaGraphKernelNodeSetAttribute(gn[q], cudaKernelNodeAttributeAccessPolicyWindow, &v));
      }
      continue;
    }
    // programmatic edges between kernels of the fine-level chain: this kernel
    // is scheduled once every producer CTA has started and waits in-kernel
    // for their completion.  Edges from or into background (bulk interior)
    // nodes stay plain: early CTAs of a consumer would hold SM slots while
    // waiting, slots the chain or the bulk work needs.
    std::vector<cudaGraphNode_t> plain;
    std::vector<cudaGraphNode_t> prog;
    for (int p : d.deps) {
      if (!gn[p]) continue;
      (cp.dn[p].grid.x && !cp.dn[p].background && !d.background ? prog : plain).push_back(gn[p]);
    }
    MB_CUDA(cudaGraphAddKernelNode(&gn[q], cp.graph, plain.data(), plain.size(), &kp));
    if (int e = set_priority(gn[q], d.background, d.slack)) return e;
    for (cudaGraphNode_t from : prog) {
      cudaGraphEdgeData ed{};
      ed.from_port = cudaGraphKernelNodePortProgrammatic;
      ed.to_port = 0;
      ed.type = cudaGraphDependencyTypeProgrammatic;
      MB_CUDA(cudaGraphAddDependencies_v2(cp.graph, &from, &gn[q], &ed, 1));
    }
  }
  // node priorities only take effect when the graph is instantiated with them
  MB_CUDA(cudaGraphInstantiateWithFlags(&cp.exec, cp.graph, cudaGraphInstantiateFlagUseNodePriority));
  return MB_OK;
}

int set_smem_limits(int prec) {
  // every kernel a bulk (interior) node may run may reserve unused shared
  // memory up to the spread limit (mb_set_bulk_spread)
  {
    void *fns[] = {kfunc<KStb>(prec), kfunc<KStb2>(prec), kfunc<KStbQ>(prec), kfunc<KStbPI>(prec),
                   kfunc<KStbP>(prec), kfunc<KStbRI>(prec), kfunc<KStbR>(prec), kfunc<KStbO>(prec)};
    for (void *f : fns)
      if (f) MB_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, MB_CTA_SMEM_MAX));
  }
  MB_CUDA(cudaFuncSetAttribute(kfunc<KSpl>(prec), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)std::max(spline_smem(prec), (size_t)MB_CTA_SMEM_MAX)));
  MB_CUDA(cudaFuncSetAttribute(kfunc<KRec>(prec), cudaFuncAttributeMaxDynamicSharedMemorySize, MB_CTA_SMEM_MAX));
  MB_CUDA(cudaFuncSetAttribute(kfunc<KStbTb>(prec), cudaFuncAttributeMaxDynamicSharedMemorySize, tb_smem(prec)));
  MB_CUDA(cudaFuncSetAttribute(kfunc<KPrg>(prec), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)program_smem(prec)));
  MB_CUDA(cudaFuncSetAttribute(kfunc<KPrgT>(prec), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)program_smem(prec)));
  MB_CUDA(cudaFuncSetAttribute(kfunc<KBSpl>(prec), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)((sizeof(SplParamsP) + 15) / 16 * 16 + spline_smem(prec))));
  return MB_OK;
}

// ---- persistent executor ------------------------------------------------------
// Item counts of a lowered node in the executor, and its work kind.
void program_units(const mb_ctx *c, const DevPlanNode &d, int *kind, long long *units, int *per) {
  if (d.kind == NK_STB) {
    *kind = PK_STB;
    *units = d.stb.total;
    *per = d.background ? c->prg_bulk_cells : c->prg_urgent_cells;
  } else if (d.kind == NK_REC) {
    *kind = PK_REC;
    *units = d.rec.total;
    *per = c->rec_points;
  } else {
    *kind = PK_SPL;
    *units = d.spl.nseg;
    *per = c->spl_segs;
  }
}

// Dependencies of every node over the nodes that have work (a node without
// work passes its own on to its successors).
std::vector<std::vector<int>> effective_deps(const CompiledPlan &cp, const std::vector<char> &has_work) {
  const int nd = (int)cp.dn.size();
  std::vector<std::vector<int>> eff(nd);
  for (int q = 0; q < nd; q++) {
    std::vector<int> out;
    for (int p : cp.dn[q].deps) {
      if (has_work[p]) out.push_back(p);
      else out.insert(out.end(), eff[p].begin(), eff[p].end());
    }
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
    eff[q] = std::move(out);
  }
  return eff;
}

// Lays out the nodes `order` (plan indices, a topological order) of a plan
// as one executor program: node table, successor lists over these nodes
// only, parameter blob and the claim / done / pending state with its launch
// values, in one device allocation owned by the plan.  `nurgent` leading
// nodes are urgent, the rest bulk.  `ctas_per_sm` caps the grid (0: as many
// CTAs as fit).
int program_from(mb_ctx *c, CompiledPlan &cp, const std::vector<int> &order, const std::vector<std::vector<int>> &eff,
                 int nurgent, int ctas_per_sm, PrgLaunch &L) {
  const int nd = (int)cp.dn.size();
  const int nn = (int)order.size();
  if (nn > PRG_MAX_NODES) return MB_ERR_UNSUPPORTED;
  std::vector<int> pos(nd, -1);
  for (int i = 0; i < nn; i++) pos[order[i]] = i;
  std::vector<std::vector<int>> succ(nn);
  std::vector<unsigned int> pending(nn, 0);
  for (int i = 0; i < nn; i++)
    for (int p : eff[order[i]]) {
      if (pos[p] < 0) continue;  // outside this program: ordered by the launch
      succ[pos[p]].push_back(i);
      pending[i]++;
    }
  std::vector<PrgNode> nodes(nn);
  std::vector<int> sl;
  std::vector<unsigned char> blob;
  long long items = 0;
  for (int i = 0; i < nn; i++) {
    const int q = order[i];
    const DevPlanNode &d = cp.dn[q];
    int kind = 0, per = 1;
    long long units = 0;
    program_units(c, d, &kind, &units, &per);
    if (units >= (1LL << 31) - (1LL << 25)) return MB_ERR_UNSUPPORTED;  // item bounds are 32-bit
    PrgNode &N = nodes[i];
    N = PrgNode{};
    N.kind = kind;
    N.units = units;
    N.per_item = per;
    N.items = (int)((units + per - 1) / per);
    items += N.items;
    const void *src = kind == PK_STB ? (const void *)&d.stb : kind == PK_REC ? (const void *)&d.rec : (const void *)&d.spl;
    const size_t sz = kind == PK_STB ? sizeof(StbParams) : kind == PK_REC ? sizeof(RecOpsParams) : sizeof(SplParamsP);
    const size_t padded = (sz + 15) / 16 * 16;
    N.param_off = (int)blob.size();
    N.param_bytes = (int)padded;
    blob.resize(blob.size() + padded, 0);
    std::memcpy(blob.data() + N.param_off, src, sz);
    N.succ0 = (int)sl.size();
    N.nsucc = (int)succ[i].size();
    N.plan_index = q;
    sl.insert(sl.end(), succ[i].begin(), succ[i].end());
  }
  // one allocation: nodes | succ | blob | init state | state
  auto al = [](size_t v) { return (v + 255) / 256 * 256; };
  const size_t o_nodes = 0, o_succ = al(std::max(nn, 1) * sizeof(PrgNode)),
               o_blob = o_succ + al(std::max<size_t>(sl.size(), 1) * sizeof(int));
  const size_t st_bytes = (3 * (size_t)nn + 2) * sizeof(unsigned int);  // claim, done, pending, generation, bulk
  const size_t o_init = o_blob + al(std::max<size_t>(blob.size(), 16)), o_state = o_init + al(st_bytes);
  const size_t total = o_state + al(st_bytes);
  std::vector<unsigned char> host(total, 0);
  if (nn) std::memcpy(host.data() + o_nodes, nodes.data(), nn * sizeof(PrgNode));
  if (!sl.empty()) std::memcpy(host.data() + o_succ, sl.data(), sl.size() * sizeof(int));
  if (!blob.empty()) std::memcpy(host.data() + o_blob, blob.data(), blob.size());
  if (nn) std::memcpy(host.data() + o_init + 2 * nn * sizeof(unsigned int), pending.data(), nn * sizeof(unsigned int));
  unsigned char *dp = nullptr;
  if (cudaMalloc(&dp, total) != cudaSuccess) return MB_ERR_NOMEM;
  cp.dev_allocs.push_back(dp);
  MB_CUDA(cudaMemcpy(dp, host.data(), total, cudaMemcpyHostToDevice));
  L.state = (unsigned int *)(dp + o_state);
  L.init = (const unsigned int *)(dp + o_init);
  L.state_bytes = st_bytes;
  PrgArgs &a = L.prg;
  a = PrgArgs{};
  a.nodes = (const PrgNode *)(dp + o_nodes);
  a.succ = (const int *)(dp + o_succ);
  a.blob = dp + o_blob;
  a.claim = L.state;
  a.done = L.state + nn;
  a.pending = L.state + 2 * nn;
  a.gen = L.state + 3 * nn;
  a.bulk_active = L.state + 3 * nn + 1;
  a.bulk_limit = c->prg_bulk_limit;
  a.err = c->d_prg_err;
  a.host_err = c->d_prg_err_host;
  a.nnodes = nn;
  a.nurgent = nurgent;
  a.timeout_ns = c->prg_timeout_ns;
  L.smem = program_smem(c->prec);
  int per_sm = 0;
  MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfunc<KPrg>(c->prec), PRG_THREADS, L.smem));
  if (per_sm < 1) return MB_ERR_UNSUPPORTED;
  if (ctas_per_sm > 0) per_sm = std::min(per_sm, ctas_per_sm);
  L.grid = (int)std::max<long long>(1, std::min<long long>((long long)per_sm * c->num_sms, items));
  return MB_OK;
}

// Lays the lowered nodes out as an executor program: nodes without work are
// dropped (their successors inherit their dependencies), urgent nodes come
// first and bulk (interior block-step) nodes after them, each class in plan
// order, which is a topological order.
int build_program(mb_ctx *c, CompiledPlan &cp) {
  const int nd = (int)cp.dn.size();
  std::vector<char> has_work(nd, 0);
  for (int q = 0; q < nd; q++) {
    int kind = 0, per = 1;
    long long units = 0;
    program_units(c, cp.dn[q], &kind, &units, &per);
    has_work[q] = units > 0;
  }
  const std::vector<std::vector<int>> eff = effective_deps(cp, has_work);
  std::vector<int> order;
  for (int pass = 0; pass < 2; pass++)
    for (int q = 0; q < nd; q++)
      if (has_work[q] && cp.dn[q].background == (pass == 1)) order.push_back(q);
  int nurgent = 0;
  for (int q : order) nurgent += cp.dn[q].background ? 0 : 1;
  if (int e = program_from(c, cp, order, eff, nurgent, 0, cp.prgm)) return e;
  cp.prg_built = true;
  return MB_OK;
}

// Graph mode 4: the bulk nodes (interiors of split levels) and the nodes the
// executor does not run (drag, L2, same-level pulls) stay graph kernel nodes;
// the other nodes of the fine levels' chain run as executor programs, one
// per segment: the chain nodes with the same number of bulk nodes on their
// longest path from the plan's start.  A segment's program is one graph
// node (after a copy that resets its state) that waits for every node its
// members wait for outside it; inside, the executor orders its members by
// their dependencies.  Its grid is capped so that the bulk node beside it
// keeps most of every SM.
int build_hybrid(mb_ctx *c, CompiledPlan &cp) {
  const int nd = (int)cp.dn.size();
  std::vector<char> has_work(nd, 0), alone(nd, 0);
  for (int q = 0; q < nd; q++) {
    const DevPlanNode &d = cp.dn[q];
    alone[q] = d.background || (d.kind != NK_STB && d.kind != NK_REC && d.kind != NK_SPL);
    if (alone[q]) {
      has_work[q] = d.grid.x > 0;
    } else {
      int kind = 0, per = 1;
      long long units = 0;
      program_units(c, d, &kind, &units, &per);
      has_work[q] = units > 0;
    }
  }
  const std::vector<std::vector<int>> eff = effective_deps(cp, has_work);
  std::vector<int> rank(nd, 0);
  int maxr = 0;
  for (int q = 0; q < nd; q++) {
    for (int p : eff[q]) rank[q] = std::max(rank[q], rank[p] + (alone[p] ? 1 : 0));
    maxr = std::max(maxr, rank[q]);
  }
  std::vector<std::vector<int>> seg(maxr + 1), solo(maxr + 1);
  for (int q = 0; q < nd; q++) {
    if (!has_work[q]) continue;
    (alone[q] ? solo : seg)[rank[q]].push_back(q);
  }
  MB_CUDA(cudaGraphCreate(&cp.graph, 0));
  std::vector<cudaGraphNode_t> gnode(nd, nullptr);  // graph node each plan node completes in
  cp.segs.assign(maxr + 1, PrgLaunch{});
  for (int r = 0; r <= maxr; r++) {
    if (!seg[r].empty()) {
      PrgLaunch &L = cp.segs[r];
      if (int e = program_from(c, cp, seg[r], eff, (int)seg[r].size(), c->hyb_ctas_per_sm, L)) return e;
      std::vector<cudaGraphNode_t> deps;
      for (int q : seg[r])
        for (int p : eff[q])
          if (rank[p] != r || alone[p]) deps.push_back(gnode[p]);
      std::sort(deps.begin(), deps.end());
      deps.erase(std::unique(deps.begin(), deps.end()), deps.end());
      cudaGraphNode_t cpy = nullptr, run = nullptr;
      MB_CUDA(cudaGraphAddMemcpyNode1D(&cpy, cp.graph, deps.data(), deps.size(), L.state, L.init, L.state_bytes,
                                       cudaMemcpyDeviceToDevice));
      cudaKernelNodeParams kp{};
      kp.func = kfunc<KPrg>(c->prec);
      kp.gridDim = dim3(L.grid);
      kp.blockDim = dim3(PRG_THREADS);
      kp.sharedMemBytes = (unsigned)L.smem;
      void *args[1] = {&L.prg};
      kp.kernelParams = args;
      MB_CUDA(cudaGraphAddKernelNode(&run, cp.graph, &cpy, 1, &kp));
      if (int e = set_priority(run, false)) return e;
      for (int q : seg[r]) gnode[q] = run;
    }
    for (int q : solo[r]) {
      DevPlanNode &d = cp.dn[q];
      std::vector<cudaGraphNode_t> deps;
      for (int p : eff[q]) deps.push_back(gnode[p]);
      std::sort(deps.begin(), deps.end());
      deps.erase(std::unique(deps.begin(), deps.end()), deps.end());
      cudaKernelNodeParams kp{};
      kp.func = d.func;
      kp.gridDim = d.grid;
      kp.blockDim = d.block;
      kp.sharedMemBytes = (unsigned)d.smem;
      kp.kernelParams = d.args;
      MB_CUDA(cudaGraphAddKernelNode(&gnode[q], cp.graph, deps.data(), deps.size(), &kp));
      if (int e = set_priority(gnode[q], d.background)) return e;
    }
  }
  MB_CUDA(cudaGraphInstantiateWithFlags(&cp.exec, cp.graph, cudaGraphInstantiateFlagUseNodePriority));
  cp.kernels = 0;
  for (int r = 0; r <= maxr; r++) cp.kernels += (seg[r].empty() ? 0 : 1) + (long long)solo[r].size();
  cp.prg_built = true;
  return MB_OK;
}

int launch_program(mb_ctx *c, CompiledPlan &cp, cudaStream_t s) {
  PrgLaunch &L = cp.prgm;
  if (L.prg.nnodes == 0) return MB_OK;
  L.prg.timeout_ns = c->prg_timeout_ns;
  L.prg.trace = c->d_trace;
  L.prg.trace_n = c->d_trace_n;
  L.prg.trace_cap = c->trace_cap;
  L.prg.launch = c->prg_launches++;
  L.prg.bulk_limit = c->prg_bulk_limit;
  MB_CUDA(cudaMemcpyAsync(L.state, L.init, L.state_bytes, cudaMemcpyDeviceToDevice, s));
  void *args[1] = {&L.prg};
  void *fn = c->d_trace ? kfunc<KPrgT>(c->prec) : kfunc<KPrg>(c->prec);
  MB_CUDA(cudaLaunchKernel(fn, dim3(L.grid), dim3(PRG_THREADS), args, L.smem, s));
  return MB_OK;
}

// error word of the persistent executor: MB_ERR_TIMEOUT once after a launch
// gave up waiting (valid after the launch's stream has been synchronised)
int program_status(mb_ctx *c) {
  if (!c->h_prg_err || *(volatile unsigned int *)c->h_prg_err == 0u) return MB_OK;
  *(volatile unsigned int *)c->h_prg_err = 0u;
  cudaMemset(c->d_prg_err, 0, sizeof(unsigned int));
  return MB_ERR_TIMEOUT;
}

// Levels whose block-step kernel computes CF_FCSRC cells with the per-cell
// code that k_fc_pull runs (every kernel but the two-cell one, variant 2), so
// that an NK_FCP node gives bitwise the step's values.  In unshifted FP32
// storage the per-cell code compiled into k_fc_pull rounds a few values
// differently from the block-step kernels' copy: no level there.
unsigned fc_levels(const mb_ctx *c) {
  if (c->prec == MB_PREC_F32U) return 0;
  unsigned m = 0;
  for (int l = 0; l < MB_MAX_LEVEL; l++)
    if (c->stb_variant[l] != 2) m |= 1u << l;
  return m;
}

CompiledPlan *get_plan(mb_ctx *c, int n, bool final_macros, int *err, bool batch = false) {
  // batches and the persistent executor run the plain node kinds only
  // batches and the executor run the plain node kinds only
  const bool fuse = c->fuse_cc && !options_on(c) && !batch && c->use_graph < 3;
  const bool early = c->fuse_early && !options_on(c) && !batch && c->use_graph < 3;
  const bool ffc = c->fuse_fc && !options_on(c) && !batch && c->use_graph < 3;
  std::string key = c->state.key() + "/" + std::to_string(n) + (final_macros ? "F" : "P") + (fuse ? "c" : "") +
                    (c->fuse_tmp ? "t" : "") + (early ? "e" : "") + (ffc ? "f" : "") +
                    (c->split_waits ? "w" : "");
  auto it = c->plans.find(key);
  if (it != c->plans.end()) return it->second.get();
  auto cp = std::make_unique<CompiledPlan>();
  PlanCompiler pc(c->geo, c->bl, c->hflags, c->spl_lines);
  pc.split_cells = c->split_cells;
  pc.split_mask = c->split_mask;
  if (fuse) pc.cc = &c->cc;
  pc.fuse_tmp = c->fuse_tmp != 0;
  if (early) pc.early_levels = c->early_levels;
  pc.fuse_fc = ffc;
  pc.fc_levels = fc_levels(c);
  pc.split_waits = c->split_waits != 0;
  SchedState s = c->state;
  cp->nodes = pc.compile(s, n, final_macros);
  cp->end = s;
  *err = lower_plan(c, *cp);
  if (*err) return nullptr;
  CompiledPlan *raw = cp.get();
  c->plans[key] = std::move(cp);
  return raw;
}

// n coarse steps of the reference's main loop (a step, getDrag_block and
// error_L2 each step) as one plan: the drag and the L2 change of a step run
// beside the rest of the plan where their reads and writes allow.
CompiledPlan *get_diag_plan(mb_ctx *c, int n, int *err) {
  const bool fuse = c->fuse_cc && !options_on(c) && c->use_graph < 3;
  const bool early = c->fuse_early && !options_on(c) && c->use_graph < 3;
  const bool ffc = c->fuse_fc && !options_on(c) && c->use_graph < 3;
  const std::string key = c->state.key() + "/" + std::to_string(n) + "D" + (fuse ? "c" : "") +
                          (c->fuse_tmp ? "t" : "") + (early ? "e" : "") + (ffc ? "f" : "") +
                    (c->split_waits ? "w" : "");
  auto it = c->plans.find(key);
  if (it != c->plans.end()) return it->second.get();
  auto cp = std::make_unique<CompiledPlan>();
  PlanCompiler pc(c->geo, c->bl, c->hflags, c->spl_lines);
  pc.split_cells = c->split_cells;
  pc.split_mask = c->split_mask;
  pc.drag_area = c->drag_area;
  if (fuse) pc.cc = &c->cc;
  pc.fuse_tmp = c->fuse_tmp != 0;
  if (early) pc.early_levels = c->early_levels;
  pc.fuse_fc = ffc;
  pc.fc_levels = fc_levels(c);
  pc.split_waits = c->split_waits != 0;
  SchedState s = c->state;
  cp->nodes = pc.compile_diag(s, n);
  cp->end = s;
  *err = lower_plan(c, *cp);
  if (*err) return nullptr;
  CompiledPlan *raw = cp.get();
  c->plans[key] = std::move(cp);
  return raw;
}

// Coarse steps of the next plan a call of `remaining` more steps replays, and
// whether it is the call's last (rho/u of every cell written in its last
// step).  Graphs and direct launches take plans of a whole number of
// scheduler periods, at least plan_steps long, so that one compiled plan
// serves every repetition and the next step's level-0 interior overlaps the
// chain everywhere except across the few graph boundaries; the call's tail
// is one plan of the remaining steps.  The executor keeps its launches of
// prg_periods periods and single final-state steps.  Diagnostic plans write
// rho/u every step, so they have no final flag.
int next_chunk(const mb_ctx *c, int remaining, bool diag, bool *fin) {
  if (c->use_graph == 3) {
    const int G = c->period * c->prg_periods;
    *fin = diag || remaining == 1;
    if (diag) return 1;
    return remaining - 1 >= G ? G : 1;
  }
  const int per = std::max(c->period, 1);
  const int G = (std::max(c->plan_steps, 1) + per - 1) / per * per;
  if (diag) {
    *fin = true;
    return std::min(remaining, G);
  }
  if (remaining > G) {
    *fin = false;
    return G;
  }
  *fin = true;
  return remaining;
}

int exec_plan(mb_ctx *c, CompiledPlan *cp, cudaStream_t s) {
  int e;
  if (c->use_graph == 3) {
    if (options_on(c)) return MB_ERR_UNSUPPORTED;  // the executor runs the BGK/SBB step only
    if (!cp->prg_built && (e = build_program(c, *cp))) return e;
    if ((e = launch_program(c, *cp, s))) return e;
    c->state = cp->end;
    c->kernels_last_call += 1;
    return MB_OK;
  }
  if (c->use_graph == 4 && options_on(c)) return MB_ERR_UNSUPPORTED;
  if (c->use_graph) {
    if (!cp->exec) {
      cudaAccessPolicyWindow w{};
      e = c->use_graph == 4 ? build_hybrid(c, *cp) : build_graph(*cp, c->use_graph == 2, l2_window(c, &w) ? &w : nullptr);
      if (e) return e;
    }
    MB_CUDA(cudaGraphLaunch(cp->exec, s));
  } else {
    e = run_direct(*cp, s);
    if (e) return e;
  }
  c->state = cp->end;
  c->kernels_last_call += cp->kernels;
  return MB_OK;
}

int exec_nodes_once(mb_ctx *c, std::vector<PlanNode> nodes, cudaStream_t s) {
  CompiledPlan cp;
  cp.nodes = std::move(nodes);
  int e = lower_plan(c, cp);
  if (e) return e;
  e = run_direct(cp, s);
  if (e) return e;
  // the temporary device buffers are freed by ~CompiledPlan after the work completes
  MB_CUDA(cudaStreamSynchronize(s));
  return MB_OK;
}

}  // namespace

// =============================================================================
// C ABI
// =============================================================================
extern "C" int mb_create(const mb_geometry *geo, int precision, mb_ctx **out) {
  if (!geo || !out) return MB_ERR_INVALID;
  *out = nullptr;
  if (precision != MB_PREC_F64 && precision != MB_PREC_F32 && precision != MB_PREC_F16S && precision != MB_PREC_F32U &&
      precision != MB_PREC_F16C)
    return MB_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return MB_ERR_NODEVICE;
  auto c = std::make_unique<mb_ctx>();
  c->prec = precision;
  // measured on config 2: overlapping the split coarse interior with the
  // fine levels gains 5% (FP32) and 13% (FP16 storage) per step once the
  // spline launches spread over the SMs (mb_set_cta_spread); FP64 unmeasured
  c->split_cells = precision == MB_PREC_F64 ? (1LL << 62) : 1000000;
  // measured per coarse step of the 3-level cylinder: FP16 storage steps
  // cell pairs on every level, whose shared addresses and paired accesses
  // cut its issue-bound instruction count (85.4 against 86.7 us with cell
  // ranges on level 0 and one cell per thread elsewhere; level 0 alone 39.7
  // against 46.0 us); FP32 storage steps level 0 in cell pairs too (104.3
  // against 109.9 us per step with quads; level 0 alone 52.8 against 61.0 us)
  if (precision == MB_PREC_F16S || precision == MB_PREC_F16C)
    for (int l = 0; l < MB_MAX_LEVEL; l++) c->stb_variant[l] = 4;
  if (precision == MB_PREC_F32 || precision == MB_PREC_F32U) c->stb_variant[0] = 4;
  // measured on config 2 (sweeps of both): the interior CTAs reserve shared
  // memory they do not use, so an SM holds three of them (cell pairs, 60 KB)
  // and keeps room for the fine levels' chain, and the splines ask for
  // 48 / 64 KB: FP32 104.3 against 111.2 us per step without the reserve
  // and 115.8 with two CTAs per SM; FP16 storage 84.4 against 85.5
  if (precision == MB_PREC_F32 || precision == MB_PREC_F32U) {
    c->bulk_cta_smem = 60 * 1024;
    c->spl_cta_smem = 48 * 1024;
  } else if (precision == MB_PREC_F16S || precision == MB_PREC_F16C) {
    c->bulk_cta_smem = 60 * 1024;
    c->spl_cta_smem = 64 * 1024;
  }
  cudaGetDevice(&c->device);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  c->geo = *geo;
  const mb_layout &L = geo->layout;
  const mb_config &cfg = geo->config;
  c->nblk = L.number_area;
  if (c->nblk < 1 || c->nblk > MB_MAX_AREA) return MB_ERR_INVALID;
  if (c->nblk > REC_MAX_BLOCKS) return MB_ERR_UNSUPPORTED;
  const size_t sb = prec_bytes(precision), rb = real_bytes(precision);
  const int pitch_align = (int)(128 / sb);

  // feq(rho0, U0): init_General state and the block-edge equilibrium
  for (int k = 0; k < 9; k++) {
    const double eu = ex(k) * cfg.U0[0] + ey(k) * cfg.U0[1];
    const double uv = cfg.U0[0] * cfg.U0[0] + cfg.U0[1] * cfg.U0[1];
    c->feqc[k] = wd(k) * cfg.rho0 * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uv);
  }
  c->shift_mode = default_shift(precision);
  c->shift = make_shift(c.get(), c->shift_mode);
  // measured on config 2's developed shedding against FP64 storage (mean Cd,
  // rms Cl, St): stochastic rounding +9e-5, -4.6e-3, -6.9e-4 in FP16 storage
  // (round to nearest -8.7e-3, -0.36, -7.1e-2) for 4 % more time per step;
  // h16c -5.3e-4, -4.2e-3, -5.1e-4 (round to nearest -6.2e-3, -8.9e-2, -2.6e-3)
  c->shift.sr = precision == MB_PREC_F16C || precision == MB_PREC_F16S ? MB_ROUND_STOCHASTIC : MB_ROUND_NEAREST;

  // block layouts and flags
  c->bl.resize(c->nblk);
  c->hflags.resize(c->nblk);
  for (int a = 0; a < c->nblk; a++) {
    const mb_area &A = geo->Areas[a];
    BlockLayout &b = c->bl[a];
    b.nx = A.nx;
    b.ny = A.ny;
    if ((long long)A.nx * A.ny > (1LL << 31) / 2) return MB_ERR_UNSUPPORTED;
    b.pitch = (A.nx + pitch_align - 1) / pitch_align * pitch_align;
    const long long pe = (long long)b.pitch * b.ny;
    b.plane = (pe + 127) / 128 * 128;
    auto &fl = c->hflags[a];
    fl.assign((size_t)b.plane, CT_PAD);
    for (int j = 0; j < A.ny; j++)
      for (int i = 0; i < A.nx; i++) {
        const int t = cell_type(*geo, a, i, j);
        uint8_t v = t == MB_FLUID ? CT_FLUID : (t == MB_SOLID_SBB ? CT_SOLID : CT_COPY);
        if (i == 0 || j == 0 || i == A.nx - 1 || j == A.ny - 1) v |= CF_EDGE;
        fl[(size_t)j * b.pitch + i] = v;
      }
  }
  mark_macro_sources(*geo, c->bl, c->hflags);
  mark_fc_sources(*geo, c->bl, c->hflags);
  // same-level copies the block step of their level can perform: flag the
  // targets and keep, per target cell, where its source is
  c->cc = cc_levels(*geo, c->bl, c->hflags);
  for (CcLevel &cl : c->cc) {
    if (!cl.fusable) continue;
    for (const CcLink &lk : cl.links)
      if (lk.tcell >= (1LL << 31) || lk.scell >= (1LL << 31)) cl.fusable = false;  // 32-bit cells in CcEntry
    if (!cl.fusable) continue;
    for (const CcLink &lk : cl.links) c->hflags[lk.tblk][(size_t)lk.tcell] |= CF_CCPULL;
  }

  // coarse-fine line table for the spline kernel; slots: 3 x 9 values per fine point
  c->spl_lines.resize(L.number_line);
  long long slot_pts = 0;
  for (int b = 0; b < L.number_line; b++) {
    const mb_line &l = geo->Line_Inf_C[b];
    SplLine &s = c->spl_lines[b];
    s.coarse = l.areac_n;
    s.fine = l.areaf_n;
    s.Nc = l.Nc;
    s.Nf = l.Nf;
    const mb_area &ac = geo->Areas[l.areac_n], &af = geo->Areas[l.areaf_n];
    s.r = af.m / ac.m;
    const bool vc = l.line_C.xstart == l.line_C.xend, vf = l.line_F.xstart == l.line_F.xend;
    s.ci0 = l.line_C.xstart; s.cj0 = l.line_C.ystart; s.cdi = vc ? 0 : 1; s.cdj = vc ? 1 : 0;
    s.fi0 = l.line_F.xstart; s.fj0 = l.line_F.ystart; s.fdi = vf ? 0 : 1; s.fdj = vf ? 1 : 0;
    s.slot0 = (int)slot_pts;
    s.para = (af.tau - 1.0) / (s.r * (ac.tau - 1.0));
    if (l.Nc < 2 || l.Nf < 1 || s.r < 1) return MB_ERR_GEOMETRY;
    if ((long long)(l.Nf - 1) > (long long)s.r * (l.Nc - 1)) return MB_ERR_GEOMETRY;
    slot_pts += l.Nf;
  }
  c->n_slot_points = slot_pts;

  // fine levels without same-level copies, whose splines can do the next
  // temporal interpolation in place: CF_TSKIP on the edge cells it writes
  for (int l = 1; l < L.LEVEL; l++) {
    if (L.LCCP[l] != L.LCCP[l + 1] || L.LTCFFCP[l] == L.LTCFFCP[l + 1]) continue;
    bool ok = true;
    for (int b = L.LTCFFCP[l]; b < L.LTCFFCP[l + 1] && ok; b++) {
      const int a = geo->Line_Inf_C[b].areaf_n;
      ok = a >= L.ASP[l] && a < L.ASP[l + 1];
      const SplLine &sl = c->spl_lines[b];
      for (int ip = 0; ok && ip < sl.Nf; ip++) {
        const int i = sl.fi0 + ip * sl.fdi, j = sl.fj0 + ip * sl.fdj;
        ok = (c->hflags[a][(size_t)j * c->bl[a].pitch + i] & 3) == CT_COPY;
      }
    }
    if (!ok) continue;
    c->early_levels |= 1u << l;
    for (int b = L.LTCFFCP[l]; b < L.LTCFFCP[l + 1]; b++) {
      const int a = geo->Line_Inf_C[b].areaf_n;
      const SplLine &sl = c->spl_lines[b];
      for (int ip = 0; ip < sl.Nf; ip++)
        c->hflags[a][(size_t)(sl.fj0 + ip * sl.fdj) * c->bl[a].pitch + (sl.fi0 + ip * sl.fdi)] |= CF_TSKIP;
    }
  }

  // device allocations (Multi-block-LBM.cu:26-113, without x/y/force/f arrays).
  // F and rho/u of the fine blocks (m > 1) and the interface slots are carved
  // from one arena, the range an L2 access-policy window can keep resident.
  int e;
  auto a256 = [](size_t n) { return (std::max<size_t>(n, 1) + 255) & ~(size_t)255; };
  const size_t slot_bytes = (size_t)std::max<long long>(slot_pts, 1) * 27 * rb;
  size_t fine = a256(slot_bytes);
  for (int a = 0; a < c->nblk; a++)
    if (geo->Areas[a].m > 1) fine += 2 * a256((size_t)9 * c->bl[a].plane * sb) + 3 * a256((size_t)c->bl[a].plane * rb);
  {
    void *p;
    if (cudaMalloc(&p, fine) != cudaSuccess) return MB_ERR_NOMEM;
    c->allocs.push_back(p);
    c->fine_arena = p;
    c->fine_bytes = fine;
  }
  size_t fine_off = 0;
  auto take = [&](size_t n) {
    void *p = (char *)c->fine_arena + fine_off;
    fine_off += a256(n);
    return p;
  };
  c->d_slots = take(slot_bytes);
  c->blk.resize(c->nblk);
  for (int a = 0; a < c->nblk; a++) {
    IfBlk &B = c->blk[a];
    const BlockLayout &b = c->bl[a];
    const bool in_arena = geo->Areas[a].m > 1;
    for (int q = 0; q < 2; q++) {
      void *p;
      if (in_arena) {
        p = take((size_t)9 * b.plane * sb);
      } else {
        if (cudaMalloc(&p, (size_t)9 * b.plane * sb) != cudaSuccess) return MB_ERR_NOMEM;
        c->allocs.push_back(p);
      }
      B.F[q] = p;
    }
    void *m[5];
    for (int q = 0; q < 5; q++) {
      if (in_arena && q < 3) {
        m[q] = take((size_t)b.plane * rb);
        continue;
      }
      if (cudaMalloc(&m[q], (size_t)b.plane * rb) != cudaSuccess) return MB_ERR_NOMEM;
      c->allocs.push_back(m[q]);
    }
    B.rho = m[0]; B.ux = m[1]; B.uy = m[2]; B.upx = m[3]; B.upy = m[4];
    uint8_t *fl;
    if ((e = dalloc(c.get(), &fl, (size_t)b.plane))) return e;
    MB_CUDA(cudaMemcpy(fl, c->hflags[a].data(), (size_t)b.plane, cudaMemcpyHostToDevice));
    B.flags = fl;
    B.nx = b.nx; B.ny = b.ny; B.pitch = b.pitch; B.m = geo->Areas[a].m;
    B.plane = b.plane;
    B.tau = geo->Areas[a].tau;
  }
  if ((e = dalloc(c.get(), &c->d_blk, c->nblk))) return e;
  MB_CUDA(cudaMemcpy(c->d_blk, c->blk.data(), c->nblk * sizeof(IfBlk), cudaMemcpyHostToDevice));
  c->d_cclist.assign(L.LEVEL, nullptr);
  for (int l = 0; l < L.LEVEL; l++) {
    const CcLevel &cl = c->cc[l];
    if (!cl.fusable) continue;
    std::vector<CcEntry> ents;
    for (const CcLink &lk : cl.links) {
      const int sp = c->bl[lk.sblk].pitch;
      ents.push_back({lk.tblk, lk.sblk, (int)lk.tcell, (int)(lk.scell % sp), (int)(lk.scell / sp), 0});
    }
    if ((e = dalloc(c.get(), &c->d_cclist[l], ents.size()))) return e;
    MB_CUDA(cudaMemcpy(c->d_cclist[l], ents.data(), ents.size() * sizeof(CcEntry), cudaMemcpyHostToDevice));
  }
  if (L.number_line) {
    // LU coefficients of each line's system (init_tri_A rows): c'_i = u_i / den_i,
    // den_i = 2 - l_i c'_{i-1}; stored as c' then 1/den, in the arithmetic type
    std::vector<double> coef;
    c->spl_coef0.resize(L.number_line);
    for (int b = 0; b < L.number_line; b++) {
      const SplLine &s = c->spl_lines[b];
      const int N = s.Nc;
      c->spl_coef0[b] = (int)(coef.size() / 2);
      std::vector<double> cp(N), iv(N);
      double prev = 0;
      for (int i = 0; i < N; i++) {
        const double l = (i <= 1 || i == N - 1) ? 0.0 : 0.5, u = (i == 0 || i >= N - 2) ? 0.0 : 0.5;
        const double den = 2.0 - l * prev;
        cp[i] = u / den;
        iv[i] = 1.0 / den;
        prev = cp[i];
      }
      coef.insert(coef.end(), cp.begin(), cp.end());
      coef.insert(coef.end(), iv.begin(), iv.end());
    }
    const size_t rb = real_bytes(precision);
    std::vector<unsigned char> raw(coef.size() * rb);
    for (size_t q = 0; q < coef.size(); q++) {
      if (rb == 8) std::memcpy(&raw[q * 8], &coef[q], 8);
      else { const float fv = (float)coef[q]; std::memcpy(&raw[q * 4], &fv, 4); }
    }
    void *pc;
    if (cudaMalloc(&pc, raw.size()) != cudaSuccess) return MB_ERR_NOMEM;
    c->allocs.push_back(pc);
    c->d_spl_coef = pc;
    MB_CUDA(cudaMemcpy(pc, raw.data(), raw.size(), cudaMemcpyHostToDevice));
  }

  // drag links (fdrag_store, force_block.h:78-127): i-outer, j-inner, k
  c->drag_area = cfg.drag_area < 0 ? c->nblk - 1 : cfg.drag_area;
  if (c->drag_area >= c->nblk) return MB_ERR_INVALID;
  if ((e = upload_drag_links(c.get()))) return e;
  if ((e = dalloc(c.get(), &c->d_drag_out, 2))) return e;
  MB_CUDA(cudaMallocHost(&c->h_drag_out, 2 * sizeof(double)));

  // L2 tables and scratch
  {  // tiles of 256 cells of one row: at most ceil(nx / 256) + 2 per row over both parts
    long long cell = 0, tiles = 0;
    for (int a = 0; a < c->nblk; a++) {
      tiles += (long long)((c->bl[a].nx + 255) / 256 + 2) * c->bl[a].ny;
      cell += (long long)c->bl[a].nx * c->bl[a].ny;
    }
    if (tiles >= (1LL << 31)) return MB_ERR_UNSUPPORTED;
    c->total_cells = cell;
    c->l2_tiles = (int)tiles;
    c->l2_grid = (int)std::min<long long>(tiles, 148LL * 8);
    for (int q = 0; q < L2_NPARTS; q++) {
      if ((e = dalloc(c.get(), &c->d_l2_partial[q], c->l2_grid))) return e;
      if ((e = dalloc(c.get(), &c->d_l2_ticket[q], 1))) return e;
      MB_CUDA(cudaMemset(c->d_l2_ticket[q], 0, sizeof(unsigned int)));
    }
    if ((e = dalloc(c.get(), &c->d_l2_out, 2 * L2_NPARTS))) return e;
    MB_CUDA(cudaMallocHost(&c->h_l2_out, 2 * L2_NPARTS * sizeof(double)));
  }
  if ((e = dalloc(c.get(), &c->d_count, 1))) return e;

  // scheduler state (Multi-block-LBM.cu:45-47 markers)
  c->state.parity.assign(c->nblk, 0);
  c->state.marker.assign(L.number_line, {2, 1, 0});
  {
    // period of the (parity, marker) state over coarse steps
    PlanCompiler pc(c->geo, c->bl, c->hflags, c->spl_lines);
    SchedState s = c->state;
    int per = 0;
    for (int n = 1; n <= 12; n++) {
      SchedState t = s;
      (void)pc;
      // advance symbolically by one coarse step without building nodes
      for (int l = 0; l < L.LEVEL; l++) {
        int steps = 1;
        for (int q = 1; q <= l; q++) steps *= L.mi[q];
        if (steps & 1)
          for (int a = L.ASP[l]; a < L.ASP[l + 1]; a++) t.parity[a] ^= 1;
        if (l != L.LEVEL - 1) {
          const int rot = steps % 3;
          for (int b = L.LS3CFFCP[l]; b < L.LS3CFFCP[l + 1]; b++)
            for (int r = 0; r < rot; r++)
              for (int p = 0; p < 3; p++) t.marker[b][p] = t.marker[b][p] == 0 ? 2 : t.marker[b][p] - 1;
        }
      }
      s = t;
      if (s == c->state) { per = n; break; }
    }
    c->period = per > 0 ? per : 6;
  }
  {
    long long upd = 0;
    for (int l = 0; l < L.LEVEL; l++) {
      long long steps = 1;
      for (int q = 1; q <= l; q++) steps *= L.mi[q];
      for (int a = L.ASP[l]; a < L.ASP[l + 1]; a++) upd += steps * (long long)c->bl[a].nx * c->bl[a].ny;
    }
    c->updates_per_step = upd;
  }
  // error word of the persistent executor, mirrored into mapped host memory
  if ((e = dalloc(c.get(), &c->d_prg_err, 1))) return e;
  MB_CUDA(cudaMemset(c->d_prg_err, 0, sizeof(unsigned int)));
  MB_CUDA(cudaHostAlloc(&c->h_prg_err, sizeof(unsigned int), cudaHostAllocMapped));
  *c->h_prg_err = 0u;
  MB_CUDA(cudaHostGetDevicePointer((void **)&c->d_prg_err_host, c->h_prg_err, 0));
  if ((e = set_smem_limits(precision))) return e;
  *out = c.release();
  return MB_OK;
}

extern "C" int mb_destroy(mb_ctx *c) {
  if (!c) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->plans.clear();
  if (c->l2_persist) {  // the set-aside goes back to normal lines
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
  }
  for (void *p : c->allocs) cudaFree(p);
  if (c->h_drag_out) cudaFreeHost(c->h_drag_out);
  if (c->h_l2_out) cudaFreeHost(c->h_l2_out);
  if (c->h_prg_err) cudaFreeHost(c->h_prg_err);
  if (c->d_diag) cudaFree(c->d_diag);
  if (c->h_diag) cudaFreeHost(c->h_diag);
  if (c->d_trace) cudaFree(c->d_trace);
  if (c->d_trace_n) cudaFree(c->d_trace_n);
  delete c;
  return MB_OK;
}

extern "C" int mb_set_split_cells(mb_ctx *c, long long cells) {
  if (!c || cells < 0) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->split_cells = cells;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_shift(mb_ctx *c, int mode) {
  if (!c || (mode != MB_SHIFT_W && mode != MB_SHIFT_FEQ0)) return MB_ERR_INVALID;
  if (mode == c->shift_mode) return MB_OK;
  cudaDeviceSynchronize();
  c->plans.clear();
  c->shift_mode = mode;
  const int sr = c->shift.sr;
  c->shift = make_shift(c, mode);
  c->shift.sr = sr;
  c->inited = false;  // the stored words mean something else now: mb_init (or a restore) comes next
  return MB_OK;
}

extern "C" int mb_set_rounding(mb_ctx *c, int mode) {
  if (!c || (mode != MB_ROUND_NEAREST && mode != MB_ROUND_STOCHASTIC)) return MB_ERR_INVALID;
  if (mode == MB_ROUND_STOCHASTIC && c->prec != MB_PREC_F16C && c->prec != MB_PREC_F16S) return MB_ERR_INVALID;
  if (mode == c->shift.sr) return MB_OK;
  cudaDeviceSynchronize();
  c->plans.clear();  // the kernels read the mode from their parameters
  c->shift.sr = mode;
  return MB_OK;
}

extern "C" int mb_set_l2_persist(mb_ctx *c, int mb) {
  if (!c || mb < 0) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->plans.clear();
  int dev = 0, maxp = 0;
  MB_CUDA(cudaGetDevice(&dev));
  MB_CUDA(cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, dev));
  const size_t want = std::min(std::min((size_t)mb << 20, (size_t)std::max(maxp, 0)), c->fine_bytes);
  MB_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
  if (!want) MB_CUDA(cudaCtxResetPersistingL2Cache());
  c->l2_persist = want;
  return MB_OK;
}

extern "C" int mb_set_hybrid_ctas(mb_ctx *c, int per_sm) {
  if (!c || per_sm < 1 || per_sm > 32) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->plans.clear();
  c->hyb_ctas_per_sm = per_sm;
  return MB_OK;
}

extern "C" int mb_set_plan_steps(mb_ctx *c, int n) {
  if (!c || n < 1 || n > 4096) return MB_ERR_INVALID;
  c->plan_steps = n;
  return MB_OK;
}

extern "C" int mb_set_bulk_spread(mb_ctx *c, int kb) {
  if (!c || kb < 0 || kb * 1024 > MB_CTA_SMEM_MAX) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->plans.clear();
  c->bulk_cta_smem = kb * 1024;
  return MB_OK;
}

extern "C" int mb_set_cta_spread(mb_ctx *c, int spline_kb, int records_kb) {
  if (!c || spline_kb < 0 || records_kb < 0 || spline_kb * 1024 > MB_CTA_SMEM_MAX || records_kb * 1024 > MB_CTA_SMEM_MAX)
    return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->spl_cta_smem = spline_kb * 1024;
  c->rec_cta_smem = records_kb * 1024;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_interface_shape(mb_ctx *c, int rec_points, int spline_segments) {
  if (!c || (rec_points != 32 && rec_points != 64) || spline_segments < 1 || spline_segments > SPL_WARPS)
    return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->rec_points = rec_points;
  c->spl_segs = spline_segments;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_split_levels(mb_ctx *c, unsigned level_mask) {
  if (!c || level_mask >= (1u << MB_MAX_LEVEL)) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->split_mask = level_mask;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_stream_cells(mb_ctx *c, long long cells, int bulk) {
  if (!c || cells < 0 || bulk < 0 || bulk > 1) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->stream_cells = cells;
  c->bulk_levels = bulk;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_stb_variant(mb_ctx *c, int level, int variant) {
  if (!c || level < 0 || level >= c->geo.layout.LEVEL || variant < 0 || variant > 6) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->stb_variant[level] = variant;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_collision(mb_ctx *c, int kind, double s_e, double s_eps, double s_q) {
  if (!c || (kind != MB_COLL_BGK && kind != MB_COLL_MRT) || !std::isfinite(s_e) || !std::isfinite(s_eps) ||
      !std::isfinite(s_q) || s_e >= 2.0 || s_eps >= 2.0 || s_q >= 2.0)
    return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->opt.coll = kind;
  c->opt.mrt_s[0] = s_e;
  c->opt.mrt_s[1] = s_eps;
  c->opt.mrt_s[2] = s_q;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_body_force(mb_ctx *c, double fx, double fy) {
  if (!c || !std::isfinite(fx) || !std::isfinite(fy)) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->opt.force[0] = fx;
  c->opt.force[1] = fy;
  c->opt.has_force = fx != 0.0 || fy != 0.0;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_cell_types(mb_ctx *c, int a, const int *types) {
  if (!c || a < 0 || a >= c->nblk || !types) return MB_ERR_INVALID;
  const BlockLayout &b = c->bl[a];
  auto movable = [](int t) { return t == MB_FLUID || t == MB_SOLID_SBB || t == MB_SOLID_SLIP || t == MB_SOLID_HBB; };
  std::vector<uint8_t> fl = c->hflags[a];
  long long alt_before = 0, alt_after = 0;
  for (int j = 0; j < b.ny; j++)
    for (int i = 0; i < b.nx; i++) {
      uint8_t &f = fl[(size_t)j * b.pitch + i];
      const int was = flag_code(f), t = types[(size_t)j * b.nx + i];
      if (movable(was) != movable(t) || (!movable(was) && t != was)) return MB_ERR_INVALID;
      if ((f & 3) == CT_SOLID && (f & (CF_HBB | CF_SLIP))) alt_before++;  // on FLUID cells bit 16 is CF_FCSRC
      if (!movable(t)) continue;
      f = uint8_t((f & ~(3 | CF_HBB | CF_SLIP)) | (t == MB_FLUID ? CT_FLUID : CT_SOLID) |
                  (t == MB_SOLID_HBB ? CF_HBB : 0) | (t == MB_SOLID_SLIP ? CF_SLIP : 0));
      if ((f & 3) == CT_SOLID && (f & (CF_HBB | CF_SLIP))) alt_after++;
    }
  cudaDeviceSynchronize();
  c->hflags[a] = fl;
  mark_fc_sources(c->geo, c->bl, c->hflags);  // f_c points of FLUID cells only
  fl = c->hflags[a];
  MB_CUDA(cudaMemcpy((void *)c->blk[a].flags, fl.data(), fl.size(), cudaMemcpyHostToDevice));
  c->n_alt_walls += alt_after - alt_before;
  int e;
  if (a == c->drag_area && (e = upload_drag_links(c))) return e;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_fusion(mb_ctx *c, int flags) {
  if (!c || flags < 0 || flags > 31) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->fuse_cc = flags & 1;
  c->fuse_tmp = (flags >> 1) & 1;
  c->fuse_early = (flags >> 2) & 1;
  c->fuse_fc = (flags >> 3) & 1;
  c->split_waits = (flags >> 4) & 1;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_bulk_occupancy(mb_ctx *c, int ctas_per_sm) {
  if (!c || ctas_per_sm < 0) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  c->bulk_ctas_per_sm = ctas_per_sm;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_program_timeout(mb_ctx *c, double seconds) {
  if (!c || !(seconds > 0) || seconds > 600) return MB_ERR_INVALID;
  c->prg_timeout_ns = (unsigned long long)(seconds * 1e9);
  return MB_OK;
}

extern "C" int mb_set_program_shape(mb_ctx *c, int bulk_cells, int urgent_cells, int periods_per_launch,
                                    int bulk_ctas) {
  if (!c || bulk_cells < 1 || urgent_cells < 1 || bulk_cells > (1 << 24) || urgent_cells > (1 << 24) ||
      periods_per_launch < 1 || periods_per_launch > 16 || bulk_ctas < 0)
    return MB_ERR_INVALID;
  c->prg_bulk_limit = bulk_ctas;
  cudaDeviceSynchronize();
  c->prg_bulk_cells = bulk_cells;
  c->prg_urgent_cells = urgent_cells;
  c->prg_periods = periods_per_launch;
  c->plans.clear();
  return MB_OK;
}

extern "C" int mb_set_program_trace(mb_ctx *c, long long capacity) {
  if (!c || capacity < 0 || capacity > (1LL << 26)) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  if (c->d_trace) cudaFree(c->d_trace);
  if (c->d_trace_n) cudaFree(c->d_trace_n);
  c->d_trace = nullptr;
  c->d_trace_n = nullptr;
  c->trace_cap = 0;
  if (capacity == 0) return MB_OK;
  if (cudaMalloc(&c->d_trace, (size_t)capacity * sizeof(PrgTraceRec)) != cudaSuccess) return MB_ERR_NOMEM;
  if (cudaMalloc(&c->d_trace_n, sizeof(unsigned int)) != cudaSuccess) return MB_ERR_NOMEM;
  MB_CUDA(cudaMemset(c->d_trace_n, 0, sizeof(unsigned int)));
  c->trace_cap = (unsigned int)capacity;
  return MB_OK;
}

extern "C" int mb_program_trace(mb_ctx *c, void *records, long long max_records, long long *n_records) {
  if (!c || !n_records || max_records < 0) return MB_ERR_INVALID;
  *n_records = 0;
  if (!c->d_trace) return MB_OK;
  MB_CUDA(cudaDeviceSynchronize());
  unsigned int n = 0;
  MB_CUDA(cudaMemcpy(&n, c->d_trace_n, sizeof(n), cudaMemcpyDeviceToHost));
  const long long have = std::min<long long>(n, c->trace_cap);
  const long long m = std::min<long long>(have, max_records);
  if (m > 0 && records) MB_CUDA(cudaMemcpy(records, c->d_trace, (size_t)m * sizeof(PrgTraceRec), cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemset(c->d_trace_n, 0, sizeof(unsigned int)));
  *n_records = m;
  return MB_OK;
}

extern "C" int mb_sync(mb_ctx *c, mb_stream stream) {
  if (!c) return MB_ERR_INVALID;
  MB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  return program_status(c);
}

// One executor launch over a single node with no work.  With stall = 1 the
// node starts with one unmet dependency that no node satisfies: every CTA
// waits out the executor timeout, sets the error word and exits.
extern "C" int mb_program_selftest(mb_ctx *c, int stall, mb_stream stream) {
  if (!c || stall < 0 || stall > 1) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  MB_CUDA(cudaStreamSynchronize(s));
  if (int st = program_status(c)) return st;
  PrgNode N{};
  N.kind = PK_NOP;
  N.items = 1;
  N.units = 1;
  N.per_item = 1;
  unsigned int st0[5] = {0u, 0u, (unsigned int)stall, 0u, 0u};
  unsigned char *dp = nullptr;
  if (cudaMalloc(&dp, 512) != cudaSuccess) return MB_ERR_NOMEM;
  int rc = MB_OK;
  do {
    if (cudaMemcpy(dp, &N, sizeof(N), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dp + 256, st0, sizeof(st0), cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = MB_ERR_CUDA;
      break;
    }
    PrgArgs a{};
    a.nodes = (const PrgNode *)dp;
    a.succ = (const int *)(dp + 128);
    a.blob = dp + 128;
    a.claim = (unsigned int *)(dp + 256);
    a.done = a.claim + 1;
    a.pending = a.claim + 2;
    a.gen = a.claim + 3;
    a.bulk_active = a.claim + 4;
    a.err = c->d_prg_err;
    a.host_err = c->d_prg_err_host;
    a.nnodes = 1;
    a.nurgent = 1;
    a.timeout_ns = c->prg_timeout_ns;
    void *args[1] = {&a};
    if (cudaLaunchKernel(kfunc<KPrg>(c->prec), dim3(2 * c->num_sms), dim3(PRG_THREADS), args, program_smem(c->prec), s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      rc = MB_ERR_CUDA;
      break;
    }
    unsigned int done = 0;
    if (cudaMemcpy(&done, a.done, sizeof(done), cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = MB_ERR_CUDA;
      break;
    }
    rc = program_status(c);
    if (rc == MB_OK && done != 1u) rc = MB_ERR_STATE;
  } while (0);
  cudaFree(dp);
  return rc;
}

extern "C" int mb_set_graph_mode(mb_ctx *c, int mode) {
  if (!c || mode < 0 || mode > 4) return MB_ERR_INVALID;
  if (mode != c->use_graph) {
    cudaDeviceSynchronize();
    c->plans.clear();
  }
  c->use_graph = mode;
  return MB_OK;
}

// init_General (lbm/init_block.h:2-51), init_Fstore and init_tri_A
// (multi/init_multi.h:3-51): uniform rho0/U0 with f = F = feq, u_prev = U0,
// every ring slot = the fine edge F (= feq), the spline matrix is implicit.
extern "C" int mb_init(mb_ctx *c, mb_stream stream) {
  if (!c) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  const mb_config &cfg = c->geo.config;
  const int th = 256;
  for (int a = 0; a < c->nblk; a++) {
    const IfBlk &B = c->blk[a];
    const long long n = B.plane;
    for (int q = 0; q < 2; q++) {
      const int gr = launch_grid(9 * n, th);
      const double *f = c->feqc;
      MB_DISPATCH(c->prec, (k_fill_planes<P><<<gr, th, 0, s>>>((S *)B.F[q], n, f[0], f[1], f[2], f[3], f[4], f[5],
                                                               f[6], f[7], f[8], c->shift.v)));
    }
    const int gr = launch_grid(n, th);
    if (c->prec == MB_PREC_F64) {
      k_fill<double><<<gr, th, 0, s>>>((double *)B.rho, n, cfg.rho0);
      k_fill<double><<<gr, th, 0, s>>>((double *)B.ux, n, cfg.U0[0]);
      k_fill<double><<<gr, th, 0, s>>>((double *)B.uy, n, cfg.U0[1]);
      k_fill<double><<<gr, th, 0, s>>>((double *)B.upx, n, cfg.U0[0]);
      k_fill<double><<<gr, th, 0, s>>>((double *)B.upy, n, cfg.U0[1]);
    } else {
      k_fill<float><<<gr, th, 0, s>>>((float *)B.rho, n, (float)cfg.rho0);
      k_fill<float><<<gr, th, 0, s>>>((float *)B.ux, n, (float)cfg.U0[0]);
      k_fill<float><<<gr, th, 0, s>>>((float *)B.uy, n, (float)cfg.U0[1]);
      k_fill<float><<<gr, th, 0, s>>>((float *)B.upx, n, (float)cfg.U0[0]);
      k_fill<float><<<gr, th, 0, s>>>((float *)B.upy, n, (float)cfg.U0[1]);
    }
  }
  if (c->n_slot_points > 0) {
    // slot layout [point][slot][k]: fill k-periodic values through a host pattern
    const long long n = c->n_slot_points * 27;
    const size_t rb = real_bytes(c->prec);
    std::vector<unsigned char> host((size_t)n * rb);
    for (long long q = 0; q < n; q++) {
      const double v = c->feqc[q % 9];
      if (rb == 8) std::memcpy(&host[q * 8], &v, 8);
      else { const float fv = (float)v; std::memcpy(&host[q * 4], &fv, 4); }
    }
    MB_CUDA(cudaMemcpyAsync(c->d_slots, host.data(), host.size(), cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaStreamSynchronize(s));
  }
  MB_CUDA(cudaGetLastError());
  c->state.parity.assign(c->nblk, 0);
  c->state.marker.assign(c->geo.layout.number_line, {2, 1, 0});
  c->inited = true;
  return MB_OK;
}

// After fields were set from outside (mb_set_fields), the state that the
// reference derives from the initial fields in init_Fstore and error_L2:
// ring slots of every coarse-fine line <- the fine edge F, u_prev <- u.
extern "C" int mb_sync_history(mb_ctx *c, mb_stream stream) {
  if (!c) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  for (const SplLine &L : c->spl_lines) {
    const IfBlk &B = c->blk[L.fine];
    const void *F = B.F[c->state.parity[L.fine]];
    MB_DISPATCH(c->prec, (k_slots_from_edge<P><<<(L.Nf + 127) / 128, 128, 0, s>>>(
                             (const S *)F, B.plane, L.fi0, L.fj0, L.fdi, L.fdj, B.pitch, L.Nf,
                             (typename Prec<P>::R *)c->d_slots, L.slot0, c->shift.v)));
  }
  const size_t rb = real_bytes(c->prec);
  for (int a = 0; a < c->nblk; a++) {
    const IfBlk &B = c->blk[a];
    MB_CUDA(cudaMemcpyAsync(B.upx, B.ux, (size_t)B.plane * rb, cudaMemcpyDeviceToDevice, s));
    MB_CUDA(cudaMemcpyAsync(B.upy, B.uy, (size_t)B.plane * rb, cudaMemcpyDeviceToDevice, s));
  }
  MB_CUDA(cudaStreamSynchronize(s));
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

extern "C" int mb_step(mb_ctx *c, int n, mb_stream stream) {
  if (!c || n < 0) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  c->kernels_last_call = 0;
  int remaining = n;
  while (remaining > 0) {
    bool fin;
    const int chunk = next_chunk(c, remaining, false, &fin);
    int err = 0;
    CompiledPlan *cp = get_plan(c, chunk, fin, &err);
    if (!cp) return err ? err : MB_ERR_INVALID;
    if ((err = exec_plan(c, cp, s))) return err;
    remaining -= chunk;
  }
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

namespace {
// Makes a compiled plan ready to replay: the executor program (mode 3) or the
// instantiated CUDA graph, uploaded on `up` so that its first launch pays no
// upload.  Direct launches (mode 0) need nothing.
int ready_plan(mb_ctx *c, CompiledPlan *cp, cudaStream_t up) {
  if (c->use_graph == 3) return cp->prg_built ? MB_OK : build_program(c, *cp);
  if (!c->use_graph || cp->exec) return MB_OK;
  if (c->use_graph == 4 && options_on(c)) return MB_ERR_UNSUPPORTED;
  cudaAccessPolicyWindow w{};
  if (int e = c->use_graph == 4 ? build_hybrid(c, *cp) : build_graph(*cp, c->use_graph == 2, l2_window(c, &w) ? &w : nullptr))
    return e;
  MB_CUDA(cudaGraphUpload(cp->exec, up));
  return MB_OK;
}

// Host side of mb_prepare / mb_prepare_diag: walks the chunks the step call
// will take from the current state (the scheduler state is restored after).
int prepare_chunks(mb_ctx *c, int n, bool diag) {
  cudaStream_t up = nullptr;
  MB_CUDA(cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking));
  const SchedState save = c->state;
  int remaining = n, err = MB_OK;
  while (remaining > 0 && err == MB_OK) {
    bool fin;
    const int chunk = next_chunk(c, remaining, diag, &fin);
    // mb_step_diag's plans carry their diagnostics; the executor's are
    // final-state steps with drag and L2 launched apart
    CompiledPlan *cp = diag && c->use_graph != 3 ? get_diag_plan(c, chunk, &err) : get_plan(c, chunk, fin, &err);
    if (!cp) { err = err ? err : MB_ERR_INVALID; break; }
    if ((err = ready_plan(c, cp, up))) break;
    c->state = cp->end;
    remaining -= chunk;
  }
  c->state = save;
  const cudaError_t se = cudaStreamSynchronize(up);
  cudaStreamDestroy(up);
  if (err) return err;
  return se == cudaSuccess ? MB_OK : MB_ERR_CUDA;
}

// Grows the per-step result buffers of mb_step_diag to n steps (device and
// pinned host memory); the stream drains first when they are replaced.
int ensure_diag(mb_ctx *c, size_t n, cudaStream_t s) {
  if (n <= c->diag_cap) return MB_OK;
  MB_CUDA(cudaStreamSynchronize(s));
  const size_t cap = std::max(n, 2 * c->diag_cap);
  if (c->d_diag) cudaFree(c->d_diag);
  if (c->h_diag) cudaFreeHost(c->h_diag);
  c->d_diag = nullptr;
  c->h_diag = nullptr;
  c->diag_cap = 0;
  if (cudaMalloc(&c->d_diag, cap * DIAG_STRIDE * sizeof(double)) != cudaSuccess) return MB_ERR_NOMEM;
  if (cudaMallocHost(&c->h_diag, cap * DIAG_STRIDE * sizeof(double)) != cudaSuccess) return MB_ERR_NOMEM;
  c->diag_cap = cap;
  return MB_OK;
}
}  // namespace

// Compiles (and instantiates and uploads as graphs) every plan mb_step(n) will
// replay from the current state, so that a later mb_step spends no host time
// on it.
extern "C" int mb_prepare(mb_ctx *c, int n) {
  if (!c || n < 0) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  return prepare_chunks(c, n, false);
}

// The same for mb_step_diag(n), which also gets its result buffers sized.
extern "C" int mb_prepare_diag(mb_ctx *c, int n) {
  if (!c || n < 0) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  if (int e = ensure_diag(c, (size_t)n, nullptr)) return e;
  return prepare_chunks(c, n, true);
}

// Text description of the plan mb_step(n) starts with from the current
// state: one line per lowered node (index, kind, level, region, grid, graph
// priority class, label, dependencies).  The plan is compiled if needed; the
// scheduler state is unchanged.
extern "C" int mb_plan_describe(mb_ctx *c, int n, char *buf, long long cap, long long *len) {
  if (!c || n < 1 || (!buf && cap > 0)) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  int err = 0;
  const SchedState save = c->state;
  bool fin;
  const int chunk = next_chunk(c, n, false, &fin);
  CompiledPlan *cp = get_plan(c, chunk, fin, &err);
  c->state = save;
  if (!cp) return err ? err : MB_ERR_INVALID;
  if (c->use_graph && c->use_graph != 3) mark_slack(*cp);
  std::string out;
  static const char *kinds[] = {"stb", "rec", "spl", "ccp", "fcp", "drag", "l2"};
  for (size_t q = 0; q < cp->dn.size(); q++) {
    const DevPlanNode &d = cp->dn[q];
    const PlanNode &nd = cp->nodes[q];
    char line[256];
    std::snprintf(line, sizeof line, "%zu %s L%d r%d grid %u %s %s deps", q,
                  (int)d.kind >= 0 && (int)d.kind < 7 ? kinds[(int)d.kind] : "?", nd.level, nd.region, d.grid.x,
                  d.background ? "bulk" : (d.slack ? "slack" : "chain"), nd.label.c_str());
    out += line;
    for (int p : d.deps) out += " " + std::to_string(p);
    if (d.kind == NK_FCP) out += " ; fc " + std::to_string(d.stb.fc_n);
    out += "\n";
  }
  if (len) *len = (long long)out.size();
  if (cap > 0) {
    const size_t m = std::min<size_t>(out.size(), (size_t)cap - 1);
    std::memcpy(buf, out.data(), m);
    buf[m] = 0;
  }
  return MB_OK;
}

extern "C" int mb_block_step(mb_ctx *c, int area, mb_stream stream) {
  if (!c || area < 0 || area >= c->nblk) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  PlanNode nd;
  nd.kind = NK_STB;
  nd.a0 = area;
  nd.a1 = area + 1;
  nd.macro_all = 1;
  for (int a = 0; a < c->nblk; a++)
    if (c->state.parity[a]) nd.parity |= 1ull << a;
  int e = exec_nodes_once(c, {nd}, (cudaStream_t)stream);
  if (e) return e;
  c->state.parity[area] ^= 1;
  return MB_OK;
}

static int single_op(mb_ctx *c, int kind, int index, double xm, mb_stream stream) {
  if (!c) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  PlanCompiler pc(c->geo, c->bl, c->hflags, c->spl_lines);
  return exec_nodes_once(c, pc.compile_single(kind, index, xm, c->state), (cudaStream_t)stream);
}

extern "C" int mb_c_c_boundary_transfer(mb_ctx *c, int line, mb_stream s) {
  if (!c || line < 0 || line >= c->geo.layout.number_line2) return MB_ERR_INVALID;
  return single_op(c, Op::CC, line, 0, s);
}
extern "C" int mb_space_interpolation(mb_ctx *c, int line, mb_stream s) {
  if (!c || line < 0 || line >= c->geo.layout.number_line) return MB_ERR_INVALID;
  return single_op(c, Op::SPL, line, 0, s);
}
extern "C" int mb_temporal_interpolation(mb_ctx *c, int line, double xm, mb_stream s) {
  if (!c || line < 0 || line >= c->geo.layout.number_line) return MB_ERR_INVALID;
  return single_op(c, Op::TEMPORAL, line, xm, s);
}
extern "C" int mb_c_f_boundary_transfer(mb_ctx *c, int line, mb_stream s) {
  if (!c || line < 0 || line >= c->geo.layout.number_line) return MB_ERR_INVALID;
  return single_op(c, Op::CF, line, 0, s);
}
extern "C" int mb_f_c_boundary_transfer(mb_ctx *c, int line, mb_stream s) {
  if (!c || line < 0 || line >= c->geo.layout.number_line) return MB_ERR_INVALID;
  return single_op(c, Op::FC, line, 0, s);
}
extern "C" int mb_rotate_markers(mb_ctx *c, int line) {
  if (!c || line < 0 || line >= c->geo.layout.number_line) return MB_ERR_INVALID;
  auto &m = c->state.marker[line];
  for (int p = 0; p < 3; p++) m[p] = m[p] == 0 ? 2 : m[p] - 1;
  return MB_OK;
}

// getDrag_block (lbm/force_block.h:180-216): momentum exchange over the
// stored links of the drag block, Cd = Fx/(rho0 |U0|^2 m R).
namespace {
// getDrag_block's kernel part: Fx, Fy into out[0..1] (device memory)
int launch_drag(mb_ctx *c, double *out, cudaStream_t s) {
  const int a = c->drag_area;
  const IfBlk &B = c->blk[a];
  DragParams p{};
  p.links = c->d_links;
  p.n = c->n_drag;
  p.F = B.F[c->state.parity[a] ^ 1];
  p.plane = B.plane;
  for (int k = 0; k < 9; k++) p.feqc[k] = c->feqc[k];
  p.sh = c->shift.v;
  p.out = out;
  void *args[] = {&p};
  MB_CUDA(cudaLaunchKernel(kfunc<KDrag>(c->prec), dim3(1), dim3(DRAG_THREADS), args, 0, s));
  return MB_OK;
}

// error_L2's kernel part: the two weighted sums of each part (the interiors
// of the split levels, then each level's other cells) into out[2q..2q+1]
// (device memory; zero for a part without cells); the host adds the parts
// in that order
int launch_l2(mb_ctx *c, double *out, cudaStream_t s) {
  const L2Part *pt = nullptr;
  if (int e = l2_parts(c, current_split_levels(c), &pt)) return e;
  MB_CUDA(cudaMemsetAsync(out, 0, 2 * L2_NPARTS * sizeof(double), s));
  for (int q = 0; q < L2_NPARTS; q++) {
    if (pt[q].grid == 0) continue;
    L2Params p = l2_params(c, pt, q, out + 2 * q);
    void *args[] = {&p};
    MB_CUDA(cudaLaunchKernel(kfunc<KL2>(c->prec), dim3(l2_grid_of(c, pt, q)), dim3(256), args, 0, s));
  }
  return MB_OK;
}

double l2_value(const double *v) {
  double num = v[0], den = v[1];
  for (int q = 1; q < L2_NPARTS; q++) {
    num += v[2 * q];
    den += v[2 * q + 1];
  }
  return std::sqrt(num) / std::sqrt(den);
}

double drag_norm(const mb_ctx *c) {
  const mb_config &cfg = c->geo.config;
  const double u0 = std::sqrt(cfg.U0[0] * cfg.U0[0] + cfg.U0[1] * cfg.U0[1]);
  return cfg.rho0 * u0 * u0 * c->geo.Areas[c->drag_area].m * cfg.R;
}
}  // namespace

extern "C" int mb_drag(mb_ctx *c, double force[2], double *cd, double *cl, mb_stream stream) {
  if (!c || !force) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  if (int e = launch_drag(c, c->d_drag_out, s)) return e;
  MB_CUDA(cudaMemcpyAsync(c->h_drag_out, c->d_drag_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  if (int st = program_status(c)) return st;
  force[0] = c->h_drag_out[0];
  force[1] = c->h_drag_out[1];
  const double den = drag_norm(c);
  if (cd) *cd = force[0] / den;
  if (cl) *cl = force[1] / den;
  return MB_OK;
}

extern "C" int mb_drag_link_count(mb_ctx *c, int *n) {
  if (!c || !n) return MB_ERR_INVALID;
  *n = c->n_drag;
  return MB_OK;
}

// error_L2 (lbm/error_L2.h:57-91)
extern "C" int mb_error_L2(mb_ctx *c, double *e, mb_stream stream) {
  if (!c || !e) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  if (int r = launch_l2(c, c->d_l2_out, s)) return r;
  MB_CUDA(cudaMemcpyAsync(c->h_l2_out, c->d_l2_out, 2 * L2_NPARTS * sizeof(double), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  if (int st = program_status(c)) return st;
  *e = l2_value(c->h_l2_out);
  return MB_OK;
}

// The reference's main loop (Multi-block-LBM.cu:144-158): n coarse steps,
// each followed by getDrag_block and error_L2, with the per-step results
// copied to pinned host memory asynchronously; one synchronisation at the end.
extern "C" int mb_step_diag(mb_ctx *c, int n, double *cd, double *cl, double *err, mb_stream stream) {
  if (!c || n < 0) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  if (n == 0) return MB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (int e = ensure_diag(c, (size_t)n, s)) return e;
  c->kernels_last_call = 0;
  if (c->use_graph != 3) {
    // plans of whole periods with their diagnostics; each plan's results go
    // to the host with one copy
    for (int q = 0; q < n;) {
      bool fin;
      const int chunk = next_chunk(c, n - q, true, &fin);
      int e = 0;
      CompiledPlan *cp = get_diag_plan(c, chunk, &e);
      if (!cp) return e ? e : MB_ERR_INVALID;
      if ((e = exec_plan(c, cp, s))) return e;
      MB_CUDA(cudaMemcpyAsync(c->h_diag + DIAG_STRIDE * q, cp->d_diag_res, (size_t)chunk * DIAG_STRIDE * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
      q += chunk;
    }
  } else {
    for (int q = 0; q < n; q++) {
      int e = 0;
      CompiledPlan *cp = get_plan(c, 1, true, &e);
      if (!cp) return e ? e : MB_ERR_INVALID;
      if ((e = exec_plan(c, cp, s))) return e;
      if ((e = launch_drag(c, c->d_diag + DIAG_STRIDE * q, s))) return e;
      if ((e = launch_l2(c, c->d_diag + DIAG_STRIDE * q + 2, s))) return e;
      MB_CUDA(cudaMemcpyAsync(c->h_diag + DIAG_STRIDE * q, c->d_diag + DIAG_STRIDE * q, DIAG_STRIDE * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
      c->kernels_last_call += 2;
    }
  }
  MB_CUDA(cudaStreamSynchronize(s));
  if (int st = program_status(c)) return st;
  const double den = drag_norm(c);
  for (int q = 0; q < n; q++) {
    const double *v = c->h_diag + DIAG_STRIDE * q;
    if (cd) cd[q] = v[0] / den;
    if (cl) cl[q] = v[1] / den;
    if (err) err[q] = l2_value(v + 2);
  }
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

extern "C" int mb_check_finite(mb_ctx *c, long long *bad, mb_stream stream) {
  if (!c || !bad) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  MB_CUDA(cudaMemsetAsync(c->d_count, 0, sizeof(unsigned long long), s));
  for (int a = 0; a < c->nblk; a++) {
    const IfBlk &B = c->blk[a];
    const void *F = B.F[c->state.parity[a]];
    const int gr = launch_grid((long long)B.nx * B.ny, 256);
    MB_DISPATCH(c->prec, (k_count_nonfinite<P><<<gr, 256, 0, s>>>((const S *)F, B.plane, B.flags, B.nx, B.ny, B.pitch,
                                                                    c->d_count, c->shift.v)));
  }
  unsigned long long h = 0;
  MB_CUDA(cudaMemcpyAsync(&h, c->d_count, sizeof(h), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  if (int st = program_status(c)) return st;
  *bad = (long long)h;
  return h ? MB_ERR_NUMERIC : MB_OK;
}

static int ensure_stage(mb_ctx *c, size_t elems) {
  if (c->stage_elems >= elems) return MB_OK;
  if (c->d_stage) cudaFree(c->d_stage);
  c->d_stage = nullptr;
  c->stage_elems = 0;
  if (cudaMalloc(&c->d_stage, elems * sizeof(double)) != cudaSuccess) return MB_ERR_NOMEM;
  c->stage_elems = elems;
  return MB_OK;
}

extern "C" int mb_copy_fields(mb_ctx *c, int a, double *rho, double *ux, double *uy, double *F, int *solid,
                              mb_stream stream) {
  if (!c || a < 0 || a >= c->nblk) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  MB_CUDA(cudaStreamSynchronize(s));
  if (int st = program_status(c)) return st;
  const IfBlk &B = c->blk[a];
  const long long n = (long long)B.nx * B.ny;
  // one staging area for every requested field: all conversions and copies
  // are queued together and the call waits once
  int e = ensure_stage(c, (size_t)12 * n);
  if (e) return e;
  const int gr = launch_grid(9 * n, 256);
  if (F) {
    const void *Fs = B.F[c->state.parity[a]];
    MB_DISPATCH(c->prec,
                (k_planes_to_f64<P><<<gr, 256, 0, s>>>((const S *)Fs, B.plane, B.nx, B.ny, B.pitch, c->d_stage, c->shift.v)));
    MB_CUDA(cudaMemcpyAsync(F, c->d_stage, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  void *M[3] = {B.rho, B.ux, B.uy};
  double *H[3] = {rho, ux, uy};
  for (int q = 0; q < 3; q++) {
    if (!H[q]) continue;
    double *st = c->d_stage + (9 + q) * n;
    if (c->prec == MB_PREC_F64) k_field_to_f64<double><<<gr, 256, 0, s>>>((const double *)M[q], B.nx, B.ny, B.pitch, st);
    else k_field_to_f64<float><<<gr, 256, 0, s>>>((const float *)M[q], B.nx, B.ny, B.pitch, st);
    MB_CUDA(cudaMemcpyAsync(H[q], st, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  if (solid) {  // host work while the copies run
    const auto &fl = c->hflags[a];
    for (int j = 0; j < B.ny; j++)
      for (int i = 0; i < B.nx; i++) {
        solid[(size_t)j * B.nx + i] = flag_code(fl[(size_t)j * B.pitch + i]);
      }
  }
  MB_CUDA(cudaStreamSynchronize(s));
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

extern "C" int mb_set_fields(mb_ctx *c, int a, const double *rho, const double *ux, const double *uy,
                             const double *F, mb_stream stream) {
  if (!c || a < 0 || a >= c->nblk) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  const IfBlk &B = c->blk[a];
  const long long n = (long long)B.nx * B.ny;
  int e = ensure_stage(c, (size_t)12 * n);
  if (e) return e;
  const int gr = launch_grid(9 * n, 256);
  if (F) {
    MB_CUDA(cudaMemcpyAsync(c->d_stage, F, 9 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    void *Fd = B.F[c->state.parity[a]];
    MB_DISPATCH(c->prec,
                (k_f64_to_planes<P><<<gr, 256, 0, s>>>((S *)Fd, B.plane, B.nx, B.ny, B.pitch, c->d_stage, c->shift.v)));
  }
  void *M[3] = {B.rho, B.ux, B.uy};
  const double *H[3] = {rho, ux, uy};
  for (int q = 0; q < 3; q++) {
    if (!H[q]) continue;
    double *st = c->d_stage + (9 + q) * n;
    MB_CUDA(cudaMemcpyAsync(st, H[q], n * sizeof(double), cudaMemcpyHostToDevice, s));
    if (c->prec == MB_PREC_F64) k_f64_to_field<double><<<gr, 256, 0, s>>>((double *)M[q], B.nx, B.ny, B.pitch, st);
    else k_f64_to_field<float><<<gr, 256, 0, s>>>((float *)M[q], B.nx, B.ny, B.pitch, st);
  }
  MB_CUDA(cudaStreamSynchronize(s));  // the host arrays may be reused on return
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// ---------------------------------------------------------------------------
// Checkpoint / restart.  The reference has none (its steady_<n>.dat files hold
// no distributions).  A checkpoint is the raw device state: both distribution
// buffers of every block (so the drag's read buffer survives too), rho/u and
// u_prev, the ring slots and the scheduler state (buffer parities, ring
// markers), behind a header that pins the layout, so a restart is bit-exact.
// ---------------------------------------------------------------------------
namespace {
struct CkptHeader {
  char magic[8];
  int version, precision, nblk, nline;
  long long slot_points, body_bytes;
  unsigned long long geo_hash;
};
unsigned long long fnv1a(const void *p, size_t n) {
  const unsigned char *b = (const unsigned char *)p;
  unsigned long long h = 1469598103934665603ull;
  for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}
size_t ckpt_bytes(const mb_ctx *c) {
  size_t n = sizeof(CkptHeader);
  for (int a = 0; a < c->nblk; a++) {
    const IfBlk &B = c->blk[a];
    n += 2 * 9 * (size_t)B.plane * prec_bytes(c->prec) + 5 * (size_t)B.plane * real_bytes(c->prec);
  }
  n += (size_t)c->n_slot_points * 27 * real_bytes(c->prec);
  n += sizeof(int) * (c->nblk + 3 * c->geo.layout.number_line);
  return n;
}
}  // namespace

extern "C" int mb_checkpoint_size(mb_ctx *c, long long *bytes) {
  if (!c || !bytes) return MB_ERR_INVALID;
  *bytes = (long long)ckpt_bytes(c);
  return MB_OK;
}

extern "C" int mb_checkpoint_save(mb_ctx *c, void *host, long long bytes, mb_stream stream) {
  if (!c || !host) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  if (bytes < (long long)ckpt_bytes(c)) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char *o = (unsigned char *)host;
  CkptHeader h{};
  std::memcpy(h.magic, "MBLBMCK1", 8);
  h.version = 1;
  h.precision = c->prec | (c->shift_mode << 8);  // the stored words depend on both
  h.nblk = c->nblk;
  h.nline = c->geo.layout.number_line;
  h.slot_points = c->n_slot_points;
  h.body_bytes = (long long)(ckpt_bytes(c) - sizeof(CkptHeader));
  h.geo_hash = fnv1a(&c->geo, sizeof(c->geo));
  std::memcpy(o, &h, sizeof h);
  o += sizeof h;
  const size_t sb = prec_bytes(c->prec), rb = real_bytes(c->prec);
  for (int a = 0; a < c->nblk; a++) {
    const IfBlk &B = c->blk[a];
    for (int q = 0; q < 2; q++) {
      MB_CUDA(cudaMemcpyAsync(o, B.F[q], 9 * (size_t)B.plane * sb, cudaMemcpyDeviceToHost, s));
      o += 9 * (size_t)B.plane * sb;
    }
    void *m[5] = {B.rho, B.ux, B.uy, B.upx, B.upy};
    for (int q = 0; q < 5; q++) {
      MB_CUDA(cudaMemcpyAsync(o, m[q], (size_t)B.plane * rb, cudaMemcpyDeviceToHost, s));
      o += (size_t)B.plane * rb;
    }
  }
  if (c->n_slot_points) {
    MB_CUDA(cudaMemcpyAsync(o, c->d_slots, (size_t)c->n_slot_points * 27 * rb, cudaMemcpyDeviceToHost, s));
    o += (size_t)c->n_slot_points * 27 * rb;
  }
  for (int a = 0; a < c->nblk; a++, o += sizeof(int)) std::memcpy(o, &c->state.parity[a], sizeof(int));
  for (int b = 0; b < c->geo.layout.number_line; b++)
    for (int p = 0; p < 3; p++, o += sizeof(int)) std::memcpy(o, &c->state.marker[b][p], sizeof(int));
  MB_CUDA(cudaStreamSynchronize(s));
  return MB_OK;
}

extern "C" int mb_checkpoint_load(mb_ctx *c, const void *host, long long bytes, mb_stream stream) {
  if (!c || !host) return MB_ERR_INVALID;
  if (bytes < (long long)sizeof(CkptHeader)) return MB_ERR_INVALID;
  const unsigned char *o = (const unsigned char *)host;
  CkptHeader h;
  std::memcpy(&h, o, sizeof h);
  if (std::memcmp(h.magic, "MBLBMCK1", 8) || h.version != 1 || h.precision != (c->prec | (c->shift_mode << 8)) || h.nblk != c->nblk ||
      h.nline != c->geo.layout.number_line || h.slot_points != c->n_slot_points ||
      h.geo_hash != fnv1a(&c->geo, sizeof(c->geo)) || bytes < (long long)ckpt_bytes(c))
    return MB_ERR_INVALID;
  o += sizeof h;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t sb = prec_bytes(c->prec), rb = real_bytes(c->prec);
  for (int a = 0; a < c->nblk; a++) {
    const IfBlk &B = c->blk[a];
    for (int q = 0; q < 2; q++) {
      MB_CUDA(cudaMemcpyAsync(B.F[q], o, 9 * (size_t)B.plane * sb, cudaMemcpyHostToDevice, s));
      o += 9 * (size_t)B.plane * sb;
    }
    void *m[5] = {B.rho, B.ux, B.uy, B.upx, B.upy};
    for (int q = 0; q < 5; q++) {
      MB_CUDA(cudaMemcpyAsync(m[q], o, (size_t)B.plane * rb, cudaMemcpyHostToDevice, s));
      o += (size_t)B.plane * rb;
    }
  }
  if (c->n_slot_points) {
    MB_CUDA(cudaMemcpyAsync(c->d_slots, o, (size_t)c->n_slot_points * 27 * rb, cudaMemcpyHostToDevice, s));
    o += (size_t)c->n_slot_points * 27 * rb;
  }
  for (int a = 0; a < c->nblk; a++, o += sizeof(int)) std::memcpy(&c->state.parity[a], o, sizeof(int));
  for (int b = 0; b < c->geo.layout.number_line; b++)
    for (int p = 0; p < 3; p++, o += sizeof(int)) std::memcpy(&c->state.marker[b][p], o, sizeof(int));
  MB_CUDA(cudaStreamSynchronize(s));
  c->inited = true;
  return MB_OK;
}

// output (output/output.h:2-38): Tecplot POINT zones with %g values
extern "C" int mb_write_tecplot(mb_ctx *c, const char *path) {
  if (!c || !path) return MB_ERR_INVALID;
  FILE *fp = std::fopen(path, "w");
  if (!fp) return MB_ERR_INVALID;
  std::fprintf(fp, "Title= \"LBM 2D\"\n");
  std::fprintf(fp, "VARIABLES= \"X\",\"Y\",\"solid\",\"rho\",\"U\",\"V\",\n");
  int err = MB_OK;
  for (int a = 0; a < c->nblk && err == MB_OK; a++) {
    const mb_area &A = c->geo.Areas[a];
    const size_t n = (size_t)A.nx * A.ny;
    std::vector<double> rho(n), ux(n), uy(n);
    std::vector<int> solid(n);
    err = mb_copy_fields(c, a, rho.data(), ux.data(), uy.data(), nullptr, solid.data(), nullptr);
    if (err) break;
    std::fprintf(fp, "ZONE T= \"zone_level%d\",I= %d,J= %d,F=POINT\n", a, A.nx, A.ny);
    const double dx = 1.0 / A.m;
    for (int j = 0; j < A.ny; j++)
      for (int i = 0; i < A.nx; i++) {
        const size_t q = (size_t)j * A.nx + i;
        std::fprintf(fp, "%g\t%g\t%d\t%g\t%g\t%g\n", i * dx + A.base_x, j * dx + A.base_y, solid[q], rho[q], ux[q],
                     uy[q]);
      }
  }
  std::fclose(fp);
  return err;
}

extern "C" int mb_stats(mb_ctx *c, long long *kl, long long *kps, long long *ups) {
  if (!c) return MB_ERR_INVALID;
  if (kl) *kl = c->kernels_last_call;
  if (kps) {
    // launches of one final-state coarse step from the current scheduler
    // state (its plan is compiled here if no step call has needed it yet)
    *kps = 0;
    if (c->inited) {
      int err = 0;
      const SchedState save = c->state;
      CompiledPlan *cp = get_plan(c, 1, true, &err);
      c->state = save;
      if (!cp) return err ? err : MB_ERR_INVALID;
      *kps = cp->kernels;
    }
  }
  if (ups) *ups = c->updates_per_step;
  return MB_OK;
}

extern "C" int mb_time_block_step(mb_ctx *c, int level, int n, mb_stream stream, double *ms, double *bytes,
                                  long long *cells) {
  if (!c || level < 0 || level >= c->geo.layout.LEVEL || n < 1) return MB_ERR_INVALID;
  if (!c->inited) return MB_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  const mb_layout &L = c->geo.layout;
  uint64_t par = 0;
  for (int a = 0; a < c->nblk; a++)
    if (c->state.parity[a]) par |= 1ull << a;
  std::vector<StbParams> ps;
  long long tot = 0;
  for (int a0 = L.ASP[level]; a0 < L.ASP[level + 1]; a0 += STB_MAX_BLOCKS) {
    const int a1 = std::min(L.ASP[level + 1], a0 + STB_MAX_BLOCKS);
    ps.push_back(make_stb(c, a0, a1, par, 0, 0, STB_ALL, stb_tile(c, level, STB_ALL), 0));
    for (int a = a0; a < a1; a++) tot += (long long)c->blk[a].nx * c->blk[a].ny;
  }
  void *fn = nullptr;
  auto grid_of = [&](const StbParams &p) {
    dim3 gr;
    stb_launch_shape(c, level, STB_ALL, false, p, &fn, &gr);
    return gr;
  };
  { dim3 g0 = grid_of(ps[0]); (void)g0; }
  // the n launches replay as one CUDA graph on a private stream, so that
  // the host's launch rate does not bound launches of a few microseconds
  MB_CUDA(cudaStreamSynchronize(s));
  cudaStream_t cs;
  MB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t gr = nullptr;
  cudaGraphExec_t ge = nullptr;
  MB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  for (int it = 0; it < n; it++)
    for (auto &p : ps) {
      void *args[] = {&p};
      const dim3 threads(fn == kfunc<KStb>(c->prec) ? STB_CHAIN_THREADS : 256);  // the grid's CTA size
      if (cudaLaunchKernel(fn, grid_of(p), threads, args, 0, cs) != cudaSuccess) break;
    }
  const cudaError_t ce = cudaStreamEndCapture(cs, &gr);
  if (ce != cudaSuccess || cudaGraphInstantiate(&ge, gr, 0) != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    cudaStreamDestroy(cs);
    return MB_ERR_CUDA;
  }
  cudaEvent_t e0, e1;
  MB_CUDA(cudaEventCreate(&e0));
  MB_CUDA(cudaEventCreate(&e1));
  MB_CUDA(cudaGraphLaunch(ge, cs));  // warm-up
  MB_CUDA(cudaEventRecord(e0, cs));
  MB_CUDA(cudaGraphLaunch(ge, cs));
  MB_CUDA(cudaEventRecord(e1, cs));
  MB_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  MB_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGraphExecDestroy(ge);
  cudaGraphDestroy(gr);
  cudaStreamDestroy(cs);
  if (ms) *ms = t / n;
  if (bytes) *bytes = (double)tot * 18.0 * (double)prec_bytes(c->prec);
  if (cells) *cells = tot;
  return MB_OK;
}

// =============================================================================
// Batches: many independent cases advanced together.  Cases whose compiled
// plans have the same structure (node kinds, dependencies and launch shapes;
// e.g. nested-frame layouts with the same number of levels, whatever their
// sizes) share one DAG: each plan node becomes one launch over all cases
// (kb_block_step, kb_records, kb_spline), and the DAG is replayed as a CUDA
// graph.  Cases keep their own state and remain usable one by one between
// batch calls.
// =============================================================================
namespace {
struct BatchPlan {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<SchedState> end;  // per case
  std::vector<void *> dev;
  long long kernels = 0;
  bool uploaded = false;
  ~BatchPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void *p : dev) cudaFree(p);
  }
};
}  // namespace

struct mb_batch {
  std::vector<mb_ctx *> cases;
  int prec = 0;
  int period = 1;
  std::map<std::string, std::unique_ptr<BatchPlan>> plans;
  long long updates_per_step = 0;
  long long kernels_last_call = 0;
  double *d_drag = nullptr;  // 2 per case
  double *h_drag = nullptr;  // pinned
  // block-step schedule: 0 one CTA per tile of 256 cells (kb_block_step);
  // k > 0 a persistent grid of k CTAs per SM over equal shares of the
  // tiles (kb_block_step_ps)
  int stb_ctas_per_sm = 0;
  // block-step kernel: 0 one cell per thread, 1 cell pairs (one CTA per
  // pair-kernel CTA, kb_block_step_pt, or with a schedule k > 0 a persistent
  // grid over them, kb_block_step_pp) on the nodes where every case's launch
  // fits the pair form
  int stb_kernel = 0;
  int num_sms = 148;
  long long steps_done = 0;  // coarse steps of mb_batch_step calls (the autotuner's included)
};

namespace {
int batch_plan(mb_batch *b, int n, bool fin, BatchPlan **out) {
  const std::string key = b->cases[0]->state.key() + "/" + std::to_string(n) + (fin ? "F" : "P");
  auto it = b->plans.find(key);
  if (it != b->plans.end()) {
    *out = it->second.get();
    return MB_OK;
  }
  const int nc = (int)b->cases.size();
  std::vector<CompiledPlan *> parts(nc, nullptr);
  std::vector<int> errs(nc, 0);
  {  // every case compiles its own plan: spread the cases over host threads
    const int nt = std::max(1, std::min<int>(nc, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next{0};
    auto work = [&]() {
      cudaSetDevice(b->cases[0]->device);
      for (int c = next++; c < nc; c = next++) parts[c] = get_plan(b->cases[c], n, fin, &errs[c], true);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
  }
  for (int c = 0; c < nc; c++)
    if (!parts[c]) return errs[c] ? errs[c] : MB_ERR_INVALID;
  const auto &d0 = parts[0]->dn;
  for (int c = 1; c < nc; c++) {  // one DAG for all cases
    const auto &dc = parts[c]->dn;
    if (dc.size() != d0.size()) return MB_ERR_UNSUPPORTED;
    for (size_t q = 0; q < d0.size(); q++)
      if (dc[q].kind != d0[q].kind || dc[q].deps != d0[q].deps || dc[q].block.x != d0[q].block.x ||
          dc[q].background != d0[q].background)
        return MB_ERR_UNSUPPORTED;
  }
  auto bp = std::make_unique<BatchPlan>();
  MB_CUDA(cudaGraphCreate(&bp->graph, 0));
  std::vector<cudaGraphNode_t> gn(d0.size(), nullptr);
  for (size_t q = 0; q < d0.size(); q++) {
    const DevPlanNode &n0 = d0[q];
    size_t psz;
    void *func;
    unsigned block = n0.block.x;
    size_t smem = 0;
    // cell pairs on this node: every case's launch covers a whole level or an
    // interior with 32-bit offsets
    bool pairs = n0.kind == NK_STB && b->stb_kernel == 1;
    for (int c = 0; c < nc && pairs; c++)
      pairs = parts[c]->dn[q].stb.region != STB_RIM && rows_fit(b->cases[c], parts[c]->dn[q].stb);
    if (n0.kind == NK_STB) {
      psz = sizeof(StbParams);
      if (pairs) func = b->stb_ctas_per_sm > 0 ? kfunc<KBStbPp>(b->prec) : kfunc<KBStbPt>(b->prec);
      else func = b->stb_ctas_per_sm > 0 ? kfunc<KBStbPs>(b->prec) : kfunc<KBStb>(b->prec);
      block = 256;
    } else if (n0.kind == NK_REC) {
      psz = sizeof(RecOpsParams);
      func = kfunc<KBRec>(b->prec);
    } else {
      psz = sizeof(SplParamsP);
      func = kfunc<KBSpl>(b->prec);
      smem = (sizeof(SplParamsP) + 15) / 16 * 16 + spline_smem(b->prec) / SPL_WARPS * (n0.block.x / 32);
    }
    const size_t stride = (psz + 15) / 16 * 16;
    std::vector<unsigned char> host(stride * nc + sizeof(int) * (nc + 1), 0);
    int *cta0 = (int *)(host.data() + stride * nc);
    long long ctas = 0;
    for (int c = 0; c < nc; c++) {
      const DevPlanNode &dn = parts[c]->dn[q];
      const void *src = n0.kind == NK_STB ? (const void *)&dn.stb : n0.kind == NK_REC ? (const void *)&dn.rec
                                                                                      : (const void *)&dn.spl;
      std::memcpy(host.data() + stride * c, src, psz);
      cta0[c] = (int)ctas;
      if (pairs) ctas += dn.stb.pctas;
      else if (n0.kind == NK_STB) ctas += (dn.stb.total + 255) / 256;
      else ctas += dn.grid.x;
      if (ctas >= (1LL << 31)) return MB_ERR_UNSUPPORTED;
    }
    cta0[nc] = (int)ctas;
    std::vector<cudaGraphNode_t> deps;
    for (int p : n0.deps)
      if (gn[p]) deps.push_back(gn[p]);
    if (ctas == 0) {
      MB_CUDA(cudaGraphAddEmptyNode(&gn[q], bp->graph, deps.data(), deps.size()));
      continue;
    }
    void *dp = nullptr;
    if (cudaMalloc(&dp, host.size()) != cudaSuccess) return MB_ERR_NOMEM;
    bp->dev.push_back(dp);
    MB_CUDA(cudaMemcpy(dp, host.data(), host.size(), cudaMemcpyHostToDevice));
    BatchArgs a{};
    a.params = (const unsigned char *)dp;
    a.cta0 = (const int *)((unsigned char *)dp + stride * nc);
    a.ncases = nc;
    a.pstride = (int)stride;
    void *args[1] = {&a};
    cudaKernelNodeParams kp{};
    kp.func = func;
    kp.gridDim = dim3((unsigned)ctas);
    if (n0.kind == NK_STB && b->stb_ctas_per_sm > 0)
      kp.gridDim = dim3((unsigned)std::min<long long>(ctas, (long long)b->num_sms * b->stb_ctas_per_sm));
    kp.blockDim = dim3(block);
    kp.sharedMemBytes = (unsigned)smem;
    kp.kernelParams = args;
    MB_CUDA(cudaGraphAddKernelNode(&gn[q], bp->graph, deps.data(), deps.size(), &kp));
    if (int e = set_priority(gn[q], n0.background)) return e;
    bp->kernels++;
  }
  MB_CUDA(cudaGraphInstantiateWithFlags(&bp->exec, bp->graph, cudaGraphInstantiateFlagUseNodePriority));
  bp->end.resize(nc);
  for (int c = 0; c < nc; c++) bp->end[c] = parts[c]->end;
  *out = bp.get();
  b->plans[key] = std::move(bp);
  return MB_OK;
}

bool batch_in_step(const mb_batch *b) {
  for (const mb_ctx *c : b->cases)
    if (!(c->state == b->cases[0]->state)) return false;
  return true;
}
}  // namespace

extern "C" int mb_batch_create(mb_ctx *const *cases, int n, mb_batch **out) {
  if (!cases || n < 1 || !out) return MB_ERR_INVALID;
  *out = nullptr;
  auto b = std::make_unique<mb_batch>();
  for (int q = 0; q < n; q++) {
    mb_ctx *c = cases[q];
    if (!c) return MB_ERR_INVALID;
    if (!c->inited) return MB_ERR_STATE;
    if (options_on(c)) return MB_ERR_UNSUPPORTED;  // batched kernels run the BGK/SBB step only
    if (q > 0 && (c->prec != cases[0]->prec || c->period != cases[0]->period ||
                  c->geo.layout.LEVEL != cases[0]->geo.layout.LEVEL || c->device != cases[0]->device))
      return MB_ERR_UNSUPPORTED;
    b->cases.push_back(c);
    b->updates_per_step += c->updates_per_step;
  }
  if (!batch_in_step(b.get())) return MB_ERR_STATE;
  b->prec = cases[0]->prec;
  b->period = cases[0]->period;
  b->num_sms = cases[0]->num_sms > 0 ? cases[0]->num_sms : 148;
  cudaDeviceSynchronize();
  for (mb_ctx *c : b->cases) {  // batched launches use one cell per thread and CUDA-graph plans
    bool clear = c->use_graph != 1;
    for (int l = 0; l < MB_MAX_LEVEL; l++) clear |= c->stb_variant[l] != 0;
    if (clear) {
      c->use_graph = 1;
      for (int l = 0; l < MB_MAX_LEVEL; l++) c->stb_variant[l] = 0;
      c->plans.clear();
    }
  }
  if (cudaMalloc(&b->d_drag, 2 * sizeof(double) * n) != cudaSuccess) return MB_ERR_NOMEM;
  if (cudaMallocHost(&b->h_drag, 2 * sizeof(double) * n) != cudaSuccess) {
    cudaFree(b->d_drag);
    return MB_ERR_NOMEM;
  }
  *out = b.release();
  return MB_OK;
}

extern "C" int mb_batch_destroy(mb_batch *b) {
  if (!b) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  b->plans.clear();
  if (b->d_drag) cudaFree(b->d_drag);
  if (b->h_drag) cudaFreeHost(b->h_drag);
  delete b;
  return MB_OK;
}

extern "C" int mb_batch_step(mb_batch *b, int n, mb_stream stream) {
  if (!b || n < 0) return MB_ERR_INVALID;
  if (!batch_in_step(b)) return MB_ERR_STATE;
  for (mb_ctx *c : b->cases)
    if (options_on(c)) return MB_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  b->kernels_last_call = 0;
  int remaining = n;
  const int G = b->period;
  while (remaining > 0) {
    int chunk;
    bool fin;
    if (remaining - 1 >= G) { chunk = G; fin = false; }
    else if (remaining > 1) { chunk = 1; fin = false; }
    else { chunk = 1; fin = true; }
    BatchPlan *bp = nullptr;
    if (int e = batch_plan(b, chunk, fin, &bp)) return e;
    MB_CUDA(cudaGraphLaunch(bp->exec, s));
    for (size_t c = 0; c < b->cases.size(); c++) b->cases[c]->state = bp->end[c];
    b->kernels_last_call += bp->kernels;
    remaining -= chunk;
  }
  b->steps_done += n;
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// Builds the graphs mb_batch_step(n) will replay from the current state.
extern "C" int mb_batch_prepare(mb_batch *b, int n) {
  if (!b || n < 0) return MB_ERR_INVALID;
  if (!batch_in_step(b)) return MB_ERR_STATE;
  const int nc = (int)b->cases.size();
  std::vector<SchedState> save(nc);
  for (int c = 0; c < nc; c++) save[c] = b->cases[c]->state;
  int remaining = n, err = MB_OK;
  const int G = b->period;
  cudaStream_t up = nullptr;
  MB_CUDA(cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking));
  while (remaining > 0 && !err) {
    int chunk;
    bool fin;
    if (remaining - 1 >= G) { chunk = G; fin = false; }
    else if (remaining > 1) { chunk = 1; fin = false; }
    else { chunk = 1; fin = true; }
    BatchPlan *bp = nullptr;
    err = batch_plan(b, chunk, fin, &bp);
    if (!err && !bp->uploaded) {  // the first replay then pays no upload
      err = cudaGraphUpload(bp->exec, up) == cudaSuccess ? MB_OK : MB_ERR_CUDA;
      bp->uploaded = true;
    }
    if (!err)
      for (int c = 0; c < nc; c++) b->cases[c]->state = bp->end[c];
    remaining -= chunk;
  }
  for (int c = 0; c < nc; c++) b->cases[c]->state = save[c];
  if (cudaStreamSynchronize(up) != cudaSuccess && !err) err = MB_ERR_CUDA;
  cudaStreamDestroy(up);
  return err;
}

extern "C" int mb_batch_drag(mb_batch *b, double *cd, double *cl, mb_stream stream) {
  if (!b) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = (int)b->cases.size();
  for (int c = 0; c < nc; c++)
    if (int e = launch_drag(b->cases[c], b->d_drag + 2 * c, s)) return e;
  MB_CUDA(cudaMemcpyAsync(b->h_drag, b->d_drag, 2 * sizeof(double) * nc, cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  for (int c = 0; c < nc; c++) {
    const double den = drag_norm(b->cases[c]);
    if (cd) cd[c] = b->h_drag[2 * c] / den;
    if (cl) cl[c] = b->h_drag[2 * c + 1] / den;
  }
  return MB_OK;
}

extern "C" int mb_batch_stats(mb_batch *b, long long *updates_per_step, long long *kernels_last_call,
                              long long *coarse_steps_done) {
  if (!b) return MB_ERR_INVALID;
  if (updates_per_step) *updates_per_step = b->updates_per_step;
  if (kernels_last_call) *kernels_last_call = b->kernels_last_call;
  if (coarse_steps_done) *coarse_steps_done = b->steps_done;
  return MB_OK;
}

// Interface work granularity of every case (mb_set_interface_shape), as
// the batch autotuner varies it.
extern "C" int mb_batch_set_interface_shape(mb_batch *b, int rec_points, int spline_segments) {
  if (!b) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  b->plans.clear();
  for (mb_ctx *c : b->cases)
    if (int e = mb_set_interface_shape(c, rec_points, spline_segments)) return e;
  return MB_OK;
}

extern "C" int mb_batch_set_schedule(mb_batch *b, int stb_ctas_per_sm) {
  if (!b || stb_ctas_per_sm < 0 || stb_ctas_per_sm > 8) return MB_ERR_INVALID;
  if (b->prec == MB_PREC_F64 && stb_ctas_per_sm > 4) return MB_ERR_INVALID;  // launch bounds: 4 CTAs per SM
  cudaDeviceSynchronize();
  b->plans.clear();
  b->stb_ctas_per_sm = stb_ctas_per_sm;
  return MB_OK;
}

extern "C" int mb_batch_set_kernel(mb_batch *b, int kernel) {
  if (!b || kernel < 0 || kernel > 1) return MB_ERR_INVALID;
  cudaDeviceSynchronize();
  b->plans.clear();
  b->stb_kernel = kernel;
  return MB_OK;
}

namespace {
// Mean device time of one coarse step of the batch with its current shapes:
// one untimed chunk (period + 1 steps) builds the graphs, then `steps` timed
// steps.  Both advance the cases.
int batch_time(mb_batch *b, int steps, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, double *ms) {
  if (int e = mb_batch_step(b, b->period + 1, s)) return e;
  if (int e = mb_batch_prepare(b, steps)) return e;
  MB_CUDA(cudaEventRecord(e0, s));
  if (int e = mb_batch_step(b, steps, s)) return e;
  MB_CUDA(cudaEventRecord(e1, s));
  MB_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  MB_CUDA(cudaEventElapsedTime(&t, e0, e1));
  *ms = t / steps;
  return MB_OK;
}
}  // namespace

// Coordinate search: first the block-step kernel and schedule (one cell per
// thread, and cell pairs, each with one CTA per tile or a persistent grid of
// 2, 4 (or 8, one cell per thread) CTAs per SM over equal shares of the
// tiles) with the default interface shape, then, with the best of
// those, the interface shapes (points per record CTA, spline segments per
// CTA).  Each candidate is timed over `steps` coarse steps after one untimed
// chunk that builds its graphs; the fastest is kept.  The timing steps
// advance the cases.
extern "C" int mb_batch_autotune(mb_batch *b, int steps, mb_stream stream, int *rec_points, int *spline_segments,
                                 int *stb_ctas_per_sm, double *ms_per_step, int *stb_kernel) {
  if (!b || steps < 1) return MB_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  static const int sched[][2] = {{0, 0}, {0, 2}, {0, 4}, {0, 8}, {1, 0}, {1, 2}, {1, 4}};  // (kernel, CTAs per SM)
  static const int cand[][2] = {{64, 1}, {32, 2}, {64, 2}, {64, 4}};
  cudaEvent_t e0, e1;
  MB_CUDA(cudaEventCreate(&e0));
  MB_CUDA(cudaEventCreate(&e1));
  double best = 1e30, ms = 0;
  int bk = 0, bkern = 0, br = 32, bs = 1, err = MB_OK;
  if ((err = mb_batch_set_interface_shape(b, 32, 1))) return err;
  for (const auto &ks : sched) {
    if (b->prec == MB_PREC_F64 && ks[1] > 4) continue;
    if ((err = mb_batch_set_kernel(b, ks[0])) || (err = mb_batch_set_schedule(b, ks[1])) ||
        (err = batch_time(b, steps, s, e0, e1, &ms)))
      break;
    if (ms < best) { best = ms; bkern = ks[0]; bk = ks[1]; }
  }
  if (!err) err = mb_batch_set_kernel(b, bkern);
  if (!err) err = mb_batch_set_schedule(b, bk);
  for (int q = 0; q < 4 && !err; q++) {
    if ((err = mb_batch_set_interface_shape(b, cand[q][0], cand[q][1])) || (err = batch_time(b, steps, s, e0, e1, &ms)))
      break;
    if (ms < best) { best = ms; br = cand[q][0]; bs = cand[q][1]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err) return err;
  if (int e = mb_batch_set_interface_shape(b, br, bs)) return e;
  if (rec_points) *rec_points = br;
  if (spline_segments) *spline_segments = bs;
  if (stb_ctas_per_sm) *stb_ctas_per_sm = bk;
  if (stb_kernel) *stb_kernel = bkern;
  if (ms_per_step) *ms_per_step = best;
  return MB_OK;
}
