// mblbm_internal.h - host-side internal types shared by the geometry, plan
// compiler and CUDA context translation units.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mblbm.h"

namespace mblbm {

// cell classes in the per-cell flag byte (bits 0-1), plus attribute bits
enum : uint8_t {
  CT_FLUID = 0,
  CT_SOLID = 1,
  CT_COPY = 2,  // C_BOUNDARY (never streamed or collided; evolution_block.h:17,44,90)
  CT_PAD = 3,   // row padding beyond nx
  CF_EDGE = 4,  // i==0 || j==0 || i==nx-1 || j==ny-1
  CF_MACRO = 8, // rho/ux/uy of this FLUID cell are read by an interface op
  CF_HBB = 16,  // CT_SOLID cell that is a half-way bounce-back wall (MB_SOLID_HBB)
  CF_FCSRC = 16, // CT_FLUID cell (not on the block edge) that is the fine point of an f_c line: a
                 // block step may do that f_c point itself (PlanNode::fc); same bit as CF_HBB
  CF_SLIP = 32, // CT_SOLID cell that is an on-node free-slip wall (MB_SOLID_SLIP)
  CF_CCPULL = 64, // C_BOUNDARY target of a same-level copy run beside its level's block step (NK_CCP)
  CF_TSKIP = 128, // fine edge cell of a temporal interpolation that a spline may do early: a block step
                  // flagged tskip leaves it alone (the spline writes its next value there)
};

bool obstacle_contains(const mb_config &c, double x, double y);
bool periodic_ghost(const mb_config &c, double x, double y);
int cell_type(const mb_geometry &g, int a, int i, int j);

// One interface point operation (16 bytes, the unit of the record kernel).
// REC_FC_SLOT: an f_c point whose fine cell's F was last written by a c_f
// record; it reads that value from the c_f's slot (slot point in
// m0 | m1 << 8 | pad << 16, marker m2), so the two can share a launch.
enum : uint8_t { REC_CC = 0, REC_TEMPORAL = 1, REC_CF = 2, REC_FC = 3, REC_FC_SLOT = 4 };
enum : uint8_t {
  RB_SRC_BUF = 1,   // current F buffer of the source block
  RB_DST_BUF = 2,   // current F buffer of the target block
  RB_WRITE_F = 4,   // write the distributions (cleared when a later op of the batch overwrites them)
  RB_WRITE_M = 8,   // write rho/ux/uy
  RB_WIDX_SHIFT = 4 // 2 bits: index of the temporal weight triple
};
struct Rec {
  uint8_t type;
  uint8_t bits;
  uint8_t dst_block;
  uint8_t src_block;
  uint8_t m0, m1, m2, pad;
  int32_t dst_cell;  // j*pitch + i in the target block
  int32_t src;       // source cell (j*pitch + i) or slot point id
};
static_assert(sizeof(Rec) == 16, "Rec must be 16 bytes");

// Static description of a coarse-fine line for the spline kernel.
struct SplLine {
  int coarse, fine;      // block ids
  int Nc, Nf, r;
  int ci0, cj0, cdi, cdj;  // coarse source line: start and unit step
  int fi0, fj0, fdi, fdj;  // fine edge line
  int slot0;             // point id of fine point 0 in the slot array
  double para;           // (tau_f - 1) / (r (tau_c - 1)), assit_multi.h:176
};

// Launch limits of one record / spline node (the launch parameters hold
// every op, line and block descriptor, see kernels.cuh).
constexpr int PLAN_MAX_REC_OPS = 24;
constexpr int PLAN_MAX_SPL_TASKS = 16;
// error_L2 parts: 0 the interiors of split levels, 1 + l level l (its rim
// when split, every cell otherwise); per coarse step a diagnostic plan
// stores Fx, Fy and the two sums of every part
constexpr int L2_NPARTS = 1 + MB_MAX_LEVEL;
constexpr int DIAG_STRIDE = 2 + 2 * L2_NPARTS;

// One line of a spline node.
struct SplTask {
  int line;       // index into the SplLine table
  int src_buf;    // current F buffer of the coarse block
  int m0;         // slot written (marker[0] at the time of the call)
  int mask_off;   // offset into the node's M-write mask (-1: write all points)
  // the temporal interpolation of the line that follows, fused (tmp = 1): F
  // of each fine edge point, buffer tbuf, <- tw0 s[tm0] - tw1 s[tm1] + tw2 s[tm2]
  int tmp = 0, tbuf = 0, tmask_off = -1;
  int tm[3] = {0, 0, 0};
  double tw[3] = {0, 0, 0};
};

// NK_CCP: same-level copies beside a block step.  NK_DRAG: getDrag_block of
// a coarse step; NK_L2: one part of its error_L2 (region STB_INTERIOR: the
// interiors of the split levels in a0's bit mask, else every other cell);
// `level` holds the step's index within the plan for both.
// NK_FCP: the CF_FCSRC cells of a block step and their f_c points, beside it.
enum NodeKind { NK_STB = 0, NK_REC = 1, NK_SPL = 2, NK_CCP = 3, NK_FCP = 4, NK_DRAG = 5, NK_L2 = 6 };
// cells a block-step node updates: all, those at distance >= 2 from the block
// edge (they read nothing an interface op writes), or the distance <= 1 rim
enum StbRegion { STB_ALL = 0, STB_INTERIOR = 1, STB_RIM = 2 };

// An f_c point (f_c_boundary_transfer, multi/FH/assit_multi.h:273-314) done
// by an NK_FCP node beside the block step that updates its fine cell: coarse
// cell dst_cell of dst_block, F in buffer dst_buf, gets feq + para (f - feq)
// of the fine cell's new values, and its rho/u.
struct FcFuse {
  int src_block, src_cell, dst_block, dst_cell;
  uint8_t bits;     // RB_WRITE_F | RB_WRITE_M still live
  uint8_t dst_buf;
  double para;      // r (tau_c - 1) / (tau_f - 1), as the record kernel computes it
};

struct PlanNode {
  NodeKind kind;
  int level = -1;             // STB
  int a0 = 0, a1 = 0;         // STB: block range [a0, a1)
  int region = STB_ALL;       // STB: StbRegion
  uint64_t parity = 0;        // STB: current buffer of each block before the step
  int macro_all = 0;          // STB: write rho/u of every FLUID cell
  int ccpull = 0;             // STB: skips CF_CCPULL cells (an NK_CCP node of the same level writes them)
  int part = 0;               // L2: the error_L2 part (L2_NPARTS)
  int tskip = 0;              // STB: leaves CF_TSKIP cells alone (a spline writes them)
  int fcskip = 0;             // STB: leaves CF_FCSRC cells alone (an NK_FCP node updates them)
  std::vector<FcFuse> fc;     // FCP: the f_c points it does
  std::vector<Rec> recs;      // REC
  std::vector<std::pair<int, int>> ops;  // REC: (first record, count) of each reference line op
  double tw[4][3] = {};       // REC: temporal weight triples (a, b, c)
  int ntw = 0;
  std::vector<SplTask> spl;   // SPL
  std::vector<uint8_t> spl_mask;
  std::vector<int> deps;      // earlier nodes this one waits for (transitively reduced)
  std::string label;
};

// Symbolic scheduler state: current buffer per block and ring markers per line.
struct SchedState {
  std::vector<int> parity;             // per block
  std::vector<std::array<int, 3>> marker;  // per coarse-fine line
  bool operator==(const SchedState &o) const { return parity == o.parity && marker == o.marker; }
  std::string key() const;
};

struct BlockLayout {
  int nx, ny, pitch;
  long long plane;  // elements between planes k and k+1
};

// One call of the reference scheduler: a block step of a level or one line op.
struct Op {
  // DRAG, L2: the per-step diagnostics of a diagnostic plan (line = the coarse
  // step's index within the plan; level = the part of an L2 op)
  enum Kind { STB = 0, CC = 1, TEMPORAL = 2, CF = 3, FC = 4, SPL = 5, DRAG = 7, L2 = 8 } kind;
  int level = -1, line = -1;
  double xm = 0;
  int macro_all = 0;
  std::vector<int> parity;  // current buffer of every block at the call
  std::array<int, 3> mk{};  // ring markers of the line at the call
  // SPL with the line's next temporal interpolation fused (fuse_temporal):
  // the temporal op's xm, markers and block buffers
  int tmp = 0;
  double txm = 0;
  std::array<int, 3> tmk{};
  std::vector<int> tparity;
  int tskip = 0;  // STB: leaves CF_TSKIP cells alone (fuse_early)
};

// Same-level copies (c_c_boundary_transfer) of one level with chains
// resolved: after the copies of the level run in order, target cell
// (tblk, tcell) holds what source cell (sblk, scell) has after the level's
// block step.  Cells are pitched (j * pitch + i).
struct CcLink {
  int tblk, sblk;
  long long tcell, scell;
};
struct CcLevel {
  bool fusable = false;           // `links` can run beside the level's block step
  std::vector<CcLink> links;      // FLUID source, C_BOUNDARY target: run beside the block step (CF_CCPULL)
  std::vector<CcLink> rec_links;  // other sources (their rho/u may come from later ops): point copies after the step
};
// One CcLevel per level, from the line tables (Line_Inf_CC, LCCP).
std::vector<CcLevel> cc_levels(const mb_geometry &g, const std::vector<BlockLayout> &bl,
                               const std::vector<std::vector<uint8_t>> &flags);

// Compiles n coarse steps of evolution() (evolution.h:2-65) starting from
// state s into plan nodes with dependency edges; advances s.  final_macros:
// the last sub-step of every level writes rho/u of all FLUID cells.
struct PlanCompiler {
  const mb_geometry &g;
  const std::vector<BlockLayout> &bl;
  const std::vector<std::vector<uint8_t>> &flags;  // per block, pitched
  const std::vector<SplLine> &spl_lines;
  // levels with at least this many cells step their interior and rim as two nodes
  long long split_cells = 1000000;
  // nonzero: level l splits exactly when bit l is set (overrides split_cells)
  unsigned split_mask = 0;
  // non-null: same-level copies of fusable levels run inside the block step
  const std::vector<CcLevel> *cc = nullptr;
  // a spline of a coarse-fine line also does the line's temporal
  // interpolation of the fine level's next substep (fuse_temporal)
  bool fuse_tmp = false;
  // levels (bit per level) whose splines do that interpolation in place, the
  // level's substep between them leaving the edge cells alone (fuse_early);
  // their edge cells carry CF_TSKIP
  unsigned early_levels = 0;
  // f_c points whose fine cell the level's last block step has just updated
  // run in an NK_FCP node beside that step (FcFuse), which updates the
  // CF_FCSRC cells of the step, when no op between them touches their cells
  bool fuse_fc = false;
  unsigned fc_levels = ~0u;  // fine levels (bit per level) whose f_c points may fuse
  // record launches keep ops that wait for the latest block step apart from
  // ops that do not
  bool split_waits = false;
  PlanCompiler(const mb_geometry &g_, const std::vector<BlockLayout> &bl_,
               const std::vector<std::vector<uint8_t>> &fl, const std::vector<SplLine> &sl)
      : g(g_), bl(bl_), flags(fl), spl_lines(sl) {}
  std::vector<PlanNode> compile(SchedState &s, int n_coarse, bool final_macros) const;
  // n coarse steps, each with rho/u of every FLUID cell written and followed
  // by its drag and relative L2 change (the reference's main loop,
  // Multi-block-LBM.cu:148-158)
  std::vector<PlanNode> compile_diag(SchedState &s, int n_coarse) const;
  int drag_area = -1;  // block of getDrag_block (compile_diag)
  unsigned split_levels() const;  // levels stepped as interior and rim nodes (bit per level)
  // one reference call (Op::Kind, level or line index) at state s, state unchanged
  std::vector<PlanNode> compile_single(int kind, int index, double xm, const SchedState &s) const;
  // line ops expanded into launches (REC / SPL batches, STB nodes) with DAG edges
  std::vector<PlanNode> build(const std::vector<Op> &ops) const;
  // ops with the fusions switched on (fuse_early, fuse_tmp) applied
  std::vector<Op> fused(const std::vector<Op> &ops) const;
};

// Cells whose rho/ux/uy an interface op reads (the CF_MACRO attribute).
void mark_macro_sources(const mb_geometry &g, const std::vector<BlockLayout> &bl,
                        std::vector<std::vector<uint8_t>> &flags);
// FLUID cells off the block edge that are fine points of f_c lines (CF_FCSRC);
// the bit is cleared on every other FLUID cell.
void mark_fc_sources(const mb_geometry &g, const std::vector<BlockLayout> &bl,
                     std::vector<std::vector<uint8_t>> &flags);

}  // namespace mblbm
