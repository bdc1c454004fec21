// plan.cpp - plan compiler: the reference level scheduler as a dependency DAG.
//
// evolution() (evolution.h:2-65 of zhangya9741/Multi-block-LBM-GPU) issues,
// per level and sub-step, temporal interpolation, the block step of every
// block of the level, same-level copies, spatial interpolation with ring
// rotation, recursion into the next level and the fine-to-coarse transfers,
// one kernel per line on the default stream.  Here the same sequence is
// replayed symbolically (parities of the ping-pong buffers and ring markers
// are tracked on the host), every line op is expanded into point records,
// consecutive ops are merged into one launch when no point of the launch
// reads what an earlier op of it writes (or the other way round), and the
// launches become nodes of a DAG whose edges are exactly the read/write
// conflicts.  Replaying the DAG in any topological order gives the values of
// the sequential order.
#include <algorithm>
#include <cstdio>
#include <map>
#include <set>
#include <unordered_map>
#include <unordered_set>

#include "mblbm_internal.h"

namespace mblbm {

std::string SchedState::key() const {
  std::string k;
  for (int p : parity) k.push_back(char('0' + p));
  k.push_back('|');
  for (auto &m : marker) {
    k.push_back(char('0' + m[0]));
    k.push_back(char('0' + m[1]));
    k.push_back(char('0' + m[2]));
  }
  return k;
}

namespace {

// resource kinds of an access key
// RK_UP: u_prev of error_L2; RK_DIAG: the per-step diagnostic results
enum : uint64_t { RK_F0 = 0, RK_F1 = 1, RK_M = 2, RK_SLOT = 3, RK_UP = 5, RK_DIAG = 6 };

inline uint64_t key(uint64_t kind, uint64_t owner, uint64_t idx) { return (kind << 56) | (owner << 48) | idx; }
inline uint32_t summ(uint64_t k) { return uint32_t(k >> 48); }  // kind<<8 | owner
inline uint64_t fkey(int buf, int block, long long cell) { return key(buf ? RK_F1 : RK_F0, block, cell); }
// records of one op share their type and buffer bits
inline int run_key(const Rec &r) { return (r.type << 8) | (r.bits & (RB_SRC_BUF | RB_DST_BUF)); }

// A whole-block access of a block step: every cell of block `s & 0xff` whose
// distance to the block edge lies in [dlo, dhi] (FLUID cells only if
// fluid_only: the rho/u written by the step).
struct Whole {
  uint32_t s;       // kind<<8 | block
  bool fluid_only;
  uint8_t dlo, dhi;
  bool skip_cc = false;  // CF_CCPULL cells excluded (written by an NK_CCP node instead)
  bool skip_t = false;   // CF_TSKIP cells excluded (written by a spline instead)
  bool skip_fc = false;  // FLUID CF_FCSRC cells excluded (written by an NK_FCP node instead)
};
constexpr uint8_t DMAX = 255;

struct Access {
  std::unordered_set<uint64_t> r, w;
  std::vector<Whole> wr, ww;
  std::set<uint32_t> rs, ws;  // summaries of r / w keys and whole entries
  void read(uint64_t k) { r.insert(k); rs.insert(summ(k)); }
  void write(uint64_t k) { w.insert(k); ws.insert(summ(k)); }
  void read_whole(uint32_t s, uint8_t dlo = 0, uint8_t dhi = DMAX) { wr.push_back({s, false, dlo, dhi}); rs.insert(s); }
  void write_whole(uint32_t s, bool fo, uint8_t dlo = 0, uint8_t dhi = DMAX, bool skip_cc = false,
                   bool skip_t = false, bool skip_fc = false) {
    ww.push_back({s, fo, dlo, dhi, skip_cc, skip_t, skip_fc});
    ws.insert(s);
  }
  void merge(const Access &o) {
    for (auto k : o.r) r.insert(k);
    for (auto k : o.w) w.insert(k);
    wr.insert(wr.end(), o.wr.begin(), o.wr.end());
    ww.insert(ww.end(), o.ww.begin(), o.ww.end());
    rs.insert(o.rs.begin(), o.rs.end());
    ws.insert(o.ws.begin(), o.ws.end());
  }
};

bool sets_intersect(const std::set<uint32_t> &a, const std::set<uint32_t> &b) {
  auto i = a.begin();
  auto j = b.begin();
  while (i != a.end() && j != b.end()) {
    if (*i == *j) return true;
    if (*i < *j) ++i; else ++j;
  }
  return false;
}

// distance ranges [lo, hi] a block-step region reads and writes
void region_ranges(int region, uint8_t &rlo, uint8_t &rhi, uint8_t &wlo, uint8_t &whi) {
  if (region == STB_INTERIOR) { rlo = 1; rhi = DMAX; wlo = 2; whi = DMAX; }
  else if (region == STB_RIM) { rlo = 0; rhi = 2; wlo = 0; whi = 1; }
  else { rlo = 0; rhi = DMAX; wlo = 0; whi = DMAX; }
}

}  // namespace

// ---------------------------------------------------------------------------
// CF_MACRO marks: FLUID cells whose rho/ux/uy are read by c_c (source line),
// init_Spline3 (coarse line) or f_c (fine points).
// ---------------------------------------------------------------------------
static void mark_line(const mb_geometry &g, const std::vector<BlockLayout> &bl,
                      std::vector<std::vector<uint8_t>> &flags, int a, const mb_p4 &p, int n, int stride) {
  for (int ip = 0; ip < n; ip++) {
    int i, j;
    if (p.xstart == p.xend) { i = p.xstart; j = p.ystart + ip * stride; }
    else { i = p.xstart + ip * stride; j = p.ystart; }
    if (i < 0 || j < 0 || i >= bl[a].nx || j >= bl[a].ny) continue;
    flags[a][(size_t)j * bl[a].pitch + i] |= CF_MACRO;
  }
  (void)g;
}

void mark_macro_sources(const mb_geometry &g, const std::vector<BlockLayout> &bl,
                        std::vector<std::vector<uint8_t>> &flags) {
  const mb_layout &L = g.layout;
  for (int c = 0; c < L.number_line2; c++) {
    const mb_line &l = g.Line_Inf_CC[c];
    mark_line(g, bl, flags, l.areac_n, l.line_C, l.Nc, 1);
  }
  for (int b = 0; b < L.number_line; b++) {
    const mb_line &lc = g.Line_Inf_C[b];
    mark_line(g, bl, flags, lc.areac_n, lc.line_C, lc.Nc, 1);
    const mb_line &lf = g.Line_Inf_F[b];
    const int r = g.Areas[lf.areaf_n].m / g.Areas[lf.areac_n].m;
    mark_line(g, bl, flags, lf.areaf_n, lf.line_F, lf.Nc, r);
  }
}

void mark_fc_sources(const mb_geometry &g, const std::vector<BlockLayout> &bl,
                     std::vector<std::vector<uint8_t>> &flags) {
  const mb_layout &L = g.layout;
  for (size_t a = 0; a < flags.size(); a++)
    for (auto &f : flags[a])
      if ((f & 3) == CT_FLUID) f = uint8_t(f & ~CF_FCSRC);
  for (int b = 0; b < L.number_line; b++) {
    const mb_line &lf = g.Line_Inf_F[b];
    const int a = lf.areaf_n;
    const int r = g.Areas[a].m / g.Areas[lf.areac_n].m;
    for (int ip = 0; ip < lf.Nc; ip++) {
      int i, j;
      if (lf.line_C.xstart == lf.line_C.xend) { i = lf.line_F.xstart; j = lf.line_F.ystart + ip * r; }
      else { i = lf.line_F.xstart + ip * r; j = lf.line_F.ystart; }
      if (i < 0 || j < 0 || i >= bl[a].nx || j >= bl[a].ny) continue;
      uint8_t &f = flags[a][(size_t)j * bl[a].pitch + i];
      if ((f & (3 | CF_EDGE)) == CT_FLUID) f = uint8_t(f | CF_FCSRC);
    }
  }
}

// ---------------------------------------------------------------------------
// Same-level copies of each level with chains resolved (a copy whose source
// an earlier copy of the level wrote passes that copy's source on).  Copies
// from a FLUID source to a C_BOUNDARY target can run beside the block step
// (the target computes the source's new values; the step leaves C_BOUNDARY
// targets alone); the others stay point copies after the step: the rho/u a
// non-FLUID source carries may be written by an interface op between the
// step and the copy, and a FLUID target is the block step's own work.  A level is fusable when every copy stays within
// the level's first block-step launch (its first 16 blocks), no line reads a
// cell it writes, and no point copy reads a copy target.
// ---------------------------------------------------------------------------
std::vector<CcLevel> cc_levels(const mb_geometry &g, const std::vector<BlockLayout> &bl,
                               const std::vector<std::vector<uint8_t>> &flags) {
  const mb_layout &L = g.layout;
  std::vector<CcLevel> out(L.LEVEL);
  if (L.number_line2 == 0) return out;
  for (int level = 0; level < L.LEVEL; level++) {
    CcLevel &cl = out[level];
    std::map<std::pair<int, long long>, std::pair<int, long long>> src;  // target -> final source
    std::vector<std::pair<int, long long>> order;
    bool ok = true;
    for (int c = L.LCCP[level]; c < L.LCCP[level + 1]; c++) {
      const mb_line &l = g.Line_Inf_CC[c];
      const int A = l.areac_n, B = l.areaf_n;
      const int a0 = L.ASP[level], a1 = L.ASP[level + 1];
      // every copy of the level within the first launch chunk of 16 blocks
      if (A < a0 || A >= a1 || B < a0 || B >= a1 || A - a0 >= 16 || B - a0 >= 16 || A > 255 || B > 255) ok = false;
      std::set<std::pair<int, long long>> reads, writes;
      for (int ip = 0; ip < l.Nc && ok; ip++) {
        int i1 = 0, j1 = 0, i2 = 0, j2 = 0;  // c_c_boundary_transfer :20-33
        if (l.line_C.xstart == l.line_C.xend) { i1 = l.line_C.xstart; j1 = l.line_C.ystart + ip; i2 = l.line_F.xstart; j2 = l.line_F.ystart + ip; }
        if (l.line_C.ystart == l.line_C.yend) { i1 = l.line_C.xstart + ip; j1 = l.line_C.ystart; i2 = l.line_F.xstart + ip; j2 = l.line_F.ystart; }
        if (i1 < 0 || j1 < 0 || i1 >= bl[A].nx || j1 >= bl[A].ny || i2 < 0 || j2 < 0 || i2 >= bl[B].nx ||
            j2 >= bl[B].ny || i1 >= (1 << 28) || j1 >= (1 << 28)) {
          ok = false;
          break;
        }
        const std::pair<int, long long> sc{A, (long long)j1 * bl[A].pitch + i1}, tc{B, (long long)j2 * bl[B].pitch + i2};
        reads.insert(sc);
        writes.insert(tc);
        auto it = src.find(sc);
        const std::pair<int, long long> fin = it != src.end() ? it->second : sc;
        if (!src.count(tc)) order.push_back(tc);
        src[tc] = fin;
      }
      for (auto &w : writes)
        if (reads.count(w)) ok = false;  // the reference's threads would race
    }
    for (auto &t : order) {
      const CcLink lk{t.first, src[t].first, t.second, src[t].second};
      if ((flags[lk.sblk][(size_t)lk.scell] & 3) == CT_FLUID && (flags[lk.tblk][(size_t)lk.tcell] & 3) == CT_COPY)
        cl.links.push_back(lk);
      else
        cl.rec_links.push_back(lk);
    }
    for (const CcLink &lk : cl.rec_links)
      if (src.count({lk.sblk, lk.scell})) ok = false;
    if ((int)cl.rec_links.size() > PLAN_MAX_REC_OPS) ok = false;
    cl.fusable = ok && !cl.links.empty();
  }
  return out;
}

// ---------------------------------------------------------------------------
// symbolic evolution (evolution.h:2-65)
// ---------------------------------------------------------------------------
static void emit(const mb_geometry &g, int level, SchedState &s, std::vector<Op> &ops, bool final_chain) {
  const mb_layout &L = g.layout;
  if (level == L.LEVEL) return;
  for (int i = 0; i < L.mi[level]; i++) {
    if (!(level == 0 || i == 0)) {
      for (int b = L.LTCFFCP[level]; b < L.LTCFFCP[level + 1]; b++) {
        Op o;
        o.kind = Op::TEMPORAL;
        o.line = b;
        o.level = level;
        o.xm = 1.0 * i / L.mi[level];
        o.parity = s.parity;
        o.mk = s.marker[b];
        ops.push_back(o);
      }
    }
    const bool last = final_chain && (i == L.mi[level] - 1);
    {
      Op o;
      o.kind = Op::STB;
      o.level = level;
      o.parity = s.parity;
      o.macro_all = last ? 1 : 0;
      ops.push_back(o);
      for (int a = L.ASP[level]; a < L.ASP[level + 1]; a++) s.parity[a] ^= 1;
    }
    if (L.number_line2 != 0) {
      for (int c = L.LCCP[level]; c < L.LCCP[level + 1]; c++) {
        Op o;
        o.kind = Op::CC;
        o.line = c;
        o.level = level;
        o.parity = s.parity;
        ops.push_back(o);
      }
    }
    if (level != L.LEVEL - 1) {
      for (int b = L.LS3CFFCP[level]; b < L.LS3CFFCP[level + 1]; b++) {
        Op o;
        o.kind = Op::SPL;
        o.line = b;
        o.level = level;
        o.parity = s.parity;
        o.mk = s.marker[b];
        ops.push_back(o);
        for (int p = 0; p < 3; p++) s.marker[b][p] = (s.marker[b][p] == 0) ? 2 : s.marker[b][p] - 1;
      }
    }
    emit(g, level + 1, s, ops, last);
    if (level != 0 && i == L.mi[level] - 1) {
      for (int b = L.LTCFFCP[level]; b < L.LTCFFCP[level + 1]; b++) {
        Op o;
        o.kind = Op::CF;
        o.line = b;
        o.level = level;
        o.parity = s.parity;
        o.mk = s.marker[b];
        ops.push_back(o);
        o.kind = Op::FC;
        ops.push_back(o);
      }
    }
  }
}

static inline void line_pt(const mb_p4 &p, int ip, int stride, int &i, int &j) {
  if (p.xstart == p.xend) { i = p.xstart; j = p.ystart + ip * stride; }
  else { i = p.xstart + ip * stride; j = p.ystart; }
}

// A spline of line b runs at the place of b's next temporal interpolation
// and does it too, when only ops of the fine level (its block steps and
// same-level copies, splines and other lines' temporal interpolations) lie
// between them.  None of those reads what the spline writes (slots of b,
// rho/u of b's fine edge points, C_BOUNDARY cells the fine step leaves
// alone) or writes what it reads (F and rho/u of coarse line cells), so the
// spline may move there; the temporal interpolation itself stays in place.
// The temporal launch before the fine step then leaves the fine chain.
static std::vector<Op> fuse_temporal(const std::vector<Op> &ops) {
  const int n = int(ops.size());
  std::vector<int> with(n, -1);
  std::vector<char> moved(n, 0);
  for (int ti = 0; ti < n; ti++) {
    const Op &t = ops[ti];
    if (t.kind != Op::TEMPORAL) continue;
    int si = ti - 1;
    for (; si >= 0; si--) {
      const Op &q = ops[si];
      if (q.kind == Op::SPL && q.line == t.line) break;
      const bool ok = q.kind == Op::SPL || ((q.kind == Op::STB || q.kind == Op::CC) && q.level == t.level) ||
                      (q.kind == Op::TEMPORAL && q.level == t.level && q.line != t.line);
      if (!ok) { si = -1; break; }
    }
    if (si < 0 || moved[si]) continue;
    with[ti] = si;
    moved[si] = 1;
  }
  std::vector<Op> out;
  out.reserve(n);
  for (int i = 0; i < n; i++) {
    if (moved[i]) continue;
    if (with[i] < 0) { out.push_back(ops[i]); continue; }
    Op f = ops[with[i]];
    f.tmp = 1;
    f.txm = ops[i].xm;
    f.tmk = ops[i].mk;
    f.tparity = ops[i].parity;
    out.push_back(f);
  }
  return out;
}

// The same fusion without moving the spline, for levels in early_levels
// (no same-level copies): the spline writes the interpolated values at its
// own place into the buffer the level's next block step will read, and the
// one block step of the level between them (the substep without an
// interpolation) leaves those edge cells alone (tskip) instead of copying
// its input there.  The spline then runs beside that block step.
static std::vector<Op> fuse_early(const std::vector<Op> &ops, unsigned levels) {
  const int n = int(ops.size());
  std::vector<int> with(n, -1), stb_of(n, -1);
  std::vector<char> used(n, 0);
  for (int ti = 0; ti < n; ti++) {
    const Op &t = ops[ti];
    if (t.kind != Op::TEMPORAL || !((levels >> t.level) & 1u)) continue;
    int si = ti - 1, stb = -1, nstb = 0;
    for (; si >= 0; si--) {
      const Op &q = ops[si];
      if (q.kind == Op::SPL && q.line == t.line) break;
      if (q.kind == Op::STB && q.level == t.level) { stb = si; nstb++; continue; }
      const bool ok = q.kind == Op::SPL || (q.kind == Op::TEMPORAL && q.level == t.level && q.line != t.line);
      if (!ok) { si = -1; break; }
    }
    if (si < 0 || used[si] || nstb != 1) continue;
    with[si] = ti;
    used[si] = 1;
    stb_of[ti] = stb;
  }
  // all or none of a run of interpolations (lines may share corner cells,
  // whose last writer must stay the last line of the run), with the splines
  // in the order of the interpolations
  std::vector<int> from(n, -1);
  for (int i = 0; i < n; i++)
    if (with[i] >= 0) from[with[i]] = i;
  for (int t0 = 0; t0 < n;) {
    if (ops[t0].kind != Op::TEMPORAL) { t0++; continue; }
    int t1 = t0;
    while (t1 < n && ops[t1].kind == Op::TEMPORAL && ops[t1].level == ops[t0].level) t1++;
    bool all = true;
    for (int t = t0; t < t1; t++) all = all && from[t] >= 0 && (t == t0 || from[t] > from[t - 1]);
    if (!all)
      for (int t = t0; t < t1; t++)
        if (from[t] >= 0) {
          with[from[t]] = -1;
          used[from[t]] = 0;
          stb_of[t] = -1;
          from[t] = -1;
        }
    t0 = t1;
  }
  std::vector<char> drop(n, 0), skip(n, 0);
  for (int i = 0; i < n; i++)
    if (with[i] >= 0) {
      drop[with[i]] = 1;
      skip[stb_of[with[i]]] = 1;
    }
  std::vector<Op> out;
  out.reserve(n);
  for (int i = 0; i < n; i++) {
    if (drop[i]) continue;
    Op o = ops[i];
    if (with[i] >= 0) {
      const Op &t = ops[with[i]];
      o.tmp = 1;
      o.txm = t.xm;
      o.tmk = t.mk;
      o.tparity = t.parity;
    }
    if (skip[i]) o.tskip = 1;
    out.push_back(std::move(o));
  }
  return out;
}

std::vector<Op> PlanCompiler::fused(const std::vector<Op> &ops) const {
  std::vector<Op> o = early_levels ? fuse_early(ops, early_levels) : ops;
  return fuse_tmp ? fuse_temporal(o) : o;
}

std::vector<PlanNode> PlanCompiler::compile(SchedState &s, int n_coarse, bool final_macros) const {
  std::vector<Op> ops;
  for (int n = 0; n < n_coarse; n++) emit(g, 0, s, ops, final_macros && n == n_coarse - 1);
  return build(fused(ops));
}

unsigned PlanCompiler::split_levels() const {
  const mb_layout &L = g.layout;
  unsigned m = 0;
  for (int l = 0; l < L.LEVEL; l++) {
    long long cells = 0;
    for (int a = L.ASP[l]; a < L.ASP[l + 1]; a++) cells += (long long)bl[a].nx * bl[a].ny;
    if (split_mask ? ((split_mask >> l) & 1u) != 0 : cells >= split_cells) m |= 1u << l;
  }
  return m;
}

// error_L2 runs in parts: the interiors of split levels (which only their
// block step writes, so the part runs beside the rest of the step and the
// next step's interior waits for nothing else), then one part per level (its
// rim when split, all its cells otherwise), so that each level's next step
// waits only for the part that reads its own cells.
std::vector<PlanNode> PlanCompiler::compile_diag(SchedState &s, int n_coarse) const {
  std::vector<Op> ops;
  const bool any_split = split_levels() != 0;
  for (int n = 0; n < n_coarse; n++) {
    const size_t first = ops.size();
    emit(g, 0, s, ops, true);
    if (fuse_tmp || early_levels) {
      std::vector<Op> step(ops.begin() + first, ops.end());
      ops.resize(first);
      for (Op &o : fused(step)) ops.push_back(std::move(o));
    }
    for (int part = any_split ? 0 : 1; part <= g.layout.LEVEL; part++) {
      Op o;
      o.kind = Op::L2;
      o.level = part;  // 0: interiors of split levels, 1 + l: the rest of level l
      o.line = n;
      o.parity = s.parity;
      ops.push_back(o);
    }
    Op o;
    o.kind = Op::DRAG;
    o.line = n;
    o.parity = s.parity;
    ops.push_back(o);
  }
  return build(ops);
}

std::vector<PlanNode> PlanCompiler::compile_single(int kind, int index, double xm, const SchedState &s) const {
  Op o;
  o.kind = Op::Kind(kind);
  o.parity = s.parity;
  if (kind == Op::STB) {
    o.level = index;
    o.macro_all = 1;
  } else {
    o.line = index;
    if (kind != Op::CC) o.mk = s.marker[index];
    o.xm = xm;
  }
  std::vector<Op> ops{o};
  return build(ops);
}

std::vector<PlanNode> PlanCompiler::build(const std::vector<Op> &ops) const {
  const mb_layout &L = g.layout;
  auto pitch_cell = [&](int a, int i, int j) -> long long { return (long long)j * bl[a].pitch + i; };
  auto is_fluid = [&](int a, long long cell) { return (flags[a][cell] & 3) == CT_FLUID; };
  auto edge_dist = [&](int a, long long cell) -> int {
    const int i = int(cell % bl[a].pitch), j = int(cell / bl[a].pitch);
    return std::min(std::min(i, j), std::min(bl[a].nx - 1 - i, bl[a].ny - 1 - j));
  };
  auto covers = [&](const Whole &wh, uint64_t k) {
    if (summ(k) != wh.s) return false;
    const int blk = int((k >> 48) & 0xff);
    const long long cell = (long long)(k & 0xffffffffffffull);
    const int d = edge_dist(blk, cell);
    if (d < wh.dlo || d > wh.dhi) return false;
    if (wh.skip_cc && (flags[blk][cell] & CF_CCPULL)) return false;
    if (wh.skip_t && (flags[blk][cell] & CF_TSKIP)) return false;
    if (wh.skip_fc && (flags[blk][cell] & (3 | CF_FCSRC)) == (CT_FLUID | CF_FCSRC)) return false;
    return !wh.fluid_only || is_fluid(blk, cell);
  };

  // CF_FCSRC cells of each block (the fine points of f_c lines that are FLUID
  // and off the block edge): what an NK_FCP node updates beside the step
  std::vector<std::vector<long long>> fcsrc(L.number_area);
  if (fuse_fc) {
    for (int b = 0; b < L.number_line; b++) {
      const mb_line &lf = g.Line_Inf_F[b];
      const int a = lf.areaf_n;
      const int r = g.Areas[a].m / g.Areas[lf.areac_n].m;
      for (int ip = 0; ip < lf.Nc; ip++) {
        int i, j;
        if (lf.line_C.xstart == lf.line_C.xend) { i = lf.line_F.xstart; j = lf.line_F.ystart + ip * r; }
        else { i = lf.line_F.xstart + ip * r; j = lf.line_F.ystart; }
        if (i < 0 || j < 0 || i >= bl[a].nx || j >= bl[a].ny) continue;
        const long long cell = pitch_cell(a, i, j);
        if ((flags[a][(size_t)cell] & (3 | CF_FCSRC)) == (CT_FLUID | CF_FCSRC)) fcsrc[a].push_back(cell);
      }
    }
    for (auto &v : fcsrc) {
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
    }
  }

  // One write of an op (the F part or the M part of a record, or the rho/u
  // write of a spline point) with the reads it needs.
  struct Part {
    int node, idx;
    uint8_t bit;  // RB_WRITE_F / RB_WRITE_M of record idx, or 0: spline mask entry idx
    uint64_t wkey;
    std::vector<uint64_t> rkeys;
    bool live = true;
    bool fc = false;  // an f_c point done by block-step node `node` (its fc entry idx)
  };
  struct OpInfo {
    bool stb = false;
    bool cc_fused = false;      // STB: its level's same-level copies run beside it (cc_nodes)
    bool tskip = false;         // STB: leaves CF_TSKIP cells alone
    std::vector<int> stb_nodes; // STB: its nodes
    std::vector<int> cc_nodes;  // STB: NK_CCP nodes, one per launch chunk with copies
    std::vector<int> fc_nodes;  // STB: NK_FCP node of each launch chunk with CF_FCSRC cells (-1: none)
    int diag = -1;              // SNAP / DRAG / L2 op: its Op::Kind
    int level = -1;
    std::vector<int> parity;
    std::vector<Part> parts;
    std::vector<uint64_t> always_r, always_w;  // spline: gathered cells / written slot
    int node = -1;
    Access ac;            // point accesses of a line op (records, splines)
    bool has_ac = false;
  };
  std::vector<OpInfo> info(ops.size());
  std::vector<PlanNode> nodes;
  std::vector<Access> acc;  // forward (unpruned) sets: used only to decide batching
  int open = -1;
  int last_stb = -1;  // latest STB op; same-level copies right after it can fuse into it
  bool open_after_stb = false;  // the open launch's ops touch blocks of the latest step's level
  // Reads of a C_BOUNDARY cell's F that no op has written since its block's
  // last step may read the step's input buffer instead: the step copies
  // C_BOUNDARY cells unchanged, so both buffers hold the same value there,
  // and the read no longer conflicts with a later write of the cell.  An f_c
  // read of a cell whose latest write is a c_f record takes the value from
  // that record's slot instead (REC_FC_SLOT), for the same reason.
  std::vector<int> stb_op(L.number_area, -1);  // op index of each block's latest step
  struct LastWrite {
    int op;
    int line = -1, slot = 0, marker = 0;  // c_f writes: where the value comes from
  };
  std::unordered_map<uint64_t, LastWrite> lastw;  // F key -> its latest point write
  auto src_buf = [&](int b, int p, long long cell) -> int {
    const uint8_t f = flags[b][(size_t)cell];
    if ((f & 3) != CT_COPY || (f & CF_CCPULL) || stb_op[b] < 0) return p;
    auto it = lastw.find(fkey(p, b, cell));
    return (it == lastw.end() || it->second.op < stb_op[b]) ? p ^ 1 : p;
  };

  // NK_FCP node that can do f_c point (fine cell cf of block Fb, coarse
  // target in block Cb; keys of its reads and writes) for op oi, or -1: the
  // fine block's latest step updates cf (an off-edge FLUID cell whose rho/u
  // it writes), and no op since that step writes what the point reads or
  // touches what it writes.  The node updates the step's CF_FCSRC cells
  // beside it (the step leaves them alone) and then does its points.
  auto level_of = [&](int a) {
    for (int l = 0; l < L.LEVEL; l++)
      if (a >= L.ASP[l] && a < L.ASP[l + 1]) return l;
    return -1;
  };
  auto fc_host = [&](size_t oi, int Fb, int Cb, long long cf, uint64_t kSF, uint64_t kSM, uint64_t kDF,
                     uint64_t kDM) -> int {
    const int so = stb_op[Fb];
    if (!fuse_fc || so < 0 || !((fc_levels >> level_of(Fb)) & 1u)) return -1;
    const uint8_t f = flags[Fb][(size_t)cf];
    if ((f & (3 | CF_EDGE | CF_FCSRC | CF_MACRO)) != (CT_FLUID | CF_FCSRC | CF_MACRO)) return -1;
    const int lf = level_of(Fb), lc = level_of(Cb);
    for (size_t q = size_t(so) + 1; q < oi; q++) {
      const OpInfo &Q = info[q];
      if (Q.stb) {
        if (ops[q].level == lf || ops[q].level == lc) return -1;
        continue;
      }
      if (Q.diag >= 0) return -1;
      if (!Q.has_ac) {  // same-level copies run beside their step: targets are C_BOUNDARY cells of their level
        if (ops[q].level == lc || ops[q].level == lf) return -1;
        continue;
      }
      if (Q.ac.w.count(kSF) || Q.ac.w.count(kSM) || Q.ac.w.count(kDF) || Q.ac.w.count(kDM) || Q.ac.r.count(kDF) ||
          Q.ac.r.count(kDM))
        return -1;
    }
    const OpInfo &S = info[so];
    const size_t chunk = size_t((Fb - L.ASP[lf]) / 16);
    if (chunk >= S.fc_nodes.size() || S.fc_nodes[chunk] < 0) return -1;
    const int q = S.fc_nodes[chunk];
    if (nodes[q].fc.empty())  // first point: the chunk's step nodes leave the CF_FCSRC cells to it
      for (int sn : S.stb_nodes)
        if (nodes[sn].a0 == nodes[q].a0) nodes[sn].fcskip = 1;
    return q;
  };

  // ---- forward: expand ops into records and batch them ---------------------
  for (size_t oi = 0; oi < ops.size(); oi++) {
    const Op &o = ops[oi];
    OpInfo &I = info[oi];
    if (o.kind == Op::DRAG || o.kind == Op::L2) {
      open = -1;
      I.diag = int(o.kind);
      I.parity = o.parity;
      PlanNode nd;
      nd.kind = o.kind == Op::DRAG ? NK_DRAG : NK_L2;
      nd.level = o.line;
      if (o.kind == Op::L2) {
        nd.region = o.level == 0 ? STB_INTERIOR : STB_RIM;
        nd.part = o.level;
        nd.a0 = int(split_levels());
      }
      for (int a = 0; a < L.number_area; a++)
        if (o.parity[a]) nd.parity |= (1ull << a);
      nd.label = o.kind == Op::DRAG ? "drag" : (o.level == 0 ? "l2 int" : "l2");
      I.node = int(nodes.size());
      nodes.push_back(nd);
      acc.push_back(Access());
      continue;
    }
    if (o.kind == Op::STB) {
      open = -1;
      last_stb = int(oi);
      for (int a = L.ASP[o.level]; a < L.ASP[o.level + 1]; a++) stb_op[a] = int(oi);
      if (o.tskip) {  // cells it leaves alone: no read may take them from its input buffer
        I.tskip = true;
        for (int a = L.ASP[o.level]; a < L.ASP[o.level + 1]; a++)
          for (int j = 0; j < bl[a].ny; j++)
            for (int i = 0; i < bl[a].nx; i++) {
              const long long cell = pitch_cell(a, i, j);
              if (flags[a][(size_t)cell] & CF_TSKIP) lastw[fkey(o.parity[a] ^ 1, a, cell)] = LastWrite{int(oi)};
            }
      }
      I.stb = true;
      I.level = o.level;
      I.parity = o.parity;
      const bool split = ((split_levels() >> o.level) & 1u) != 0;
      for (int a0 = L.ASP[o.level]; a0 < L.ASP[o.level + 1]; a0 += 16) {
        const int a1 = std::min(L.ASP[o.level + 1], a0 + 16);
        for (int region : split ? std::vector<int>{STB_RIM, STB_INTERIOR} : std::vector<int>{STB_ALL}) {
          PlanNode nd;
          nd.kind = NK_STB;
          nd.level = o.level;
          nd.macro_all = o.macro_all;
          nd.region = region;
          for (int a = a0; a < a1; a++)
            if (o.parity[a]) nd.parity |= (1ull << a);
          char lab[64];
          std::snprintf(lab, sizeof lab, "stb L%d a%d-%d %s", o.level, a0, a1 - 1,
                        region == STB_RIM ? "rim" : (region == STB_INTERIOR ? "int" : ""));
          nd.label = lab;
          nd.a0 = a0;
          nd.a1 = a1;
          nd.tskip = o.tskip;
          I.stb_nodes.push_back(int(nodes.size()));
          nodes.push_back(nd);
          acc.push_back(Access());
        }
        int fcn = -1;  // the chunk's NK_FCP node, used only if an f_c point fuses into it
        bool any = false;
        for (int a = a0; a < a1; a++) any = any || !fcsrc[a].empty();
        if (fuse_fc && any) {
          PlanNode nd;
          nd.kind = NK_FCP;
          nd.level = o.level;
          nd.macro_all = o.macro_all;
          nd.a0 = a0;
          nd.a1 = a1;
          for (int a = a0; a < a1; a++)
            if (o.parity[a]) nd.parity |= (1ull << a);
          nd.label = "fcp L" + std::to_string(o.level);
          fcn = int(nodes.size());
          nodes.push_back(nd);
          acc.push_back(Access());
        }
        I.fc_nodes.push_back(fcn);
      }
      continue;
    }
    bool cc_points = false;  // this op carries the point copies of a fused level
    if (o.kind == Op::CC && cc && (*cc)[o.level].fusable && last_stb >= 0 && ops[last_stb].level == o.level) {
      bool adjacent = true;  // only same-level copies of this level since the block step
      for (size_t q = size_t(last_stb) + 1; q < oi; q++)
        if (ops[q].kind != Op::CC || ops[q].level != o.level) adjacent = false;
      const bool first = !info[last_stb].cc_fused;
      if (adjacent && first) {
        OpInfo &S = info[last_stb];
        S.cc_fused = true;
        for (int q : S.stb_nodes) {
          nodes[q].ccpull = 1;
          bool any = false;
          for (const CcLink &lk : (*cc)[o.level].links) any |= lk.tblk >= nodes[q].a0 && lk.tblk < nodes[q].a1;
          if (!any || nodes[q].region == STB_INTERIOR) continue;  // one copy node per chunk
          bool have = false;
          for (int c2 : S.cc_nodes) have |= nodes[c2].a0 == nodes[q].a0;
          if (have) continue;
          PlanNode nd;
          nd.kind = NK_CCP;
          nd.level = o.level;
          nd.a0 = nodes[q].a0;
          nd.a1 = nodes[q].a1;
          nd.parity = nodes[q].parity;
          nd.label = "ccp L" + std::to_string(o.level);
          S.cc_nodes.push_back(int(nodes.size()));
          nodes.push_back(nd);
          acc.push_back(Access());
        }
      }
      if (adjacent) {
        if (!first || (*cc)[o.level].rec_links.empty())
          continue;  // I.node stays -1: the copies have no node of their own
        cc_points = true;
      }
    }
    Access ac;
    std::vector<Rec> recs;
    struct RP { uint64_t wF, wM; std::vector<uint64_t> rF, rM; };
    std::vector<RP> rparts;
    std::vector<uint64_t> spl_wM;
    std::vector<uint64_t> tmp_w, tmp_r;  // fused temporal: F writes of the fine edge, slot reads
    SplTask task{};
    const bool is_spl = (o.kind == Op::SPL);
    double tw[3] = {0, 0, 0};

    if (cc_points) {
      // the level's copies from non-FLUID sources, each its own one-point op
      for (const CcLink &lk : (*cc)[o.level].rec_links) {
        const int pA = src_buf(lk.sblk, o.parity[lk.sblk], lk.scell), pB = o.parity[lk.tblk];
        Rec r{};
        r.type = REC_CC;
        r.bits = uint8_t((pA ? RB_SRC_BUF : 0) | (pB ? RB_DST_BUF : 0) | RB_WRITE_F | RB_WRITE_M);
        r.dst_block = uint8_t(lk.tblk);
        r.src_block = uint8_t(lk.sblk);
        r.dst_cell = int32_t(lk.tcell);
        r.src = int32_t(lk.scell);
        recs.push_back(r);
        rparts.push_back({fkey(pB, lk.tblk, lk.tcell), key(RK_M, lk.tblk, lk.tcell), {fkey(pA, lk.sblk, lk.scell)},
                          {key(RK_M, lk.sblk, lk.scell)}});
      }
    } else if (o.kind == Op::CC) {
      const mb_line &l = g.Line_Inf_CC[o.line];
      const int A = l.areac_n, B = l.areaf_n;
      const int pB = o.parity[B];
      for (int ip = 0; ip < l.Nc; ip++) {
        int i1 = 0, j1 = 0, i2 = 0, j2 = 0;
        if (l.line_C.xstart == l.line_C.xend) { i1 = l.line_C.xstart; j1 = l.line_C.ystart + ip; i2 = l.line_F.xstart; j2 = l.line_F.ystart + ip; }
        if (l.line_C.ystart == l.line_C.yend) { i1 = l.line_C.xstart + ip; j1 = l.line_C.ystart; i2 = l.line_F.xstart + ip; j2 = l.line_F.ystart; }
        const long long c1 = pitch_cell(A, i1, j1), c2 = pitch_cell(B, i2, j2);
        const int pA = src_buf(A, o.parity[A], c1);
        Rec r{};
        r.type = REC_CC;
        r.bits = uint8_t((pA ? RB_SRC_BUF : 0) | (pB ? RB_DST_BUF : 0) | RB_WRITE_F | RB_WRITE_M);
        r.dst_block = uint8_t(B);
        r.src_block = uint8_t(A);
        r.dst_cell = int32_t(c2);
        r.src = int32_t(c1);
        recs.push_back(r);
        rparts.push_back({fkey(pB, B, c2), key(RK_M, B, c2), {fkey(pA, A, c1)}, {key(RK_M, A, c1)}});
      }
    } else if (o.kind == Op::TEMPORAL || o.kind == Op::CF) {
      const mb_line &l = g.Line_Inf_C[o.line];
      const int Fb = l.areaf_n, pF = o.parity[Fb];
      const SplLine &sl = spl_lines[o.line];
      std::vector<uint64_t> sr;
      if (o.kind == Op::TEMPORAL) {
        const double xm = o.xm;
        tw[0] = 0.5 * (xm - 1.0) * xm;
        tw[1] = (xm - 1.0) * (xm + 1.0);
        tw[2] = 0.5 * xm * (xm + 1.0);
        for (int p = 0; p < 3; p++) sr.push_back(key(RK_SLOT, o.line, o.mk[p]));
      } else {
        sr.push_back(key(RK_SLOT, o.line, o.mk[2]));
      }
      for (int ip = 0; ip < l.Nf; ip++) {
        int i, j;
        line_pt(l.line_F, ip, 1, i, j);
        const long long c = pitch_cell(Fb, i, j);
        Rec r{};
        r.type = (o.kind == Op::TEMPORAL) ? REC_TEMPORAL : REC_CF;
        r.bits = uint8_t((pF ? RB_DST_BUF : 0) | RB_WRITE_F);
        r.dst_block = uint8_t(Fb);
        r.src_block = uint8_t(Fb);
        r.m0 = uint8_t(o.mk[0]);
        r.m1 = uint8_t(o.mk[1]);
        r.m2 = uint8_t(o.mk[2]);
        r.dst_cell = int32_t(c);
        r.src = sl.slot0 + ip;
        recs.push_back(r);
        rparts.push_back({fkey(pF, Fb, c), ~0ull, sr, {}});
      }
    } else if (o.kind == Op::FC) {
      const mb_line &l = g.Line_Inf_F[o.line];
      const int Cb = l.areac_n, Fb = l.areaf_n;
      const int pC = o.parity[Cb];
      const int r = g.Areas[Fb].m / g.Areas[Cb].m;
      for (int ip = 0; ip < l.Nc; ip++) {
        int ic, jc, i_f, j_f;
        if (l.line_C.xstart == l.line_C.xend) { ic = l.line_C.xstart; jc = l.line_C.ystart + ip; i_f = l.line_F.xstart; j_f = l.line_F.ystart + r * ip; }
        else { ic = l.line_C.xstart + ip; jc = l.line_C.ystart; i_f = l.line_F.xstart + r * ip; j_f = l.line_F.ystart; }
        const long long cc = pitch_cell(Cb, ic, jc), cf = pitch_cell(Fb, i_f, j_f);
        const int pF = src_buf(Fb, o.parity[Fb], cf);
        Rec rr{};
        rr.type = REC_FC;
        rr.bits = uint8_t((pF ? RB_SRC_BUF : 0) | (pC ? RB_DST_BUF : 0) | RB_WRITE_F | RB_WRITE_M);
        rr.dst_block = uint8_t(Cb);
        rr.src_block = uint8_t(Fb);
        rr.dst_cell = int32_t(cc);
        rr.src = int32_t(cf);
        uint64_t rF = fkey(pF, Fb, cf);
        auto lw = lastw.find(fkey(o.parity[Fb], Fb, cf));
        if (lw != lastw.end() && lw->second.line >= 0 && lw->second.op > stb_op[Fb] && lw->second.slot < (1 << 24)) {
          rr.type = REC_FC_SLOT;
          rr.m0 = uint8_t(lw->second.slot & 0xff);
          rr.m1 = uint8_t((lw->second.slot >> 8) & 0xff);
          rr.pad = uint8_t((lw->second.slot >> 16) & 0xff);
          rr.m2 = uint8_t(lw->second.marker);
          rF = key(RK_SLOT, lw->second.line, lw->second.marker);
        }
        const uint64_t kDF = fkey(pC, Cb, cc), kDM = key(RK_M, Cb, cc), kSF = rF, kSM = key(RK_M, Fb, cf);
        const int sn = rr.type == REC_FC ? fc_host(oi, Fb, Cb, cf, kSF, kSM, kDF, kDM) : -1;
        if (sn >= 0) {  // done by the fine level's last block step
          FcFuse e{};
          e.src_block = Fb;
          e.src_cell = int(cf);
          e.dst_block = Cb;
          e.dst_cell = int(cc);
          e.bits = RB_WRITE_F | RB_WRITE_M;
          e.dst_buf = uint8_t(pC);
          e.para = (double)(g.Areas[Fb].m / g.Areas[Cb].m) * (g.Areas[Cb].tau - 1.0) / (g.Areas[Fb].tau - 1.0);
          const int idx = int(nodes[sn].fc.size());
          nodes[sn].fc.push_back(e);
          Part pf{sn, idx, RB_WRITE_F, kDF, {kSF, kSM}};
          pf.fc = true;
          Part pm{sn, idx, RB_WRITE_M, kDM, {kSM}};
          pm.fc = true;
          I.parts.push_back(pf);
          I.parts.push_back(pm);
          lastw[kDF] = LastWrite{int(oi)};
          ac.read(kSF);
          ac.read(kSM);
          ac.write(kDF);
          ac.write(kDM);
          continue;
        }
        recs.push_back(rr);
        rparts.push_back({kDF, kDM, {rF, kSM}, {kSM}});
      }
    } else if (is_spl) {
      const mb_line &l = g.Line_Inf_C[o.line];
      const int Cb = l.areac_n, Fb = l.areaf_n, pC = o.parity[Cb];
      for (int ip = 0; ip < l.Nc; ip++) {
        int i, j;
        line_pt(l.line_C, ip, 1, i, j);
        const long long c = pitch_cell(Cb, i, j);
        I.always_r.push_back(fkey(pC, Cb, c));
        I.always_r.push_back(key(RK_M, Cb, c));
      }
      for (int ip = 0; ip < l.Nf; ip++) {
        int i, j;
        line_pt(l.line_F, ip, 1, i, j);
        spl_wM.push_back(key(RK_M, Fb, pitch_cell(Fb, i, j)));
      }
      I.always_w.push_back(key(RK_SLOT, o.line, o.mk[0]));
      task.line = o.line;
      task.src_buf = pC;
      task.m0 = o.mk[0];
      task.mask_off = -1;
      if (o.tmp) {  // the fused temporal interpolation: F of every fine edge point
        const double xm = o.txm;
        task.tmp = 1;
        task.tbuf = o.tparity[Fb];
        task.tw[0] = 0.5 * (xm - 1.0) * xm;
        task.tw[1] = (xm - 1.0) * (xm + 1.0);
        task.tw[2] = 0.5 * xm * (xm + 1.0);
        std::vector<uint64_t> sr;
        for (int q = 0; q < 3; q++) {
          task.tm[q] = o.tmk[q];
          sr.push_back(key(RK_SLOT, o.line, o.tmk[q]));
        }
        for (int ip = 0; ip < l.Nf; ip++) {
          int i, j;
          line_pt(l.line_F, ip, 1, i, j);
          tmp_w.push_back(fkey(task.tbuf, Fb, pitch_cell(Fb, i, j)));
        }
        tmp_r = sr;
      }
    }
    for (size_t q = 0; q < rparts.size(); q++) {
      if (rparts[q].wF == ~0ull) continue;
      LastWrite w{int(oi)};
      if (recs[q].type == REC_CF) {
        w.line = o.line;
        w.slot = recs[q].src;
        w.marker = o.mk[2];
      }
      lastw[rparts[q].wF] = w;
    }
    for (auto k : tmp_w) lastw[k] = LastWrite{int(oi)};
    for (auto &rp : rparts) {
      for (auto k : rp.rF) ac.read(k);
      for (auto k : rp.rM) ac.read(k);
      if (rp.wF != ~0ull) ac.write(rp.wF);
      if (rp.wM != ~0ull) ac.write(rp.wM);
    }
    for (auto k : I.always_r) ac.read(k);
    for (auto k : I.always_w) ac.write(k);
    for (auto k : spl_wM) ac.write(k);
    for (auto k : tmp_w) ac.write(k);
    for (auto k : tmp_r) ac.read(k);
    I.ac = ac;
    I.has_ac = true;
    if (!is_spl && recs.empty()) continue;  // every point runs inside a block step (f_c fused)

    const NodeKind want = is_spl ? NK_SPL : NK_REC;
    // whether this op touches a block the latest block step updated: a launch
    // mixing ops that wait for that step with ops that do not would hold the
    // latter back (a temporal interpolation of the coarser level behind the
    // finer level's c_f, say)
    bool after_stb = false;
    if (last_stb >= 0 && split_waits) {
      const int ls = ops[last_stb].level;
      auto hits = [&](uint64_t k) {
        const uint64_t kind = k >> 56;
        if (kind != RK_F0 && kind != RK_F1 && kind != RK_M) return false;
        const int a = int((k >> 48) & 0xff);
        return a >= L.ASP[ls] && a < L.ASP[ls + 1];
      };
      for (auto k : ac.r) after_stb = after_stb || hits(k);
      for (auto k : ac.w) after_stb = after_stb || hits(k);
    }
    bool join = (open >= 0 && nodes[open].kind == want && open_after_stb == after_stb);
    int nruns = 0;
    // a run of records shares type and buffer bits and is affine in the point
    // index (an f_c line whose points partly moved into an NK_FCP node has gaps)
    auto breaks = [&](size_t q0, size_t q) {
      if (cc_points || run_key(recs[q]) != run_key(recs[q0]) || recs[q].type == REC_FC_SLOT ||
          recs[q0].type == REC_FC_SLOT)
        return true;
      if (q - q0 < 2) return false;
      const long long dd = (long long)recs[q0 + 1].dst_cell - recs[q0].dst_cell,
                      ds = (long long)recs[q0 + 1].src - recs[q0].src;
      return (long long)recs[q].dst_cell - recs[q - 1].dst_cell != dd || (long long)recs[q].src - recs[q - 1].src != ds;
    };
    if (want == NK_REC) {
      nruns = recs.empty() ? 0 : 1;
      for (size_t q = 1, q0 = 0; q < recs.size(); q++)
        if (breaks(q0, q)) {
          nruns++;
          q0 = q;
        }
    }
    if (join && want == NK_REC && int(nodes[open].ops.size()) + nruns > PLAN_MAX_REC_OPS) join = false;
    if (join && want == NK_SPL && int(nodes[open].spl.size()) >= PLAN_MAX_SPL_TASKS) join = false;
    if (join && want == NK_REC && o.kind == Op::TEMPORAL) {
      const PlanNode &nd = nodes[open];
      bool found = false;
      for (int t = 0; t < nd.ntw; t++)
        if (nd.tw[t][0] == tw[0] && nd.tw[t][1] == tw[1] && nd.tw[t][2] == tw[2]) found = true;
      if (!found && nd.ntw >= 4) join = false;
    }
    if (join) {
      // a launch runs its points concurrently: no point may read what another writes
      const Access &B = acc[open];
      for (auto k : ac.r)
        if (B.w.count(k)) { join = false; break; }
      if (join)
        for (auto k : ac.w)
          if (B.r.count(k)) { join = false; break; }
    }
    if (!join) {
      PlanNode nd;
      nd.kind = want;
      nd.label = is_spl ? "spl" : "rec";
      nodes.push_back(nd);
      acc.push_back(Access());
      open = int(nodes.size()) - 1;
      open_after_stb = after_stb;
    }
    PlanNode &nd = nodes[open];
    I.node = open;
    if (want == NK_REC) {
      int widx = 0;
      if (o.kind == Op::TEMPORAL) {
        widx = -1;
        for (int t = 0; t < nd.ntw; t++)
          if (nd.tw[t][0] == tw[0] && nd.tw[t][1] == tw[1] && nd.tw[t][2] == tw[2]) widx = t;
        if (widx < 0) {
          widx = nd.ntw++;
          nd.tw[widx][0] = tw[0];
          nd.tw[widx][1] = tw[1];
          nd.tw[widx][2] = tw[2];
        }
      }
      if (cc_points) {
        for (size_t q = 0; q < recs.size(); q++) nd.ops.push_back({int(nd.recs.size() + q), 1});
      } else {  // runs of records with the same type and buffer bits (each run is affine)
        size_t q0 = 0;
        for (size_t q = 1; q <= recs.size(); q++)
          if (q == recs.size() || breaks(q0, q)) {
            nd.ops.push_back({int(nd.recs.size() + q0), int(q - q0)});
            q0 = q;
          }
      }
      for (size_t q = 0; q < recs.size(); q++) {
        Rec r = recs[q];
        r.bits |= uint8_t(widx << RB_WIDX_SHIFT);
        const int idx = int(nd.recs.size());
        nd.recs.push_back(r);
        const RP &rp = rparts[q];
        I.parts.push_back({open, idx, RB_WRITE_F, rp.wF, rp.rF});
        if (rp.wM != ~0ull) I.parts.push_back({open, idx, RB_WRITE_M, rp.wM, rp.rM});
      }
    } else {
      task.mask_off = int(nd.spl_mask.size());
      for (size_t q = 0; q < spl_wM.size(); q++) {
        I.parts.push_back({open, task.mask_off + int(q), 0, spl_wM[q], {}});
        nd.spl_mask.push_back(1);
      }
      if (task.tmp) {
        task.tmask_off = int(nd.spl_mask.size());
        for (size_t q = 0; q < tmp_w.size(); q++) {
          I.parts.push_back({open, task.tmask_off + int(q), 0, tmp_w[q], tmp_r});
          nd.spl_mask.push_back(1);
        }
      }
      nd.spl.push_back(task);
    }
    acc[open].merge(ac);
  }

  // ---- backward liveness: drop writes overwritten before any read ----------
  // state of a key = kind of its nearest later access (true: a write).  Keys
  // never touched later are read (the state after the plan is observable).
  // Block steps set the state of whole regions (layers, newest last); point
  // accesses override single keys until a newer layer covers them.
  struct Layer {
    Whole w;
    bool write;
  };
  struct SummState {
    std::vector<Layer> layers;
    std::unordered_map<uint64_t, bool> ov;
  };
  std::unordered_map<uint32_t, SummState> st;
  auto state_of = [&](uint64_t k) -> bool {
    auto it = st.find(summ(k));
    if (it == st.end()) return false;
    auto o2 = it->second.ov.find(k);
    if (o2 != it->second.ov.end()) return o2->second;
    for (auto l = it->second.layers.rbegin(); l != it->second.layers.rend(); ++l)
      if (covers(l->w, k)) return l->write;
    return false;
  };
  auto set_state = [&](uint64_t k, bool w) { st[summ(k)].ov[k] = w; };
  auto apply_layer = [&](const Whole &wh, bool write) {
    SummState &ss = st[wh.s];
    for (auto it = ss.ov.begin(); it != ss.ov.end();) {
      if (covers(wh, it->first)) it = ss.ov.erase(it);
      else ++it;
    }
    ss.layers.push_back({wh, write});
  };
  for (int oi = int(ops.size()) - 1; oi >= 0; oi--) {
    OpInfo &I = info[oi];
    if (I.diag == Op::L2) {  // reads rho/u of the cells of its part
      const PlanNode &nd = nodes[I.node];
      for (int l = 0; l < L.LEVEL; l++) {
        const bool sp = (nd.a0 >> l) & 1;
        if (nd.part == 0 ? !sp : l != nd.part - 1) continue;
        const uint8_t lo = nd.part == 0 ? 2 : 0, hi = (nd.part != 0 && sp) ? 1 : DMAX;
        for (int a = L.ASP[l]; a < L.ASP[l + 1]; a++) apply_layer({uint32_t((RK_M << 8) | a), false, lo, hi}, false);
      }
      continue;
    }
    if (I.diag == Op::DRAG) {  // reads the buffer the drag block's last step read
      const int a = drag_area, p = I.parity[a] ^ 1;
      apply_layer({uint32_t(((p ? RK_F1 : RK_F0) << 8) | a), false, 0, DMAX}, false);
      continue;
    }
    if (I.stb) {
      // the op's nodes together write F of buffer 1-p and rho/u of FLUID
      // cells and read F of buffer p, over the whole block; CF_FCSRC cells of
      // chunks with a used NK_FCP node are that node's
      auto fcp_used = [&](int a) {
        const size_t chunk = size_t((a - L.ASP[I.level]) / 16);
        return chunk < I.fc_nodes.size() && I.fc_nodes[chunk] >= 0 && !nodes[I.fc_nodes[chunk]].fc.empty();
      };
      for (int a = L.ASP[I.level]; a < L.ASP[I.level + 1]; a++) {
        const int p = I.parity[a];
        const bool fs = fcp_used(a);
        apply_layer({uint32_t(((p ? RK_F0 : RK_F1) << 8) | a), false, 0, DMAX, I.cc_fused, I.tskip, fs}, true);
        apply_layer({uint32_t((RK_M << 8) | a), true, 0, DMAX, I.cc_fused, false, fs}, true);
        apply_layer({uint32_t(((p ? RK_F1 : RK_F0) << 8) | a), false, 0, DMAX}, false);
        if (fs)
          for (long long cell : fcsrc[a]) {
            set_state(fkey(p ^ 1, a, cell), true);
            set_state(key(RK_M, a, cell), true);
          }
      }
      if (I.cc_fused)  // the copies beside the step write F and rho/u of their targets
        for (const CcLink &lk : (*cc)[I.level].links) {
          set_state(fkey(I.parity[lk.tblk] ^ 1, lk.tblk, lk.tcell), true);
          set_state(key(RK_M, lk.tblk, lk.tcell), true);
        }
      continue;
    }
    for (Part &pt : I.parts) pt.live = !state_of(pt.wkey);
    for (Part &pt : I.parts)
      if (pt.live) set_state(pt.wkey, true);
    for (auto k : I.always_w) set_state(k, true);
    for (Part &pt : I.parts)
      if (pt.live)
        for (auto k : pt.rkeys) set_state(k, false);
    for (auto k : I.always_r) set_state(k, false);
    for (Part &pt : I.parts) {
      if (pt.live) continue;
      PlanNode &nd = nodes[pt.node];
      if (pt.fc) nd.fc[pt.idx].bits &= uint8_t(~pt.bit);
      else if (pt.bit) nd.recs[pt.idx].bits &= uint8_t(~pt.bit);
      else nd.spl_mask.at(pt.idx) = 0;
    }
  }

  // ---- final access sets from the surviving parts -----------------------------
  std::vector<Access> fin(nodes.size());
  for (size_t q = 0; q < nodes.size(); q++) {
    if (nodes[q].kind != NK_STB) continue;
    uint8_t rlo, rhi, wlo, whi;
    region_ranges(nodes[q].region, rlo, rhi, wlo, whi);
    for (int a = nodes[q].a0; a < nodes[q].a1; a++) {
      const int p = int((nodes[q].parity >> a) & 1);
      fin[q].read_whole(uint32_t(((p ? RK_F1 : RK_F0) << 8) | a), rlo, rhi);
      fin[q].write_whole(uint32_t(((p ? RK_F0 : RK_F1) << 8) | a), false, wlo, whi, nodes[q].ccpull != 0,
                         nodes[q].tskip != 0, nodes[q].fcskip != 0);
      fin[q].write_whole(uint32_t((RK_M << 8) | a), true, wlo, whi, nodes[q].ccpull != 0, false,
                         nodes[q].fcskip != 0);
    }
  }
  for (size_t q = 0; q < nodes.size(); q++) {  // NK_FCP: the CF_FCSRC cells, pulled from the step's input
    if (nodes[q].kind != NK_FCP || nodes[q].fc.empty()) continue;
    for (int a = nodes[q].a0; a < nodes[q].a1; a++) {
      const int p = int((nodes[q].parity >> a) & 1);
      for (long long cell : fcsrc[a]) {
        fin[q].write(fkey(p ^ 1, a, cell));
        fin[q].write(key(RK_M, a, cell));
        for (int k = 0; k < 9; k++) {
          static const int EX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, EY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
          fin[q].read(fkey(p, a, cell - ((long long)EY[k] * bl[a].pitch + EX[k])));
        }
      }
    }
  }
  for (auto &I : info) {
    if (!I.stb || !I.cc_fused) continue;
    for (const CcLink &lk : (*cc)[I.level].links) {
      int q = -1;  // the copy node of the target's launch chunk
      for (int c2 : I.cc_nodes)
        if (lk.tblk >= nodes[c2].a0 && lk.tblk < nodes[c2].a1) q = c2;
      if (q < 0) continue;  // cannot happen: fusable levels keep each copy within one chunk
      Access &A = fin[q];
      A.write(fkey(I.parity[lk.tblk] ^ 1, lk.tblk, lk.tcell));
      A.write(key(RK_M, lk.tblk, lk.tcell));
      const int ps = I.parity[lk.sblk];  // buffer the step reads
      const BlockLayout &sb = bl[lk.sblk];
      const int si = int(lk.scell % sb.pitch), sj = int(lk.scell / sb.pitch);
      for (int k = 0; k < 9; k++) {
        static const int EX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, EY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
        const int ii = si - EX[k], jj = sj - EY[k];
        if (ii < 0 || jj < 0 || ii >= sb.nx || jj >= sb.ny) continue;
        A.read(fkey(ps, lk.sblk, (long long)jj * sb.pitch + ii));
      }
      A.read(fkey(ps, lk.sblk, lk.scell));  // sources are FLUID: their rho/u come from the pulled values
    }
  }
  for (auto &I : info) {
    if (I.diag < 0) continue;
    Access &A = fin[I.node];
    if (I.diag == Op::L2) {
      const PlanNode &nd = nodes[I.node];
      for (int l = 0; l < L.LEVEL; l++) {
        const bool sp = (nd.a0 >> l) & 1;
        if (nd.part == 0 ? !sp : l != nd.part - 1) continue;
        const uint8_t lo = nd.part == 0 ? 2 : 0, hi = (nd.part != 0 && sp) ? 1 : DMAX;
        for (int a = L.ASP[l]; a < L.ASP[l + 1]; a++) {
          A.read_whole(uint32_t((RK_M << 8) | a), lo, hi);
          A.read_whole(uint32_t((RK_UP << 8) | a), lo, hi);
          A.write_whole(uint32_t((RK_UP << 8) | a), false, lo, hi);
        }
      }
      A.write(key(RK_DIAG, 0, (1 + L2_NPARTS) * nd.level + 1 + nd.part));
    } else {
      const int a = drag_area, p = I.parity[a] ^ 1;
      A.read_whole(uint32_t(((p ? RK_F1 : RK_F0) << 8) | a));
      A.write(key(RK_DIAG, 0, (1 + L2_NPARTS) * nodes[I.node].level));
    }
  }
  for (auto &I : info) {
    if (I.stb || I.diag >= 0) continue;
    for (auto &pt : I.parts) {  // a fused f_c point belongs to its block-step node
      if (!pt.live) continue;
      Access &A = fin[pt.node];
      A.write(pt.wkey);
      for (auto k : pt.rkeys) A.read(k);
    }
    if (I.node < 0) continue;
    Access &A = fin[I.node];
    for (auto k : I.always_r) A.read(k);
    for (auto k : I.always_w) A.write(k);
  }
  // drop records with nothing left to write, and nodes with nothing to do
  std::vector<int> remap(nodes.size(), -1);
  std::vector<PlanNode> kept;
  std::vector<Access> kacc;
  for (size_t q = 0; q < nodes.size(); q++) {
    PlanNode &nd = nodes[q];
    if (nd.kind == NK_FCP && nd.fc.empty()) continue;  // no f_c point fused: its step updates the cells
    if (nd.kind == NK_REC) {
      // ops keep their point ranges (each is affine in the point index); an op
      // whose every write died is dropped whole
      std::vector<Rec> live;
      std::vector<std::pair<int, int>> ops;
      for (auto &op : nd.ops) {
        bool any = false;
        for (int r = op.first; r < op.first + op.second; r++) any |= (nd.recs[r].bits & (RB_WRITE_F | RB_WRITE_M)) != 0;
        if (!any) continue;
        ops.push_back({int(live.size()), op.second});
        live.insert(live.end(), nd.recs.begin() + op.first, nd.recs.begin() + op.first + op.second);
      }
      nd.recs.swap(live);
      nd.ops.swap(ops);
      if (nd.recs.empty()) continue;
    }
    remap[q] = int(kept.size());
    kept.push_back(std::move(nd));
    kacc.push_back(std::move(fin[q]));
  }
  nodes.swap(kept);
  acc.swap(kacc);

  // ---- DAG edges: every earlier node that conflicts with a later one ------
  const int n = int(nodes.size());
  auto whole_hits_keys = [&](const Whole &wh, const std::unordered_set<uint64_t> &keys) {
    for (auto k : keys)
      if (covers(wh, k)) return true;
    return false;
  };
  auto conflict = [&](const Access &p, const Access &q) {
    // quick reject on summaries
    const bool wr = sets_intersect(p.ws, q.rs), rw = sets_intersect(p.rs, q.ws), ww = sets_intersect(p.ws, q.ws);
    if (!wr && !rw && !ww) return false;
    auto cross = [&](const std::unordered_set<uint64_t> &a, const std::unordered_set<uint64_t> &b) {
      const auto &sm = a.size() < b.size() ? a : b;
      const auto &lg = a.size() < b.size() ? b : a;
      for (auto k : sm)
        if (lg.count(k)) return true;
      return false;
    };
    auto whole_vs = [&](const std::vector<Whole> &wa, const std::unordered_set<uint64_t> &kb,
                        const std::vector<Whole> &wb) {
      for (auto &x : wa) {
        for (auto &y : wb)
          if (x.s == y.s && x.dlo <= y.dhi && y.dlo <= x.dhi) return true;
        if (whole_hits_keys(x, kb)) return true;
      }
      return false;
    };
    if (wr && (cross(p.w, q.r) || whole_vs(p.ww, q.r, q.wr) || whole_vs(q.wr, p.w, {}))) return true;
    if (rw && (cross(p.r, q.w) || whole_vs(p.wr, q.w, q.ww) || whole_vs(q.ww, p.r, {}))) return true;
    if (ww && (cross(p.w, q.w) || whole_vs(p.ww, q.w, q.ww) || whole_vs(q.ww, p.w, {}))) return true;
    return false;
  };
  std::vector<std::vector<uint64_t>> reach(n, std::vector<uint64_t>((n + 63) / 64, 0));
  for (int q = 0; q < n; q++) {
    std::vector<int> direct;
    for (int p = q - 1; p >= 0; p--)
      if (conflict(acc[p], acc[q])) direct.push_back(p);
    // transitive reduction (direct is in descending order)
    for (int p : direct) {
      if (reach[q][p >> 6] & (1ull << (p & 63))) continue;
      nodes[q].deps.push_back(p);
      reach[q][p >> 6] |= 1ull << (p & 63);
      for (size_t w = 0; w < reach[q].size(); w++) reach[q][w] |= reach[p][w];
    }
    std::sort(nodes[q].deps.begin(), nodes[q].deps.end());
  }
  return nodes;
}

}  // namespace mblbm
