// host_geometry.cpp - block layouts, geo_init and coverage analysis (host only).
//
// Replaces the compile-time tables of geo/geometry.h and the host set-up of
// geo/init_geo.h in zhangya9741/Multi-block-LBM-GPU with runtime data.  The
// integer arithmetic of geo_init/Line_init is kept exactly (block extents,
// cumulative ratio m, per-level tau, line end points), because every later
// kernel indexes cells through these tables.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <set>
#include <string>
#include <vector>

#include "../../include/mblbm.h"
#include "mblbm_internal.h"

namespace {

void set_zone(mb_zone &z, double xs, double xe, double ys, double ye, int ml, int mr, int md, int mu) {
  z.reduced = {xs, xe, ys, ye};
  z.move = {ml, mr, md, mu};
}

// Tables of geo/geometry.h:7-147, one function per _GEO_* block.
void layout_1_1(mb_layout &L) {  // geometry.h:7-27
  L.LEVEL = 1;
  L.mi[0] = 1;
  L.number_area = 1;
  L.number_line = 0;
  L.number_line2 = 0;
  L.ASP[0] = 0; L.ASP[1] = 1;
  set_zone(L.AreaZone[0], 0.0, 1.0, 0.0, 1.0, 0, 0, 0, 0);
}

void layout_2_2(mb_layout &L) {  // geometry.h:29-53
  L.LEVEL = 2;
  L.mi[0] = 1; L.mi[1] = 2;
  L.number_area = 2;
  L.number_line = 1;
  L.number_line2 = 0;
  int asp[] = {0, 1, 2};
  std::memcpy(L.ASP, asp, sizeof(asp));
  set_zone(L.AreaZone[0], 0.0, 1.0, 0.0, 0.5, 0, 0, 0, 1);
  set_zone(L.AreaZone[1], 0.0, 1.0, 0.5, 1.0, 0, 0, 0, 0);
  int lt[] = {0, 0, 1}, ls[] = {0, 1, 1}, lc[] = {0, 0, 0};
  std::memcpy(L.LTCFFCP, lt, sizeof(lt));
  std::memcpy(L.LS3CFFCP, ls, sizeof(ls));
  std::memcpy(L.LCCP, lc, sizeof(lc));
  L.NeborCF[0] = {0, 1, 3};
}

void layout_2_5(mb_layout &L) {  // geometry.h:55-100
  L.LEVEL = 2;
  L.mi[0] = 1; L.mi[1] = 2;
  L.number_area = 5;
  L.number_line = 4;
  L.number_line2 = 8;
  int asp[] = {0, 4, 5};
  std::memcpy(L.ASP, asp, sizeof(asp));
  set_zone(L.AreaZone[0], 0.0, 1.0, 0.75, 1.0, 0, 0, -1, 0);
  set_zone(L.AreaZone[1], 0.0, 1.0, 0.0, 0.25, 0, 0, 0, 1);
  set_zone(L.AreaZone[2], 0.0, 0.25 - 0.0625, 0.25, 0.75, 0, 1, 0, 0);
  set_zone(L.AreaZone[3], 0.25 + 0.0625, 1.0, 0.25, 0.75, -1, 0, 0, 0);
  set_zone(L.AreaZone[4], 0.25 - 0.0625, 0.25 + 0.0625, 0.25, 0.75, 0, 0, 0, 0);
  int lt[] = {0, 0, 4}, ls[] = {0, 4, 4}, lc[] = {0, 8, 8};
  std::memcpy(L.LTCFFCP, lt, sizeof(lt));
  std::memcpy(L.LS3CFFCP, ls, sizeof(ls));
  std::memcpy(L.LCCP, lc, sizeof(lc));
  const mb_p3i cf[] = {{0, 4, 2}, {1, 4, 3}, {2, 4, 1}, {3, 4, 0}};
  std::memcpy(L.NeborCF, cf, sizeof(cf));
  const mb_p3i cc[] = {{0, 2, 2}, {2, 0, 2}, {0, 3, 2}, {3, 0, 2},
                       {1, 2, 3}, {2, 1, 3}, {1, 3, 3}, {3, 1, 3}};
  std::memcpy(L.NeborCC, cc, sizeof(cc));
}

void layout_4_9(mb_layout &L) {  // geometry.h:102-147
  L.LEVEL = 4;
  int mi[] = {1, 2, 2, 2};
  std::memcpy(L.mi, mi, sizeof(mi));
  L.number_area = 10;
  L.number_line = 17;
  L.number_line2 = 12;
  int asp[] = {0, 4, 6, 9, 10};
  std::memcpy(L.ASP, asp, sizeof(asp));
  const double z[10][4] = {{0.0, 0.1, 0, 1.0},      {0.1, 0.4, 0.75, 1.0},   {0.4, 1.0, 0.0, 1.0},
                           {0.1, 0.4, 0.0, 0.25},   {0.1, 0.15, 0.25, 0.75}, {0.35, 0.4, 0.25, 0.75},
                           {0.15, 0.25, 0.625, 0.75}, {0.25, 0.35, 0.25, 0.75}, {0.15, 0.25, 0.25, 0.375},
                           {0.15, 0.25, 0.375, 0.625}};
  const int mv[10][4] = {{0, 1, 0, 0}, {0, 0, -1, 0}, {-1, 0, 0, 0}, {0, 0, 0, 1}, {0, 1, 0, 0},
                         {-1, 0, 0, 0}, {0, 0, -1, 0}, {-1, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 0, 0}};
  for (int a = 0; a < 10; a++)
    set_zone(L.AreaZone[a], z[a][0], z[a][1], z[a][2], z[a][3], mv[a][0], mv[a][1], mv[a][2], mv[a][3]);
  int lt[] = {0, 0, 6, 13, 17}, ls[] = {0, 10, 14, 17, 17}, lc[] = {0, 8, 8, 12, 12};
  std::memcpy(L.LTCFFCP, lt, sizeof(lt));
  std::memcpy(L.LS3CFFCP, ls, sizeof(ls));
  std::memcpy(L.LCCP, lc, sizeof(lc));
  const mb_p3i cf[] = {{0, 4, 1}, {1, 4, 2}, {1, 5, 2}, {2, 5, 0}, {3, 5, 3}, {3, 4, 3},
                       {1, 6, 2}, {1, 7, 2}, {3, 7, 3}, {3, 8, 3},
                       {4, 6, 1}, {5, 7, 0}, {4, 8, 1},
                       {4, 9, 1},
                       {6, 9, 2}, {7, 9, 0}, {8, 9, 3}};
  std::memcpy(L.NeborCF, cf, sizeof(cf));
  const mb_p3i cc[] = {{0, 1, 1}, {1, 0, 1}, {2, 1, 0}, {1, 2, 0}, {2, 3, 0}, {3, 2, 0},
                       {0, 3, 1}, {3, 0, 1}, {7, 6, 0}, {6, 7, 0}, {7, 8, 0}, {8, 7, 0}};
  std::memcpy(L.NeborCC, cc, sizeof(cc));
}

// One rectangular block given in absolute coarse cells, stored as a zone
// with zero fractions and the coordinates in the integer move, so that
// (int)(0*(L-1)) + move reproduces them exactly.
void abs_zone(mb_zone &z, int xs, int xe, int ys, int ye) { set_zone(z, 0, 0, 0, 0, xs, xe, ys, ye); }

}  // namespace

extern "C" int mb_version(void) { return MB_ABI_VERSION; }

extern "C" const char *mb_error_string(int code) {
  switch (code) {
    case MB_OK: return "ok";
    case MB_ERR_INVALID: return "invalid argument";
    case MB_ERR_CUDA: return "CUDA runtime error";
    case MB_ERR_NOMEM: return "out of memory";
    case MB_ERR_GEOMETRY: return "invalid geometry";
    case MB_ERR_UNSUPPORTED: return "unsupported";
    case MB_ERR_NUMERIC: return "non-finite value in the state";
    case MB_ERR_TIMEOUT: return "device wait timed out";
    case MB_ERR_STATE: return "call out of order";
    case MB_ERR_NODEVICE: return "no usable CUDA device";
    default: return "unknown error";
  }
}

extern "C" int mb_layout_builtin(const char *name, mb_layout *out) {
  if (!name || !out) return MB_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  std::string n(name);
  if (n == "1_1") layout_1_1(*out);
  else if (n == "2_2") layout_2_2(*out);
  else if (n == "2_5") layout_2_5(*out);
  else if (n == "4_9") layout_4_9(*out);
  else return MB_ERR_INVALID;
  return MB_OK;
}

extern "C" int mb_layout_nested(int LX, int LY, int nlevels, const int *boxes, mb_layout *out) {
  if (!out || nlevels < 1 || nlevels > MB_MAX_LEVEL || LX < 4 || LY < 4) return MB_ERR_INVALID;
  if (nlevels > 1 && !boxes) return MB_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  mb_layout &L = *out;
  L.LEVEL = nlevels;
  // region of each level, in coarse cells
  std::vector<mb_p4> R(nlevels);
  R[0] = {0, LX - 1, 0, LY - 1};
  for (int l = 1; l < nlevels; l++) {
    const int *b = boxes + 4 * (l - 1);
    R[l] = {b[0], b[1], b[2], b[3]};
    const mb_p4 &o = R[l - 1];
    // a frame needs the inner box strictly inside with room for 1-cell overlaps
    if (R[l].xstart < o.xstart + 2 || R[l].xend > o.xend - 2 || R[l].ystart < o.ystart + 2 ||
        R[l].yend > o.yend - 2 || R[l].xend - R[l].xstart < 4 || R[l].yend - R[l].ystart < 4)
      return MB_ERR_GEOMETRY;
  }
  int a = 0;
  std::vector<int> first(nlevels);
  for (int l = 0; l < nlevels; l++) {
    L.mi[l] = (l == 0) ? 1 : 2;
    L.ASP[l] = a;
    first[l] = a;
    const mb_p4 &r = R[l];
    if (l == nlevels - 1) {
      abs_zone(L.AreaZone[a++], r.xstart, r.xend, r.ystart, r.yend);
    } else {
      const mb_p4 &b = R[l + 1];
      abs_zone(L.AreaZone[a++], r.xstart, r.xend, b.yend - 1, r.yend);        // top
      abs_zone(L.AreaZone[a++], r.xstart, r.xend, r.ystart, b.ystart + 1);    // bottom
      abs_zone(L.AreaZone[a++], r.xstart, b.xstart + 1, b.ystart, b.yend);    // left
      abs_zone(L.AreaZone[a++], b.xend - 1, r.xend, b.ystart, b.yend);        // right
    }
  }
  L.ASP[nlevels] = a;
  L.number_area = a;
  // coarse-fine lines, grouped by coarse level
  int nl = 0;
  for (int l = 0; l < nlevels - 1; l++) {
    L.LS3CFFCP[l] = nl;
    const int T = first[l], B = T + 1, Lf = T + 2, Rt = T + 3;
    if (l + 1 == nlevels - 1) {
      const int Fn = first[l + 1];
      L.NeborCF[nl++] = {T, Fn, 2};
      L.NeborCF[nl++] = {B, Fn, 3};
      L.NeborCF[nl++] = {Lf, Fn, 1};
      L.NeborCF[nl++] = {Rt, Fn, 0};
    } else {
      const int t = first[l + 1], b = t + 1, lf = t + 2, rt = t + 3;
      L.NeborCF[nl++] = {T, t, 2};
      L.NeborCF[nl++] = {B, b, 3};
      L.NeborCF[nl++] = {Lf, t, 1};
      L.NeborCF[nl++] = {Lf, b, 1};
      L.NeborCF[nl++] = {Lf, lf, 1};
      L.NeborCF[nl++] = {Rt, t, 0};
      L.NeborCF[nl++] = {Rt, b, 0};
      L.NeborCF[nl++] = {Rt, rt, 0};
    }
  }
  for (int l = nlevels - 1; l <= nlevels; l++) L.LS3CFFCP[l] = nl;
  L.number_line = nl;
  L.LTCFFCP[0] = 0;
  for (int l = 1; l <= nlevels; l++) L.LTCFFCP[l] = L.LS3CFFCP[l - 1];
  // same-level lines of every frame, as the pairs of geometry.h:94-99
  int nc = 0;
  for (int l = 0; l < nlevels; l++) {
    L.LCCP[l] = nc;
    if (l == nlevels - 1) continue;
    const int T = first[l], B = T + 1, Lf = T + 2, Rt = T + 3;
    const mb_p3i pairs[8] = {{T, Lf, 2}, {Lf, T, 2}, {T, Rt, 2}, {Rt, T, 2},
                             {B, Lf, 3}, {Lf, B, 3}, {B, Rt, 3}, {Rt, B, 3}};
    for (int p = 0; p < 8; p++) L.NeborCC[nc++] = pairs[p];
  }
  L.LCCP[nlevels] = nc;
  L.number_line2 = nc;
  return MB_OK;
}

namespace {
enum Dir { LEFT = 0, RIGHT = 1, DOWN = 2, UP = 3 };

// Overlap range of two extents along the line direction, in local cells of
// each block (init_geo.h:30-45 / :64-79): start at 0 when the other block
// begins at or before this one, else at (other.start - this.start)*m; end
// at n-1 when the other block reaches at least as far, else at
// (other.end - this.start)*m.
void overlap(int cs, int ce, int fs, int fe, int mC, int nC, int mF, int nF, int &c0, int &c1, int &f0,
             int &f1) {
  c0 = (fs - cs <= 0) ? 0 : (fs - cs) * mC;
  c1 = (fe - ce >= 0) ? nC - 1 : (fe - cs) * mC;
  f0 = (cs - fs <= 0) ? 0 : (cs - fs) * mF;
  f1 = (ce - fe >= 0) ? nF - 1 : (ce - fs) * mF;
}

// Line_init (geo/init_geo.h:17-86): the pair of transfer lines between a
// coarse block C and a fine block F lying in direction d of C.  lc: C-side
// source line (m_C cells inside C) and the F edge it feeds; lf: the C edge
// and the F interior line (m_F cells inside F) that feeds it.
void make_line_pair(int d, const mb_p4 &DC, const mb_area &C, const mb_p4 &DF, const mb_area &F, mb_line &lc,
                    mb_line &lf) {
  if (d == LEFT || d == RIGHT) {
    const int xc = (d == LEFT) ? C.m : C.nx - 1 - C.m;
    const int xf = (d == LEFT) ? F.nx - 1 : 0;
    const int xce = (d == LEFT) ? 0 : C.nx - 1;
    const int xfi = (d == LEFT) ? F.nx - F.m - 1 : F.m;
    int c0, c1, f0, f1;
    overlap(DC.ystart, DC.yend, DF.ystart, DF.yend, C.m, C.ny, F.m, F.ny, c0, c1, f0, f1);
    lc.line_C = {xc, xc, c0, c1};
    lc.line_F = {xf, xf, f0, f1};
    lf.line_C = {xce, xce, c0, c1};
    lf.line_F = {xfi, xfi, f0, f1};
  } else if (d == DOWN || d == UP) {
    const int yc = (d == DOWN) ? C.m : C.ny - 1 - C.m;
    const int yf = (d == DOWN) ? F.ny - 1 : 0;
    const int yce = (d == DOWN) ? 0 : C.ny - 1;
    const int yfi = (d == DOWN) ? F.ny - F.m - 1 : F.m;
    int c0, c1, f0, f1;
    overlap(DC.xstart, DC.xend, DF.xstart, DF.xend, C.m, C.nx, F.m, F.nx, c0, c1, f0, f1);
    lc.line_C = {c0, c1, yc, yc};
    lc.line_F = {f0, f1, yf, yf};
    lf.line_C = {c0, c1, yce, yce};
    lf.line_F = {f0, f1, yfi, yfi};
  } else {
    return;  // the reference leaves both lines untouched for other codes
  }
  const bool vertical = (d == LEFT || d == RIGHT);
  lc.Nc = vertical ? lc.line_C.yend - lc.line_C.ystart + 1 : lc.line_C.xend - lc.line_C.xstart + 1;
  lc.Nf = vertical ? lc.line_F.yend - lc.line_F.ystart + 1 : lc.line_F.xend - lc.line_F.xstart + 1;
  lf.Nc = lc.Nc;
  lf.Nf = lc.Nf;
}

// Drops the periodic ghost lines (MB_DIR_PERIODIC) of a layout that an
// earlier mb_geo_init produced, with the level ranges of LCCP.
void strip_periodic(mb_layout &L) {
  int lccp[MB_MAX_LEVEL + 1];
  std::memcpy(lccp, L.LCCP, sizeof(lccp));
  int n = 0;
  for (int c = 0; c < L.number_line2; c++) {
    if (L.NeborCC[c].direction == MB_DIR_PERIODIC) {
      for (int l = 0; l <= L.LEVEL; l++)
        if (lccp[l] > c) L.LCCP[l]--;
      continue;
    }
    L.NeborCC[n++] = L.NeborCC[c];
  }
  L.number_line2 = n;
}

// Point ip of a same-level line in the orientation c_c_boundary_transfer
// gives it (multi/FH/assit_multi.h:20-33): along y when the source segment
// is vertical, along x when it is horizontal (a single point is both).
void cc_point(const mb_line &l, int ip, int &i1, int &j1, int &i2, int &j2) {
  i1 = j1 = i2 = j2 = 0;
  if (l.line_C.xstart == l.line_C.xend) { i1 = l.line_C.xstart; j1 = l.line_C.ystart + ip; i2 = l.line_F.xstart; j2 = l.line_F.ystart + ip; }
  if (l.line_C.ystart == l.line_C.yend) { i1 = l.line_C.xstart + ip; j1 = l.line_C.ystart; i2 = l.line_F.xstart + ip; j2 = l.line_F.ystart; }
}

// Periodic ghost lines (no reference counterpart).  Every level-0 cell on a
// wrapped domain edge is a ghost of its image node one period (LX-2 or LY-2
// nodes) away; the cell that computes the image is the one level-0 cell at
// that node that is not C_BOUNDARY (the first block in index order where
// several are, as for equilibrium edge cells shared by two blocks).  Runs of
// ghosts along one block edge whose image cells are consecutive in one block
// become one copy line.  The layout's own level-0 lines lose the ghost cells
// at their ends, so that each ghost has one writer and no line reads a ghost.
// The new lines follow the level-0 lines of LCCP, entries MB_DIR_PERIODIC.
int periodic_lines(mb_geometry &g) {
  mb_layout &L = g.layout;
  const mb_config &c = g.config;
  const bool px = c.periodic & MB_PERIODIC_X, py = c.periodic & MB_PERIODIC_Y;
  if (L.mi[0] != 1 || (px && c.LX < 4) || (py && c.LY < 4)) return MB_ERR_GEOMETRY;
  for (int a = L.ASP[1]; a < L.number_area; a++) {  // finer blocks stay off wrapped edges
    const mb_p4 &D = g.AreaDefine[a];
    if ((px && (D.xstart <= 0 || D.xend >= c.LX - 1)) || (py && (D.ystart <= 0 || D.yend >= c.LY - 1)))
      return MB_ERR_GEOMETRY;
  }
  auto ghost = [&](int a, int i, int j) {
    const mb_area &A = g.Areas[a];
    return mblbm::periodic_ghost(c, i + A.base_x, j + A.base_y);
  };
  // the layout's level-0 lines without ghost targets
  for (int ln = L.LCCP[0]; ln < L.LCCP[1]; ln++) {
    mb_line &l = g.Line_Inf_CC[ln];
    auto tg = [&](int ip) {
      int i1, j1, i2, j2;
      cc_point(l, ip, i1, j1, i2, j2);
      return ghost(l.areaf_n, i2, j2);
    };
    int lo = 0, hi = l.Nc;
    while (lo < hi && tg(lo)) lo++;
    while (hi > lo && tg(hi - 1)) hi--;
    for (int ip = lo; ip < hi; ip++)
      if (tg(ip)) return MB_ERR_GEOMETRY;
    if (lo == 0 && hi == l.Nc) continue;
    if (hi - lo < 2) return MB_ERR_GEOMETRY;  // keeps the line's orientation
    int i1, j1, i2, j2;
    cc_point(l, lo, i1, j1, i2, j2);
    const bool vert = l.line_C.xstart == l.line_C.xend;
    const int n = hi - lo;
    l.line_C = vert ? mb_p4{i1, i1, j1, j1 + n - 1} : mb_p4{i1, i1 + n - 1, j1, j1};
    l.line_F = vert ? mb_p4{i2, i2, j2, j2 + n - 1} : mb_p4{i2, i2 + n - 1, j2, j2};
    l.Nc = l.Nf = n;
  }
  // ghost runs: rows j = 0 and ny-1, then columns i = 0 and nx-1 without the corners
  std::vector<mb_line> extra;
  for (int a = L.ASP[0]; a < L.ASP[1]; a++) {
    const mb_area &A = g.Areas[a];
    for (int e = 0; e < 4; e++) {
      const bool vert = e >= 2;
      const int n = vert ? A.ny - 2 : A.nx;
      bool open = false;
      mb_line cur{};
      int last_ip = 0;
      for (int ip = 0; ip < n; ip++) {
        const int i = vert ? (e == 2 ? 0 : A.nx - 1) : ip;
        const int j = vert ? ip + 1 : (e == 0 ? 0 : A.ny - 1);
        if (!ghost(a, i, j)) {
          if (open) extra.push_back(cur);
          open = false;
          continue;
        }
        if (mblbm::cell_type(g, a, i, j) != MB_C_BOUNDARY) return MB_ERR_GEOMETRY;
        const int X = i + (int)A.base_x, Y = j + (int)A.base_y;
        const int Xi = !px ? X : X == 0 ? c.LX - 2 : X == c.LX - 1 ? 1 : X;
        const int Yi = !py ? Y : Y == 0 ? c.LY - 2 : Y == c.LY - 1 ? 1 : Y;
        int owner = -1, oi = 0, oj = 0;
        for (int b = L.ASP[0]; b < L.ASP[1] && owner < 0; b++) {
          const mb_area &B = g.Areas[b];
          const int ii = Xi - (int)B.base_x, jj = Yi - (int)B.base_y;
          if (ii < 0 || jj < 0 || ii >= B.nx || jj >= B.ny) continue;
          if (mblbm::cell_type(g, b, ii, jj) == MB_C_BOUNDARY) continue;
          owner = b;
          oi = ii;
          oj = jj;
        }
        if (owner < 0) return MB_ERR_GEOMETRY;
        const bool extends = open && cur.areac_n == owner && ip == last_ip + 1 &&
                             (vert ? (oi == cur.line_C.xend && oj == cur.line_C.yend + 1)
                                   : (oj == cur.line_C.yend && oi == cur.line_C.xend + 1));
        if (extends) {
          cur.Nc++;
          cur.Nf++;
          cur.line_C.xend = oi;
          cur.line_C.yend = oj;
          cur.line_F.xend = i;
          cur.line_F.yend = j;
        } else {
          if (open) extra.push_back(cur);
          cur = mb_line{};
          cur.areac_n = owner;
          cur.areaf_n = a;
          cur.Nc = cur.Nf = 1;
          cur.line_C = {oi, oi, oj, oj};
          cur.line_F = {i, i, j, j};
          open = true;
        }
        last_ip = ip;
      }
      if (open) extra.push_back(cur);
    }
  }
  const int P = (int)extra.size(), at = L.LCCP[1];
  if (L.number_line2 + P > MB_MAX_LINE2) return MB_ERR_UNSUPPORTED;
  for (int q = L.number_line2 - 1; q >= at; q--) {
    g.Line_Inf_CC[q + P] = g.Line_Inf_CC[q];
    L.NeborCC[q + P] = L.NeborCC[q];
  }
  for (int p = 0; p < P; p++) {
    g.Line_Inf_CC[at + p] = extra[p];
    L.NeborCC[at + p] = {extra[p].areac_n, extra[p].areaf_n, MB_DIR_PERIODIC};
  }
  for (int l = 1; l <= L.LEVEL; l++) L.LCCP[l] += P;
  L.number_line2 += P;
  return MB_OK;
}

}  // namespace

extern "C" int mb_geo_init(const mb_layout *layout, const mb_config *cfg, mb_geometry *geo) {
  if (!layout || !cfg || !geo) return MB_ERR_INVALID;
  if (layout->LEVEL < 1 || layout->LEVEL > MB_MAX_LEVEL || layout->number_line2 < 0 ||
      layout->number_line2 > MB_MAX_LINE2)
    return MB_ERR_INVALID;
  mb_layout L = *layout;
  strip_periodic(L);
  if (L.LEVEL < 1 || L.LEVEL > MB_MAX_LEVEL || L.number_area < 1 || L.number_area > MB_MAX_AREA ||
      L.number_line < 0 || L.number_line > MB_MAX_LINE || L.number_line2 < 0 || L.number_line2 > MB_MAX_LINE2 ||
      (L.number_line2 & 1))
    return MB_ERR_INVALID;
  if (L.ASP[0] != 0 || L.ASP[L.LEVEL] != L.number_area) return MB_ERR_INVALID;
  for (int l = 0; l < L.LEVEL; l++) {
    if (L.mi[l] < 1 || L.ASP[l + 1] < L.ASP[l]) return MB_ERR_INVALID;
    if (L.LTCFFCP[l] < 0 || L.LTCFFCP[l + 1] > L.number_line || L.LS3CFFCP[l + 1] > L.number_line ||
        L.LCCP[l + 1] > L.number_line2)
      return MB_ERR_INVALID;
  }
  for (int b = 0; b < L.number_line; b++)
    if (L.NeborCF[b].nc < 0 || L.NeborCF[b].nc >= L.number_area || L.NeborCF[b].nf < 0 ||
        L.NeborCF[b].nf >= L.number_area)
      return MB_ERR_INVALID;
  for (int c = 0; c < L.number_line2; c++)
    if (L.NeborCC[c].nc < 0 || L.NeborCC[c].nc >= L.number_area || L.NeborCC[c].nf < 0 ||
        L.NeborCC[c].nf >= L.number_area)
      return MB_ERR_INVALID;
  if (cfg->Re <= 0 || cfg->LX < 2 || cfg->LY < 2) return MB_ERR_INVALID;
  if (cfg->periodic & ~(MB_PERIODIC_X | MB_PERIODIC_Y)) return MB_ERR_INVALID;

  mb_geometry &g = *geo;
  std::memset(&g, 0, sizeof(g));
  g.layout = L;
  g.config = *cfg;
  // block extents in coarse cells (init_geo.h:91-97)
  for (int a = 0; a < L.number_area; a++) {
    const mb_zone &z = L.AreaZone[a];
    g.AreaDefine[a].xstart = (int)(z.reduced.xstart * (cfg->LX - 1)) + z.move.xstart;
    g.AreaDefine[a].xend = (int)(z.reduced.xend * (cfg->LX - 1)) + z.move.xend;
    g.AreaDefine[a].ystart = (int)(z.reduced.ystart * (cfg->LY - 1)) + z.move.ystart;
    g.AreaDefine[a].yend = (int)(z.reduced.yend * (cfg->LY - 1)) + z.move.yend;
  }
  // per-level ratio and relaxation time (init_geo.h:99-119): nu from the
  // cylinder diameter, tau_l = 0.5 + mi_l (tau_{l-1} - 0.5)
  const double u0 = std::sqrt(cfg->U0[0] * cfg->U0[0] + cfg->U0[1] * cfg->U0[1]);
  const double nu = u0 * 2 * cfg->R / cfg->Re;
  double tau = 0.5 + 3.0 * nu;
  int m = 1;
  for (int l = 0; l < L.LEVEL; l++) {
    m *= L.mi[l];
    tau = 0.5 + L.mi[l] * (tau - 0.5);
    for (int a = L.ASP[l]; a < L.ASP[l + 1]; a++) {
      mb_area &A = g.Areas[a];
      A.m = m;
      A.nx = (g.AreaDefine[a].xend - g.AreaDefine[a].xstart) * m + 1;
      A.ny = (g.AreaDefine[a].yend - g.AreaDefine[a].ystart) * m + 1;
      A.base_x = g.AreaDefine[a].xstart;
      A.base_y = g.AreaDefine[a].ystart;
      A.tau = tau;
      A.rv_tau = 1.0 / tau;
      if (A.nx < 2 || A.ny < 2) return MB_ERR_GEOMETRY;
    }
  }
  for (int b = 0; b < L.number_line; b++) {
    const int c = L.NeborCF[b].nc, f = L.NeborCF[b].nf;
    g.Line_Inf_C[b].areac_n = g.Line_Inf_F[b].areac_n = c;
    g.Line_Inf_C[b].areaf_n = g.Line_Inf_F[b].areaf_n = f;
    make_line_pair(L.NeborCF[b].direction, g.AreaDefine[c], g.Areas[c], g.AreaDefine[f], g.Areas[f],
                   g.Line_Inf_C[b], g.Line_Inf_F[b]);
  }
  for (int i = 0; i + 1 < L.number_line2; i += 2) {
    const int c = L.NeborCC[i].nc, f = L.NeborCC[i].nf;
    mb_line &l0 = g.Line_Inf_CC[i], &l1 = g.Line_Inf_CC[i + 1];
    l0.areac_n = c;
    l0.areaf_n = f;
    make_line_pair(L.NeborCC[i].direction, g.AreaDefine[c], g.Areas[c], g.AreaDefine[f], g.Areas[f], l0, l1);
    // the reverse line of a pair copies B's interior into A's edge: its
    // source and target swap places (init_geo.h:148-158)
    l1.areac_n = L.NeborCC[i + 1].nc;
    l1.areaf_n = L.NeborCC[i + 1].nf;
    std::swap(l1.line_C, l1.line_F);
  }
  if (cfg->periodic) return periodic_lines(g);
  return MB_OK;
}

// ---------------------------------------------------------------------------
// Cell flags and coverage (used by the plan compiler and by the check below).
// ---------------------------------------------------------------------------
namespace mblbm {

bool obstacle_contains(const mb_config &c, double x, double y) {
  if (c.obstacle == MB_OBST_NONE) return false;
  if (c.obstacle == MB_OBST_ELLIPSE) {
    const double dx = x - c.ell_cx, dy = y - c.ell_cy;
    const double ca = std::cos(c.ell_angle), sa = std::sin(c.ell_angle);
    const double xr = ca * dx + sa * dy, yr = -sa * dx + ca * dy;
    return (xr * xr) / (c.ell_a * c.ell_a) + (yr * yr) / (c.ell_b * c.ell_b) < 1.0;
  }
  // init_block.h:28; x, y are dyadic so the FP64 sum is exact
  return (x - c.CX) * (x - c.CX) + (y - c.CY) * (y - c.CY) < c.R * c.R;
}

// A node on an edge of the domain that mb_config.periodic wraps: a ghost of
// the node one period away (no reference counterpart).
bool periodic_ghost(const mb_config &c, double x, double y) {
  return ((c.periodic & MB_PERIODIC_X) && (x == 0.0 || x == c.LX - 1.0)) ||
         ((c.periodic & MB_PERIODIC_Y) && (y == 0.0 || y == c.LY - 1.0));
}

// Cell type of init_General (lbm/init_block.h:28-42): solid inside the
// obstacle, FLUID on the physical domain edge (FP64 coordinate equality),
// C_BOUNDARY on any other block edge, FLUID inside.  Periodic domain edges
// are C_BOUNDARY: their cells are ghosts filled by copy lines.
int cell_type(const mb_geometry &g, int a, int i, int j) {
  const mb_area &A = g.Areas[a];
  const double dx = 1.0 / A.m;
  const double x = i * dx + A.base_x, y = j * dx + A.base_y;
  const mb_config &c = g.config;
  if (obstacle_contains(c, x, y)) return MB_SOLID_SBB;
  if (periodic_ghost(c, x, y)) return MB_C_BOUNDARY;
  if (y == 0.0 || y == c.LY - 1.0 || x == 0.0 || x == c.LX - 1.0) return MB_FLUID;
  if (i == 0 || j == 0 || i == A.nx - 1 || j == A.ny - 1) return MB_C_BOUNDARY;
  return MB_FLUID;
}

}  // namespace mblbm

extern "C" int mb_geo_check_coverage(const mb_geometry *geo, int *n_uncovered) {
  if (!geo || !n_uncovered) return MB_ERR_INVALID;
  const mb_geometry &g = *geo;
  const mb_layout &L = g.layout;
  std::set<std::pair<int, long long>> written;
  auto add_line = [&](int a, const mb_p4 &p, int n, int stride) {
    for (int ip = 0; ip < n; ip++) {
      int i, j;
      if (p.xstart == p.xend) { i = p.xstart; j = p.ystart + ip * stride; }
      else { i = p.xstart + ip * stride; j = p.ystart; }
      written.insert({a, (long long)j * g.Areas[a].nx + i});
    }
  };
  for (int c = 0; c < L.number_line2; c++) {
    const mb_line &l = g.Line_Inf_CC[c];
    add_line(l.areaf_n, l.line_F, l.Nc, 1);
  }
  for (int b = 0; b < L.number_line; b++) {
    add_line(g.Line_Inf_C[b].areaf_n, g.Line_Inf_C[b].line_F, g.Line_Inf_C[b].Nf, 1);
    add_line(g.Line_Inf_F[b].areac_n, g.Line_Inf_F[b].line_C, g.Line_Inf_F[b].Nc, 1);
  }
  int miss = 0;
  for (int a = 0; a < L.number_area; a++) {
    const mb_area &A = g.Areas[a];
    for (int j = 0; j < A.ny; j++)
      for (int i = 0; i < A.nx; i++) {
        if (i != 0 && j != 0 && i != A.nx - 1 && j != A.ny - 1) continue;
        if (mblbm::cell_type(g, a, i, j) != MB_C_BOUNDARY) continue;
        if (!written.count({a, (long long)j * A.nx + i})) miss++;
      }
  }
  *n_uncovered = miss;
  return MB_OK;
}

extern "C" int mb_append_drag(const char *path, int t, double cd, double cl) {
  if (!path) return MB_ERR_INVALID;
  FILE *fp = std::fopen(path, "a");
  if (!fp) return MB_ERR_INVALID;
  std::fprintf(fp, "%d\t%g\t%g\t\n", t, cd, cl);  // force_block.h:212-215
  std::fclose(fp);
  return MB_OK;
}

extern "C" int mb_append_error_L2(const char *path, int t, double e) {
  if (!path) return MB_ERR_INVALID;
  FILE *fp = std::fopen(path, "a");
  if (!fp) return MB_ERR_INVALID;
  std::fprintf(fp, "%d\t%g\n", t, e);  // error_L2.h:85-88
  std::fclose(fp);
  return MB_OK;
}
