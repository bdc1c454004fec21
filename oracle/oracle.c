/*
 * oracle.c - FP64 CPU restatement of the reference multi-block D2Q9 step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): the product library never links,
 * loads or calls this file.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py use it.
 *
 * Each function below restates one reference function of
 * zhangya9741/Multi-block-LBM-GPU (cited file:line) in plain C, keeping the
 * FP64 operation order of the reference expressions, the structure-of-arrays
 * layout (ixy = i + j*nx) and the quirks listed at each function.  OpenMP
 * parallelises loops whose iterations are independent in the reference too,
 * so results do not depend on the thread count.
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define Q 9
#define BLOCKX 16   /* _BLOCKX, parameters.h:9  */
#define BLOCKY 16   /* _BLOCKY, parameters.h:10 */
#define BLOCK1D 256 /* _BLOCK_1D, parameters.h:11 */

/* D2Q9 tables, lbm/lbm.h:43-45 */
static const double Wt[Q] = {4. / 9, 1. / 9, 1. / 9, 1. / 9, 1. / 9, 1. / 36, 1. / 36, 1. / 36, 1. / 36};
static const int Ev[2 * Q] = {0, 1, 0, -1, 0, 1, -1, -1, 1, 0, 0, 1, 0, -1, 1, 1, -1, -1};
static const int Opp[Q] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const int Slip[Q] = {0, 1, 4, 3, 2, 8, 7, 6, 5}; /* slip_gpu, lbm/lbm.h:51 */
/* MRT moment matrix M_gpu (lbm/lbm.h:53-63); its rows are orthogonal with
 * squared norms Mn, so M^-1 = M^T diag(1/Mn) (the exact form of InvM_gpu,
 * lbm/lbm.h:64-75) */
static const int Mm[Q][Q] = {{1, 1, 1, 1, 1, 1, 1, 1, 1},   {-4, -1, -1, -1, -1, 2, 2, 2, 2},
                             {4, -2, -2, -2, -2, 1, 1, 1, 1}, {0, 1, 0, -1, 0, 1, -1, -1, 1},
                             {0, -2, 0, 2, 0, 1, -1, -1, 1},  {0, 0, 1, 0, -1, 1, 1, -1, -1},
                             {0, 0, -2, 0, 2, 1, 1, -1, -1},  {0, 1, -1, 1, -1, 0, 0, 0, 0},
                             {0, 0, 0, 0, 0, 1, -1, 1, -1}};
static const double Mn[Q] = {9, 36, 36, 6, 12, 6, 12, 4, 4};

typedef struct {
  int *solid;
  double *x, *y, *rho, *ux, *uy, *forcex, *forcey;
  double *f[Q];
  double *F[Q];
} o_d2q9; /* D2Q9, lbm/data_type_lbm.h:7-14 */

typedef struct {
  int N;
  int marker[3];
  double *F[3][Q]; /* f_t1, f_t, f_t_1 (multi/data_type_multi.h:24-30) */
} o_fstore;

typedef struct {
  int N;
  double *l, *m, *u, *Varibs_M;
  double *rho, *ux, *uy;
  double *F[Q];
} o_spline; /* FM_spline3, multi/data_type_multi.h:7-13 */

struct orc_sim {
  mb_geometry geo;
  o_d2q9 pp[MB_MAX_AREA];
  double *upx[MB_MAX_AREA], *upy[MB_MAX_AREA];
  o_fstore t3[MB_MAX_LINE];
  o_spline s3[MB_MAX_LINE];
  int drag_area;
  int n_drag;
  int *drag; /* 3 * n_drag: i, j, k */
  double U0_2;
  /* collision options: 0 BGK, 1 MRT with rates s_e, s_eps, s_q (<= 0: the
   * block's 1/tau); shear rates are always the block's 1/tau */
  int coll;
  double s_e, s_eps, s_q;
  double fx, fy;                /* uniform body force on every cell's forcex/forcey */
  int *types[MB_MAX_AREA];      /* cell-type overrides, applied after init_General */
  int n_pfill;                  /* periodic ghosts: 4 ints each, ghost block/cell, image block/cell */
  int *pfill;
};

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* feq, lbm/assit_func.h:2-9 */
double orc_feq(int k, double rh, double uxx, double uyy) {
  double eu, uv, feq0;
  eu = Ev[k] * uxx + Ev[k + Q] * uyy;
  uv = uxx * uxx + uyy * uyy;
  feq0 = Wt[k] * rh * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uv);
  return feq0;
}

/* Macros, lbm/assit_func.h:23-31 */
static inline void macros(double *rh, double *uxx, double *uyy, const double *ft) {
  *rh = ft[0] + ft[1] + ft[2] + ft[3] + ft[4] + ft[5] + ft[6] + ft[7] + ft[8];
  *uxx = ft[1] - ft[3] + ft[5] - ft[6] - ft[7] + ft[8];
  *uyy = ft[2] - ft[4] + ft[5] + ft[6] - ft[7] - ft[8];
  *uxx = *uxx / *rh;
  *uyy = *uyy / *rh;
}

/* ---------------------------------------------------------------------------
 * Geometry: Line_init (geo/init_geo.h:17-86) and geo_init (:89-165)
 * ------------------------------------------------------------------------- */
static void line_init(int Direction, const mb_p4 *aD_C, const mb_area *aC, mb_line *lC,
                      const mb_p4 *aD_F, const mb_area *aF, mb_line *lF) {
  if (Direction == 0 || Direction == 1) {
    lC->line_C.xstart = (Direction == 0 ? aC->m : aC->nx - 1 - aC->m);
    lC->line_C.xend = lC->line_C.xstart;
    lC->line_F.xstart = (Direction == 0 ? aF->nx - 1 : 0);
    lC->line_F.xend = lC->line_F.xstart;
    lF->line_C.xstart = (Direction == 0 ? 0 : aC->nx - 1);
    lF->line_C.xend = lF->line_C.xstart;
    lF->line_F.xstart = (Direction == 0 ? aF->nx - aF->m - 1 : aF->m);
    lF->line_F.xend = lF->line_F.xstart;

    lC->line_C.ystart = (aD_F->ystart - aD_C->ystart <= 0) ? 0 : (aD_F->ystart - aD_C->ystart) * aC->m;
    lC->line_C.yend = (aD_F->yend - aD_C->yend >= 0) ? aC->ny - 1 : (aD_F->yend - aD_C->ystart) * aC->m;
    lC->line_F.ystart = (aD_C->ystart - aD_F->ystart <= 0) ? 0 : (aD_C->ystart - aD_F->ystart) * aF->m;
    lC->line_F.yend = (aD_C->yend - aD_F->yend >= 0) ? aF->ny - 1 : (aD_C->yend - aD_F->ystart) * aF->m;
    lF->line_C.ystart = lC->line_C.ystart;
    lF->line_C.yend = lC->line_C.yend;
    lF->line_F.ystart = lC->line_F.ystart;
    lF->line_F.yend = lC->line_F.yend;
    lC->Nc = lC->line_C.yend - lC->line_C.ystart + 1;
    lC->Nf = lC->line_F.yend - lC->line_F.ystart + 1;
    lF->Nc = lC->Nc;
    lF->Nf = lC->Nf;
  } else if (Direction == 2 || Direction == 3) {
    lC->line_C.ystart = (Direction == 2 ? aC->m : aC->ny - 1 - aC->m);
    lC->line_C.yend = lC->line_C.ystart;
    lC->line_F.ystart = (Direction == 2 ? aF->ny - 1 : 0);
    lC->line_F.yend = lC->line_F.ystart;
    lF->line_C.ystart = (Direction == 2 ? 0 : aC->ny - 1);
    lF->line_C.yend = lF->line_C.ystart;
    lF->line_F.ystart = (Direction == 2 ? aF->ny - aF->m - 1 : aF->m);
    lF->line_F.yend = lF->line_F.ystart;

    lC->line_C.xstart = (aD_F->xstart - aD_C->xstart <= 0) ? 0 : (aD_F->xstart - aD_C->xstart) * aC->m;
    lC->line_C.xend = (aD_F->xend - aD_C->xend >= 0) ? aC->nx - 1 : (aD_F->xend - aD_C->xstart) * aC->m;
    lC->line_F.xstart = (aD_C->xstart - aD_F->xstart <= 0) ? 0 : (aD_C->xstart - aD_F->xstart) * aF->m;
    lC->line_F.xend = (aD_C->xend - aD_F->xend >= 0) ? aF->nx - 1 : (aD_C->xend - aD_F->xstart) * aF->m;
    lF->line_C.xstart = lC->line_C.xstart;
    lF->line_C.xend = lC->line_C.xend;
    lF->line_F.xstart = lC->line_F.xstart;
    lF->line_F.xend = lC->line_F.xend;
    lC->Nc = lC->line_C.xend - lC->line_C.xstart + 1;
    lC->Nf = lC->line_F.xend - lC->line_F.xstart + 1;
    lF->Nc = lC->Nc;
    lF->Nf = lC->Nf;
  }
}

int orc_geo_init(const mb_layout *L, const mb_config *cfg, mb_geometry *g) {
  if (!L || !cfg || !g) return MB_ERR_INVALID;
  memset(g, 0, sizeof(*g));
  g->layout = *L;
  g->config = *cfg;
  const int LX = cfg->LX, LY = cfg->LY;
  for (int i = 0; i < L->number_area; i++) {
    g->AreaDefine[i].xstart = (int)(L->AreaZone[i].reduced.xstart * (LX - 1)) + L->AreaZone[i].move.xstart;
    g->AreaDefine[i].xend = (int)(L->AreaZone[i].reduced.xend * (LX - 1)) + L->AreaZone[i].move.xend;
    g->AreaDefine[i].ystart = (int)(L->AreaZone[i].reduced.ystart * (LY - 1)) + L->AreaZone[i].move.ystart;
    g->AreaDefine[i].yend = (int)(L->AreaZone[i].reduced.yend * (LY - 1)) + L->AreaZone[i].move.yend;
  }
  int mm = 1;
  double U0_2 = sqrt(cfg->U0[0] * cfg->U0[0] + cfg->U0[1] * cfg->U0[1]);
  double niu = U0_2 * 2 * cfg->R / cfg->Re;
  double tau = 0.5 + 3.0 * niu;
  double rv_tau = 1.0 / tau;
  for (int i = 0; i < L->LEVEL; i++) {
    mm *= L->mi[i];
    tau = 0.5 + L->mi[i] * (tau - 0.5);
    rv_tau = 1.0 / tau;
    for (int j = L->ASP[i]; j < L->ASP[i + 1]; j++) {
      g->Areas[j].m = mm;
      g->Areas[j].nx = (g->AreaDefine[j].xend - g->AreaDefine[j].xstart) * mm + 1;
      g->Areas[j].ny = (g->AreaDefine[j].yend - g->AreaDefine[j].ystart) * mm + 1;
      g->Areas[j].base_x = g->AreaDefine[j].xstart;
      g->Areas[j].base_y = g->AreaDefine[j].ystart;
      g->Areas[j].tau = tau;
      g->Areas[j].rv_tau = rv_tau;
    }
  }
  for (int i = 0; i < L->number_line; i++) {
    int nc = L->NeborCF[i].nc, nf = L->NeborCF[i].nf;
    g->Line_Inf_C[i].areac_n = nc;
    g->Line_Inf_C[i].areaf_n = nf;
    g->Line_Inf_F[i].areac_n = nc;
    g->Line_Inf_F[i].areaf_n = nf;
    line_init(L->NeborCF[i].direction, &g->AreaDefine[nc], &g->Areas[nc], &g->Line_Inf_C[i],
              &g->AreaDefine[nf], &g->Areas[nf], &g->Line_Inf_F[i]);
  }
  for (int i = 0; i + 1 < L->number_line2; i += 2) {
    int nc = L->NeborCC[i].nc, nf = L->NeborCC[i].nf;
    g->Line_Inf_CC[i].areac_n = nc;
    g->Line_Inf_CC[i].areaf_n = nf;
    line_init(L->NeborCC[i].direction, &g->AreaDefine[nc], &g->Areas[nc], &g->Line_Inf_CC[i],
              &g->AreaDefine[nf], &g->Areas[nf], &g->Line_Inf_CC[i + 1]);
    g->Line_Inf_CC[i + 1].areac_n = L->NeborCC[i + 1].nc;
    g->Line_Inf_CC[i + 1].areaf_n = L->NeborCC[i + 1].nf;
    mb_p4 tmp = g->Line_Inf_CC[i + 1].line_C;
    g->Line_Inf_CC[i + 1].line_C = g->Line_Inf_CC[i + 1].line_F;
    g->Line_Inf_CC[i + 1].line_F = tmp;
  }
  return MB_OK;
}

/* ---------------------------------------------------------------------------
 * Allocation (Multi-block-LBM.cu:26-113)
 * ------------------------------------------------------------------------- */
static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

orc_sim *orc_create(const mb_geometry *geo) {
  orc_sim *s = (orc_sim *)calloc(1, sizeof(orc_sim));
  if (!s) return NULL;
  s->geo = *geo;
  const mb_layout *L = &geo->layout;
  for (int a = 0; a < L->number_area; a++) {
    size_t N = (size_t)geo->Areas[a].nx * geo->Areas[a].ny;
    o_d2q9 *p = &s->pp[a];
    p->solid = (int *)calloc(N, sizeof(int));
    p->x = dalloc(N); p->y = dalloc(N); p->rho = dalloc(N); p->ux = dalloc(N); p->uy = dalloc(N);
    p->forcex = dalloc(N); p->forcey = dalloc(N);
    for (int k = 0; k < Q; k++) { p->f[k] = dalloc(N); p->F[k] = dalloc(N); }
    s->upx[a] = dalloc(N);
    s->upy[a] = dalloc(N);
  }
  for (int b = 0; b < L->number_line; b++) {
    o_fstore *t = &s->t3[b];
    t->marker[0] = 2; t->marker[1] = 1; t->marker[2] = 0; /* Multi-block-LBM.cu:45-47 */
    t->N = geo->Line_Inf_C[b].Nf;
    for (int i = 0; i < 3; i++)
      for (int k = 0; k < Q; k++) t->F[i][k] = dalloc(t->N);
    o_spline *sp = &s->s3[b];
    sp->N = geo->Line_Inf_C[b].Nc;
    sp->l = dalloc(sp->N); sp->m = dalloc(sp->N); sp->u = dalloc(sp->N);
    sp->Varibs_M = dalloc(12 * (size_t)sp->N);
    sp->rho = dalloc(sp->N); sp->ux = dalloc(sp->N); sp->uy = dalloc(sp->N);
    for (int k = 0; k < Q; k++) sp->F[k] = dalloc(sp->N);
  }
  s->drag_area = geo->config.drag_area < 0 ? L->number_area - 1 : geo->config.drag_area;
  s->U0_2 = sqrt(geo->config.U0[0] * geo->config.U0[0] + geo->config.U0[1] * geo->config.U0[1]);
  return s;
}

void orc_destroy(orc_sim *s) {
  if (!s) return;
  const mb_layout *L = &s->geo.layout;
  for (int a = 0; a < L->number_area; a++) {
    o_d2q9 *p = &s->pp[a];
    free(p->solid); free(p->x); free(p->y); free(p->rho); free(p->ux); free(p->uy);
    free(p->forcex); free(p->forcey);
    for (int k = 0; k < Q; k++) { free(p->f[k]); free(p->F[k]); }
    free(s->upx[a]); free(s->upy[a]);
  }
  for (int b = 0; b < L->number_line; b++) {
    for (int i = 0; i < 3; i++)
      for (int k = 0; k < Q; k++) free(s->t3[b].F[i][k]);
    o_spline *sp = &s->s3[b];
    free(sp->l); free(sp->m); free(sp->u); free(sp->Varibs_M);
    free(sp->rho); free(sp->ux); free(sp->uy);
    for (int k = 0; k < Q; k++) free(sp->F[k]);
  }
  free(s->drag);
  free(s->pfill);
  for (int a = 0; a < MB_MAX_AREA; a++) free(s->types[a]);
  free(s);
}

/* ---------------------------------------------------------------------------
 * init_General (lbm/init_block.h:2-51).  The ellipse branch has no reference
 * counterpart (batched cases only).
 * ------------------------------------------------------------------------- */
static int is_solid(const mb_config *c, double x, double y) {
  if (c->obstacle == MB_OBST_NONE) return 0;
  if (c->obstacle == MB_OBST_ELLIPSE) {
    double dx = x - c->ell_cx, dy = y - c->ell_cy;
    double ca = cos(c->ell_angle), sa = sin(c->ell_angle);
    double xr = ca * dx + sa * dy, yr = -sa * dx + ca * dy;
    return (xr * xr) / (c->ell_a * c->ell_a) + (yr * yr) / (c->ell_b * c->ell_b) < 1.0;
  }
  return (x - c->CX) * (x - c->CX) + (y - c->CY) * (y - c->CY) < c->R * c->R;
}

/* Periodic domain (mb_config.periodic; no reference counterpart): the level-0
 * nodes on a wrapped edge are ghosts of the node LX-2 (LY-2) nodes away. */
static int is_periodic_ghost(const mb_config *c, double x, double y) {
  return ((c->periodic & MB_PERIODIC_X) && (x == 0.0 || x == c->LX - 1.0)) ||
         ((c->periodic & MB_PERIODIC_Y) && (y == 0.0 || y == c->LY - 1.0));
}

static void init_general(orc_sim *s, int a) {
  const mb_area *ar = &s->geo.Areas[a];
  const mb_config *c = &s->geo.config;
  o_d2q9 *pp = &s->pp[a];
  const int nx = ar->nx, ny = ar->ny;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int ixy = i + j * nx;
      double dx = 1.0 / ar->m;
      pp->x[ixy] = i * dx + ar->base_x;
      pp->y[ixy] = j * dx + ar->base_y;
      pp->rho[ixy] = c->rho0;
      pp->ux[ixy] = c->U0[0];
      pp->uy[ixy] = c->U0[1];
      s->upx[a][ixy] = c->U0[0];
      s->upy[a][ixy] = c->U0[1];
      pp->forcex[ixy] = 0.0;
      pp->forcey[ixy] = 0.0;
      double X = pp->x[ixy], Y = pp->y[ixy];
      if (is_solid(c, X, Y)) pp->solid[ixy] = MB_SOLID_SBB;
      else if (is_periodic_ghost(c, X, Y)) pp->solid[ixy] = MB_C_BOUNDARY;
      else if (Y == 0.0) pp->solid[ixy] = MB_FLUID;
      else if (Y == c->LY - 1.0) pp->solid[ixy] = MB_FLUID;
      else if (X == 0.0) pp->solid[ixy] = MB_FLUID;
      else if (X == c->LX - 1.0) pp->solid[ixy] = MB_FLUID;
      else if (i == 0 || j == 0 || i == nx - 1 || j == ny - 1) pp->solid[ixy] = MB_C_BOUNDARY;
      else pp->solid[ixy] = MB_FLUID;
      for (int k = 0; k < Q; k++) {
        pp->F[k][ixy] = orc_feq(k, pp->rho[ixy], pp->ux[ixy], pp->uy[ixy]);
        pp->f[k][ixy] = pp->F[k][ixy];
      }
    }
}

/* position of point ip on a line (the is==ie test of init_multi.h:14-15 and
 * assit_multi.h:61-70) */
static inline void line_point(const mb_p4 *p, int ip, int *i, int *j) {
  if (p->xstart == p->xend) { *i = p->xstart; *j = p->ystart + ip; }
  else { *i = p->xstart + ip; *j = p->ystart; }
}

/* init_Fstore (multi/init_multi.h:3-28) */
static void init_fstore(orc_sim *s, int b) {
  const mb_line *ln = &s->geo.Line_Inf_C[b];
  const mb_area *af = &s->geo.Areas[ln->areaf_n];
  o_d2q9 *pp = &s->pp[ln->areaf_n];
  o_fstore *t = &s->t3[b];
  for (int ip = 0; ip < t->N; ip++) {
    int i, j;
    line_point(&ln->line_F, ip, &i, &j);
    int ixy = i + j * af->nx;
    for (int k = 0; k < Q; k++) {
      t->F[0][k][ip] = pp->F[k][ixy];
      t->F[1][k][ip] = pp->F[k][ixy];
      t->F[2][k][ip] = pp->F[k][ixy];
    }
  }
}

/* init_tri_A (multi/init_multi.h:30-51).  The reference writes l[ip+1]=0 from
 * thread ip while thread ip+1 writes l[ip+1]=0.5; within a warp the later
 * conditional store lands last.  The oracle takes that order (all unconditional
 * stores first, then the conditional ones): natural end rows. */
static void init_tri_a(orc_sim *s, int b) {
  o_spline *sp = &s->s3[b];
  const int N = s->geo.Line_Inf_C[b].Nc;
  for (int ip = 0; ip < sp->N; ip++) { sp->l[ip] = 0.5; sp->m[ip] = 2.0; sp->u[ip] = 0.5; }
  for (int ip = 0; ip < sp->N; ip++) {
    if (ip == 0) sp->l[ip] = 0.0;
    if (ip == N - 1) sp->u[ip] = 0.0;
    if (ip == 0 || ip == N - 2) {
      sp->u[ip] = 0.0;
      if (ip + 1 < sp->N) sp->l[ip + 1] = 0.0;
    }
  }
}

/* ---------------------------------------------------------------------------
 * Drag links: kernel_sum_N_drag + sum_N_drag + fdrag_store
 * (lbm/force_block.h:2-127).  Enumeration is i-outer, j-inner, k.
 * ------------------------------------------------------------------------- */
static void drag_setup(orc_sim *s) {
  free(s->drag);
  s->drag = NULL;
  const int a = s->drag_area;
  const mb_area *ar = &s->geo.Areas[a];
  const int *solid = s->pp[a].solid;
  int n = 0;
  for (int pass = 0; pass < 2; pass++) {
    int ii = 0;
    for (int i = 0; i < ar->nx; i++)
      for (int j = 0; j < ar->ny; j++) {
        int ixy = i + j * ar->nx;
        if (solid[ixy] != MB_SOLID_SBB && solid[ixy] != MB_SOLID_HBB) continue;
        for (int k = 0; k < Q; k++) {
          int id = i - Ev[k], jd = j - Ev[k + Q];
          if (id < 0 || id > ar->nx - 1 || jd < 0 || jd > ar->ny - 1) continue;
          if (solid[id + jd * ar->nx] == MB_FLUID) {
            if (pass == 1) { s->drag[3 * ii] = i; s->drag[3 * ii + 1] = j; s->drag[3 * ii + 2] = k; }
            ii++;
          }
        }
      }
    if (pass == 0) { n = ii; s->n_drag = n; s->drag = (int *)calloc(3 * (size_t)(n ? n : 1), sizeof(int)); }
  }
}

/* ---------------------------------------------------------------------------
 * Collision and boundary options the reference declares but never uses:
 * MRT (M_gpu, InvM_gpu, lbm/lbm.h:53-75; Meq, lbm/assit_func.h:10-22), the
 * body-force term of stb3 (evolution_block.h:97-108, forcex/forcey set to one
 * value everywhere), free slip (slip_gpu, lbm/lbm.h:51) and half-way
 * bounce-back (SOLID_HBB, lbm/lbm.h:28).  The reference gives no kernel for
 * the last three; their semantics here:
 *  - SOLID_SLIP (code 2, unused by the reference): an on-node wall like
 *    SOLID_SBB that returns F_k = f_slip(k) instead of f_opp(k);
 *  - SOLID_HBB: a FLUID cell whose upstream neighbour x - e_k is an HBB cell
 *    takes f_k(x) = F_opp(k)(x), its own post-collision value of the previous
 *    step; HBB cells are pulled (for the drag sum) but never collide;
 *  - MRT: F = f - M^-1 S (M f - meq) + dt Force_k, S = diag(0, s_e, s_eps, 0,
 *    s_q, 0, s_q, 1/tau, 1/tau), meq = Meq with A = 1, B = -3.
 * ------------------------------------------------------------------------- */
int orc_set_collision(orc_sim *s, int kind, double s_e, double s_eps, double s_q) {
  if (kind != MB_COLL_BGK && kind != MB_COLL_MRT) return MB_ERR_INVALID;
  s->coll = kind;
  s->s_e = s_e;
  s->s_eps = s_eps;
  s->s_q = s_q;
  return MB_OK;
}

void orc_set_body_force(orc_sim *s, double fx, double fy) {
  s->fx = fx;
  s->fy = fy;
  for (int a = 0; a < s->geo.layout.number_area; a++) {
    const size_t N = (size_t)s->geo.Areas[a].nx * s->geo.Areas[a].ny;
    for (size_t c = 0; c < N; c++) {
      s->pp[a].forcex[c] = fx;
      s->pp[a].forcey[c] = fy;
    }
  }
}

/* Cell types of block a (nx*ny, ixy = i + j*nx): FLUID, SOLID_SBB,
 * SOLID_SLIP or SOLID_HBB where init_General put FLUID or SOLID_SBB;
 * C_BOUNDARY cells must stay C_BOUNDARY. */
int orc_set_cell_types(orc_sim *s, int a, const int *types) {
  if (a < 0 || a >= s->geo.layout.number_area) return MB_ERR_INVALID;
  const size_t N = (size_t)s->geo.Areas[a].nx * s->geo.Areas[a].ny;
  int *solid = s->pp[a].solid;
  for (size_t c = 0; c < N; c++) {
    const int t = types[c], was = solid[c];
    const int movable = was == MB_FLUID || was == MB_SOLID_SBB || was == MB_SOLID_SLIP || was == MB_SOLID_HBB;
    if (movable != (t == MB_FLUID || t == MB_SOLID_SBB || t == MB_SOLID_SLIP || t == MB_SOLID_HBB)) return MB_ERR_INVALID;
    if (!movable && t != was) return MB_ERR_INVALID;
  }
  if (!s->types[a]) s->types[a] = (int *)malloc(N * sizeof(int));
  memcpy(s->types[a], types, N * sizeof(int));
  memcpy(solid, types, N * sizeof(int));
  if (a == s->drag_area) drag_setup(s);
  return MB_OK;
}

static void apply_options(orc_sim *s, int a) {
  const size_t N = (size_t)s->geo.Areas[a].nx * s->geo.Areas[a].ny;
  o_d2q9 *pp = &s->pp[a];
  if (s->types[a]) memcpy(pp->solid, s->types[a], N * sizeof(int));
  for (size_t c = 0; c < N; c++) {
    pp->forcex[c] = s->fx;
    pp->forcey[c] = s->fy;
  }
}

/* Periodic ghost map: for every level-0 ghost cell, the level-0 cell at its
 * image node that the block step computes (the first block in index order
 * whose cell there is not C_BOUNDARY).  Built from the cell types alone,
 * without the copy lines of the geometry. */
static int build_pfill(orc_sim *s) {
  const mb_layout *L = &s->geo.layout;
  const mb_config *c = &s->geo.config;
  free(s->pfill);
  s->pfill = NULL;
  s->n_pfill = 0;
  if (!c->periodic) return MB_OK;
  size_t cap = 0;
  for (int a = L->ASP[0]; a < L->ASP[1]; a++) cap += 2 * (size_t)(s->geo.Areas[a].nx + s->geo.Areas[a].ny);
  s->pfill = (int *)malloc(4 * sizeof(int) * (cap ? cap : 1));
  if (!s->pfill) return MB_ERR_NOMEM;
  for (int a = L->ASP[0]; a < L->ASP[1]; a++) {
    const mb_area *A = &s->geo.Areas[a];
    for (int j = 0; j < A->ny; j++)
      for (int i = 0; i < A->nx; i++) {
        const double X = i + A->base_x, Y = j + A->base_y;
        if (!is_periodic_ghost(c, X, Y)) continue;
        double Xi = X, Yi = Y;
        if (c->periodic & MB_PERIODIC_X) Xi = X == 0.0 ? c->LX - 2.0 : (X == c->LX - 1.0 ? 1.0 : X);
        if (c->periodic & MB_PERIODIC_Y) Yi = Y == 0.0 ? c->LY - 2.0 : (Y == c->LY - 1.0 ? 1.0 : Y);
        int owner = -1, cell = 0;
        for (int b = L->ASP[0]; b < L->ASP[1] && owner < 0; b++) {
          const mb_area *B = &s->geo.Areas[b];
          const int ii = (int)(Xi - B->base_x), jj = (int)(Yi - B->base_y);
          if (ii < 0 || jj < 0 || ii >= B->nx || jj >= B->ny) continue;
          if (s->pp[b].solid[ii + jj * B->nx] == MB_C_BOUNDARY) continue;
          owner = b;
          cell = ii + jj * B->nx;
        }
        if (owner < 0) return MB_ERR_GEOMETRY;
        int *e = s->pfill + 4 * s->n_pfill++;
        e[0] = a; e[1] = i + j * A->nx; e[2] = owner; e[3] = cell;
      }
  }
  return MB_OK;
}

/* after the level-0 copies: every ghost takes its image cell's state */
static void periodic_fill(orc_sim *s) {
  for (int q = 0; q < s->n_pfill; q++) {
    const int *e = s->pfill + 4 * q;
    o_d2q9 *g = &s->pp[e[0]], *o = &s->pp[e[2]];
    g->rho[e[1]] = o->rho[e[3]];
    g->ux[e[1]] = o->ux[e[3]];
    g->uy[e[1]] = o->uy[e[3]];
    for (int k = 0; k < Q; k++) g->F[k][e[1]] = o->F[k][e[3]];
  }
}

/* The state the reference derives from the initial fields, after
 * orc_set_fields replaced them: ring slots from the fine edge F (init_Fstore,
 * multi/init_multi.h:3-28) and u_prev from u. */
void orc_sync_history(orc_sim *s) {
  const mb_layout *L = &s->geo.layout;
  for (int b = 0; b < L->number_line; b++) init_fstore(s, b);
  for (int a = 0; a < L->number_area; a++) {
    const size_t N = (size_t)s->geo.Areas[a].nx * s->geo.Areas[a].ny;
    memcpy(s->upx[a], s->pp[a].ux, N * sizeof(double));
    memcpy(s->upy[a], s->pp[a].uy, N * sizeof(double));
  }
}

int orc_init(orc_sim *s) {
  const mb_layout *L = &s->geo.layout;
  for (int a = 0; a < L->number_area; a++) {
    init_general(s, a);
    apply_options(s, a);
  }
  if (build_pfill(s)) return MB_ERR_GEOMETRY;
  drag_setup(s);
  for (int b = 0; b < L->number_line; b++) { init_fstore(s, b); init_tri_a(s, b); }
  return MB_OK;
}

/* ---------------------------------------------------------------------------
 * Block step: evolution_area_stb1/2/3 (multi/FH/evolution_block.h:3-126)
 * ------------------------------------------------------------------------- */
void orc_block_step(orc_sim *s, int a) {
  const mb_area area = s->geo.Areas[a];
  const mb_config *c = &s->geo.config;
  o_d2q9 *pp = &s->pp[a];
  const int nx = area.nx, ny = area.ny;
  /* stb1: pull stream; out-of-block neighbours keep the old f (:23-24) */
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int ixy = i + j * nx;
      const int t = pp->solid[ixy];
      if (t == MB_FLUID || t == MB_SOLID_SBB || t == MB_SOLID_SLIP || t == MB_SOLID_HBB) {
        for (int k = 0; k < Q; k++) {
          int id = i - Ev[k], jd = j - Ev[k + Q];
          if (id < 0 || id > nx - 1 || jd < 0 || jd > ny - 1) continue;
          if (t == MB_FLUID && pp->solid[id + jd * nx] == MB_SOLID_HBB)
            pp->f[k][ixy] = pp->F[Opp[k]][ixy]; /* half-way bounce-back */
          else
            pp->f[k][ixy] = pp->F[k][id + jd * nx];
        }
      }
    }
  /* stb2: equilibrium on block-edge FLUID cells (:47-57), else Macros (:60-70) */
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int ixy = i + j * nx;
      if (pp->solid[ixy] != MB_FLUID) continue;
      if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1) {
        pp->rho[ixy] = c->rho0;
        pp->ux[ixy] = c->U0[0];
        pp->uy[ixy] = c->U0[1];
        for (int k = 0; k < Q; k++) pp->f[k][ixy] = orc_feq(k, c->rho0, c->U0[0], c->U0[1]);
      } else {
        double ft[Q], rh, ux, uy;
        for (int k = 0; k < Q; k++) ft[k] = pp->f[k][ixy];
        macros(&rh, &ux, &uy, ft);
        pp->rho[ixy] = rh;
        pp->ux[ixy] = ux;
        pp->uy[ixy] = uy;
      }
    }
  /* stb3: BGK with the (zero) forcing term (:90-111), on-node bounce-back (:113-117) */
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int ixy = i + j * nx;
      double dt = 1.0 / area.m;
      double ft[Q];
      for (int k = 0; k < Q; k++) ft[k] = pp->f[k][ixy];
      if (pp->solid[ixy] == MB_FLUID) {
        double rh = pp->rho[ixy], ux = pp->ux[ixy], uy = pp->uy[ixy];
        double fx = pp->forcex[ixy], fy = pp->forcey[ixy];
        double dm[Q]; /* MRT: M^-1 S (M f - meq) as S_i (m_i - meq_i) / Mn_i */
        if (s->coll == MB_COLL_MRT) {
          double m[Q], meq[Q], sr[Q];
          for (int q = 0; q < Q; q++) {
            m[q] = 0.0;
            for (int k = 0; k < Q; k++) m[q] += Mm[q][k] * ft[k];
          }
          const double uv = ux * ux + uy * uy; /* Meq, assit_func.h:10-22, A = 1, B = -3 */
          meq[0] = rh;
          meq[1] = rh * (-2.0 + 3.0 * uv);
          meq[2] = rh * (1.0 - 3.0 * uv);
          meq[3] = rh * ux;
          meq[4] = -meq[3];
          meq[5] = rh * uy;
          meq[6] = -meq[5];
          meq[7] = rh * (ux * ux - uy * uy);
          meq[8] = rh * (ux * uy);
          sr[0] = 0.0; sr[3] = 0.0; sr[5] = 0.0;
          sr[1] = s->s_e > 0 ? s->s_e : area.rv_tau;
          sr[2] = s->s_eps > 0 ? s->s_eps : area.rv_tau;
          sr[4] = sr[6] = s->s_q > 0 ? s->s_q : area.rv_tau;
          sr[7] = sr[8] = area.rv_tau;
          for (int q = 0; q < Q; q++) dm[q] = sr[q] * (m[q] - meq[q]) / Mn[q];
        }
        for (int k = 0; k < Q; k++) {
          double vx = 3.0 * (Ev[k] - ux) + 9.0 * (Ev[k] * ux + Ev[k + Q] * uy) * Ev[k];
          double vy = 3.0 * (Ev[k + Q] - uy) + 9.0 * (Ev[k] * ux + Ev[k + Q] * uy) * Ev[k + Q];
          double Fk = (1.0 - 0.5 * area.rv_tau) * Wt[k] * (vx * fx + vy * fy);
          if (s->coll == MB_COLL_MRT) {
            double r = 0.0;
            for (int q = 0; q < Q; q++) r += Mm[q][k] * dm[q];
            pp->F[k][ixy] = ft[k] - r + dt * Fk;
          } else {
            pp->F[k][ixy] = ft[k] - (ft[k] - orc_feq(k, rh, ux, uy)) * area.rv_tau + dt * Fk;
          }
        }
      } else if (pp->solid[ixy] == MB_SOLID_SBB) {
        for (int k = 0; k < Q; k++) pp->F[k][ixy] = ft[Opp[k]];
      } else if (pp->solid[ixy] == MB_SOLID_SLIP) {
        for (int k = 0; k < Q; k++) pp->F[k][ixy] = ft[Slip[k]];
      }
    }
}

/* ---------------------------------------------------------------------------
 * Interface kernels (multi/FH/assit_multi.h)
 * ------------------------------------------------------------------------- */
/* c_c_boundary_transfer (:2-46): source line_C in areac_n, target line_F in areaf_n */
void orc_c_c(orc_sim *s, int c) {
  const mb_line *ln = &s->geo.Line_Inf_CC[c];
  const int nx1 = s->geo.Areas[ln->areac_n].nx, nx2 = s->geo.Areas[ln->areaf_n].nx;
  o_d2q9 *p1 = &s->pp[ln->areac_n], *p2 = &s->pp[ln->areaf_n];
  const int xs1 = ln->line_C.xstart, xe1 = ln->line_C.xend, ys1 = ln->line_C.ystart, ye1 = ln->line_C.yend;
  const int xs2 = ln->line_F.xstart, ys2 = ln->line_F.ystart;
  for (int ip = 0; ip < ln->Nc; ip++) {
    int i1 = 0, j1 = 0, i2 = 0, j2 = 0;
    if (xs1 == xe1) { i1 = xs1; j1 = ys1 + ip; i2 = xs2; j2 = ys2 + ip; }
    if (ys1 == ye1) { i1 = xs1 + ip; j1 = ys1; i2 = xs2 + ip; j2 = ys2; }
    int ixy1 = i1 + j1 * nx1, ixy2 = i2 + j2 * nx2;
    p2->rho[ixy2] = p1->rho[ixy1];
    p2->ux[ixy2] = p1->ux[ixy1];
    p2->uy[ixy2] = p1->uy[ixy1];
    for (int k = 0; k < Q; k++) p2->F[k][ixy2] = p1->F[k][ixy1];
  }
}

/* init_Spline3 (:48-116).  The reference reads neighbour points that other
 * CTAs write in the same launch (:100-107) when Nc > 256; the oracle gathers
 * the whole line first (the result of the reference when Nc <= 256). */
static void init_spline3(orc_sim *s, int b) {
  const mb_line *ln = &s->geo.Line_Inf_C[b];
  const int nx = s->geo.Areas[ln->areac_n].nx;
  o_d2q9 *pp = &s->pp[ln->areac_n];
  o_spline *sp = &s->s3[b];
  const int N = sp->N;
  for (int ip = 0; ip < N; ip++) {
    int i, j;
    line_point(&ln->line_C, ip, &i, &j);
    int ixy = i + j * nx;
    sp->rho[ip] = pp->rho[ixy];
    sp->ux[ip] = pp->ux[ixy];
    sp->uy[ip] = pp->uy[ixy];
    for (int k = 0; k < Q; k++) sp->F[k][ip] = pp->F[k][ixy];
  }
  double *V = sp->Varibs_M;
  for (int ip = 0; ip < N; ip++) {
    if (ip == 0 || ip == N - 1) {
      V[ip] = 0.0;
      V[N + ip] = 0.0;
      V[2 * N + ip] = 0.0;
      for (int k = 0; k < Q; k++) V[(3 + k) * N + ip] = 0.0;
    } else {
      V[ip] = (6.0 * sp->rho[ip] - 3.0 * sp->rho[ip - 1] - 3.0 * sp->rho[ip + 1]);
      V[N + ip] = (6.0 * sp->ux[ip] - 3.0 * sp->ux[ip - 1] - 3.0 * sp->ux[ip + 1]);
      V[2 * N + ip] = (6.0 * sp->uy[ip] - 3.0 * sp->uy[ip - 1] - 3.0 * sp->uy[ip + 1]);
      for (int k = 0; k < Q; k++)
        V[(3 + k) * N + ip] = (6.0 * sp->F[k][ip] - 3.0 * sp->F[k][ip - 1] - 3.0 * sp->F[k][ip + 1]);
    }
  }
}

/* cusparseDgtsv2 (assit_multi.h:194-205) is NVIDIA library code; the oracle
 * solves the same diagonally dominant system (|2| > |0.5|+|0.5|) by the
 * Thomas algorithm, which needs no pivoting.  B is column-major, ldb >= n. */
void orc_gtsv(int n, int nrhs, const double *l, const double *m, const double *u, double *B, int ldb) {
  double *cp = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  for (int r = 0; r < nrhs; r++) {
    double *d = B + (size_t)r * ldb;
    cp[0] = u[0] / m[0];
    d[0] = d[0] / m[0];
    for (int i = 1; i < n; i++) {
      double den = m[i] - l[i] * cp[i - 1];
      cp[i] = u[i] / den;
      d[i] = (d[i] - l[i] * d[i - 1]) / den;
    }
    for (int i = n - 2; i >= 0; i--) d[i] = d[i] - cp[i] * d[i + 1];
  }
  free(cp);
}

/* Spline3_S (:118-134) including its 0.1666667 constant */
double orc_spline3_s(double xx, double x_1, double h, double fi_1, double fi, double mi_1, double mi) {
  double x, a, b, c, d;
  x = x_1 + h;
  a = mi_1 * (x - xx) * (x - xx) * (x - xx) * 0.1666667;
  b = mi * (xx - x_1) * (xx - x_1) * (xx - x_1) * 0.1666667;
  c = (fi_1 - mi_1 * h * h * 0.1666667) * (x - xx);
  d = (fi - mi * h * h * 0.1666667) * (xx - x_1);
  return (a + b + c + d);
}

/* calculate_Spline3_gpu (:136-185): writes fine-edge rho/ux/uy and slot marker[0] */
static void calculate_spline3(orc_sim *s, int b) {
  const mb_line *ln = &s->geo.Line_Inf_C[b];
  const mb_area *ac = &s->geo.Areas[ln->areac_n], *af = &s->geo.Areas[ln->areaf_n];
  o_d2q9 *pp = &s->pp[ln->areaf_n];
  o_spline *sp = &s->s3[b];
  double **lt3 = s->t3[b].F[s->t3[b].marker[0]];
  const int N = sp->N;
  const double *V = sp->Varibs_M;
  const int r = af->m / ac->m;
  for (int ip = 0; ip < ln->Nf; ip++) {
    int i, j;
    line_point(&ln->line_F, ip, &i, &j);
    int ixy = i + j * af->nx;
    double xx = (double)ip / (double)r;
    int I;
    if (ceil(xx) == 0) I = (int)(ceil(xx) + 1.0);
    else I = (int)(ceil(xx));
    double rho_t = orc_spline3_s(xx, (I - 1.0), 1.0, sp->rho[I - 1], sp->rho[I], V[I - 1], V[I]);
    double ux_t = orc_spline3_s(xx, (I - 1.0), 1.0, sp->ux[I - 1], sp->ux[I], V[N + I - 1], V[N + I]);
    double uy_t = orc_spline3_s(xx, (I - 1.0), 1.0, sp->uy[I - 1], sp->uy[I], V[2 * N + I - 1], V[2 * N + I]);
    pp->rho[ixy] = rho_t;
    pp->ux[ixy] = ux_t;
    pp->uy[ixy] = uy_t;
    double para = (af->tau - 1.0) / (r * (ac->tau - 1.0));
    for (int k = 0; k < Q; k++) {
      double ft = orc_spline3_s(xx, (I - 1.0), 1.0, sp->F[k][I - 1], sp->F[k][I], V[(3 + k) * N + I - 1],
                                V[(3 + k) * N + I]);
      double fe = orc_feq(k, rho_t, ux_t, uy_t);
      lt3[k][ip] = fe + para * (ft - fe);
    }
  }
}

/* space_interpolation_Spline3 (:187-211) */
void orc_space_interpolation(orc_sim *s, int b) {
  o_spline *sp = &s->s3[b];
  init_spline3(s, b);
  orc_gtsv(sp->N, 12, sp->l, sp->m, sp->u, sp->Varibs_M, sp->N);
  calculate_spline3(s, b);
}

/* temporal_interpolation (:213-247): F = a*F(t-1) - b*F(t) + c*F(t+1) on the fine edge */
void orc_temporal(orc_sim *s, int b, double xm) {
  const mb_line *ln = &s->geo.Line_Inf_C[b];
  const int nx = s->geo.Areas[ln->areaf_n].nx;
  o_d2q9 *pp = &s->pp[ln->areaf_n];
  o_fstore *t = &s->t3[b];
  double **Ft_1 = t->F[t->marker[0]], **Ft = t->F[t->marker[1]], **Ft1 = t->F[t->marker[2]];
  double a = 0.5 * (xm - 1.0) * xm;
  double bb = (xm - 1.0) * (xm + 1.0);
  double c = 0.5 * xm * (xm + 1.0);
  for (int ip = 0; ip < t->N; ip++) {
    int i, j;
    line_point(&ln->line_F, ip, &i, &j);
    int ixy = i + j * nx;
    for (int k = 0; k < Q; k++) pp->F[k][ixy] = a * Ft_1[k][ip] - bb * Ft[k][ip] + c * Ft1[k][ip];
  }
}

/* c_f_boundary_transfer (:249-271): fine edge F <- slot marker[2] */
void orc_c_f(orc_sim *s, int b) {
  const mb_line *ln = &s->geo.Line_Inf_C[b];
  const int nx = s->geo.Areas[ln->areaf_n].nx;
  o_d2q9 *pp = &s->pp[ln->areaf_n];
  o_fstore *t = &s->t3[b];
  double **Ft = t->F[t->marker[2]];
  for (int ip = 0; ip < t->N; ip++) {
    int i, j;
    line_point(&ln->line_F, ip, &i, &j);
    int ixy = i + j * nx;
    for (int k = 0; k < Q; k++) pp->F[k][ixy] = Ft[k][ip];
  }
}

/* f_c_boundary_transfer (:273-314), on Line_Inf_F */
void orc_f_c(orc_sim *s, int b) {
  const mb_line *ln = &s->geo.Line_Inf_F[b];
  const mb_area *ac = &s->geo.Areas[ln->areac_n], *af = &s->geo.Areas[ln->areaf_n];
  o_d2q9 *pc = &s->pp[ln->areac_n], *pf = &s->pp[ln->areaf_n];
  const int r = af->m / ac->m;
  for (int ip = 0; ip < ln->Nc; ip++) {
    int ic, jc, i_f, j_f;
    if (ln->line_C.xstart == ln->line_C.xend) {
      ic = ln->line_C.xstart; jc = ln->line_C.ystart + ip;
      i_f = ln->line_F.xstart; j_f = ln->line_F.ystart + r * ip;
    } else {
      ic = ln->line_C.xstart + ip; jc = ln->line_C.ystart;
      i_f = ln->line_F.xstart + r * ip; j_f = ln->line_F.ystart;
    }
    int ixyc = ic + jc * ac->nx, ixyf = i_f + j_f * af->nx;
    pc->rho[ixyc] = pf->rho[ixyf];
    pc->ux[ixyc] = pf->ux[ixyf];
    pc->uy[ixyc] = pf->uy[ixyf];
    double para = r * (ac->tau - 1.0) / (af->tau - 1.0);
    for (int k = 0; k < Q; k++) {
      double ft = pf->F[k][ixyf];
      double fe = orc_feq(k, pf->rho[ixyf], pf->ux[ixyf], pf->uy[ixyf]);
      pc->F[k][ixyc] = fe + para * (ft - fe);
    }
  }
}

/* ring rotation (evolution.h:41-46) */
void orc_rotate_markers(orc_sim *s, int b) {
  for (int p = 0; p < 3; p++) {
    int bb = s->t3[b].marker[p] - 1;
    s->t3[b].marker[p] = (bb == -1) ? 2 : bb;
  }
}

/* ---------------------------------------------------------------------------
 * Level scheduler: evolution (evolution.h:2-65)
 * ------------------------------------------------------------------------- */
static void evolution(orc_sim *s, int level) {
  const mb_layout *L = &s->geo.layout;
  /* The reference evaluates mi[LEVEL] (one past the table) before its
   * level == LEVEL return (evolution.h:4-8); either way that call does nothing. */
  if (level == L->LEVEL) return;
  for (int i = 0; i < L->mi[level]; i++) {
    if (!(level == 0 || i == 0)) {
      for (int b = L->LTCFFCP[level]; b < L->LTCFFCP[level + 1]; b++)
        orc_temporal(s, b, (1.0 * i / L->mi[level]));
    }
    for (int a = L->ASP[level]; a < L->ASP[level + 1]; a++) orc_block_step(s, a);
    if (L->number_line2 != 0)
      for (int c = L->LCCP[level]; c < L->LCCP[level + 1]; c++)
        if (L->NeborCC[c].direction != MB_DIR_PERIODIC) orc_c_c(s, c);
    if (level == 0) periodic_fill(s);
    if (level != L->LEVEL - 1) {
      for (int b = L->LS3CFFCP[level]; b < L->LS3CFFCP[level + 1]; b++) {
        orc_space_interpolation(s, b);
        orc_rotate_markers(s, b);
      }
    }
    evolution(s, level + 1);
    if (level != 0 && i == L->mi[level] - 1) {
      for (int b = L->LTCFFCP[level]; b < L->LTCFFCP[level + 1]; b++) {
        orc_c_f(s, b);
        orc_f_c(s, b);
      }
    }
  }
}

void orc_evolution(orc_sim *s, int n) {
  (void)n;
  evolution(s, 0);
}

/* ---------------------------------------------------------------------------
 * Diagnostics
 * ------------------------------------------------------------------------- */
int orc_drag_link_count(orc_sim *s) { return s->n_drag; }
void orc_drag_links(orc_sim *s, int *ijk) { memcpy(ijk, s->drag, sizeof(int) * 3 * (size_t)s->n_drag); }

/* kernel_sum_Force + getDrag_block (force_block.h:129-216): per-CTA shared-memory
 * tree over 256 links, then an in-order host sum of the CTA partials. */
void orc_drag(orc_sim *s, double force[2], double *cd, double *cl) {
  const int a = s->drag_area;
  const mb_area *ar = &s->geo.Areas[a];
  const o_d2q9 *pp = &s->pp[a];
  const int N = s->n_drag;
  const int Bx = (int)ceil(N / (double)BLOCK1D);
  double fxs[BLOCK1D], fys[BLOCK1D];
  force[0] = 0.0;
  force[1] = 0.0;
  for (int bx = 0; bx < Bx; bx++) {
    for (int tx = 0; tx < BLOCK1D; tx++) {
      int ip = bx * BLOCK1D + tx;
      fxs[tx] = 0.0;
      fys[tx] = 0.0;
      if (ip < N) {
        int i = s->drag[3 * ip], j = s->drag[3 * ip + 1], k = s->drag[3 * ip + 2];
        int id = i - Ev[k], jd = j - Ev[Q + k], kd = Opp[k];
        int ixy = i + j * ar->nx, ixyd = id + jd * ar->nx;
        fxs[tx] = (pp->f[k][ixy] * Ev[k] - pp->f[kd][ixyd] * Ev[kd]);
        fys[tx] = (pp->f[k][ixy] * Ev[k + Q] - pp->f[kd][ixyd] * Ev[kd + Q]);
      }
    }
    for (int st = BLOCK1D / 2; st > 0; st >>= 1)
      for (int tx = 0; tx < st; tx++) { fxs[tx] += fxs[tx + st]; fys[tx] += fys[tx + st]; }
    force[0] += fxs[0];
    force[1] += fys[0];
  }
  const mb_config *c = &s->geo.config;
  double den = c->rho0 * s->U0_2 * s->U0_2 * ar->m * c->R;
  if (cd) *cd = force[0] / den;
  if (cl) *cl = force[1] / den;
}

/* error_L2_area + error_L2 (lbm/error_L2.h:3-91): per 16x16 CTA tree sums, an
 * in-order host sum per block, weights 1/m, u_prev <- u. */
double orc_error_L2(orc_sim *s) {
  const mb_layout *L = &s->geo.layout;
  double uvp2_all = 0.0, uv2_all = 0.0;
  for (int a = 0; a < L->number_area; a++) {
    const mb_area *ar = &s->geo.Areas[a];
    const int nx = ar->nx, ny = ar->ny;
    const int Bx = (int)ceil(nx / (double)BLOCKX), By = (int)ceil(ny / (double)BLOCKY);
    const int NB = Bx * By;
    double *pv = (double *)malloc(sizeof(double) * 2 * (size_t)NB);
    const double *ux = s->pp[a].ux, *uy = s->pp[a].uy;
    double *upx = s->upx[a], *upy = s->upy[a];
#pragma omp parallel for schedule(static)
    for (int bip = 0; bip < NB; bip++) {
      int bx = bip % Bx, by = bip / Bx;
      double s1[BLOCKX * BLOCKY], s2[BLOCKX * BLOCKY];
      for (int tip = 0; tip < BLOCKX * BLOCKY; tip++) {
        int tx = tip % BLOCKX, ty = tip / BLOCKX;
        int i = bx * BLOCKX + tx, j = by * BLOCKY + ty;
        s1[tip] = 0.0;
        s2[tip] = 0.0;
        if (i <= nx - 1 && j <= ny - 1) {
          int ixy = i + j * nx;
          double uxt = ux[ixy], upxt = upx[ixy], uyt = uy[ixy], upyt = upy[ixy];
          s1[tip] = (uxt - upxt) * (uxt - upxt) + (uyt - upyt) * (uyt - upyt);
          s2[tip] = uxt * uxt + uyt * uyt;
          upx[ixy] = uxt;
          upy[ixy] = uyt;
        }
      }
      for (int st = BLOCKX * BLOCKY / 2; st > 0; st >>= 1)
        for (int t = 0; t < st; t++) { s1[t] += s1[t + st]; s2[t] += s2[t + st]; }
      pv[2 * bip] = s1[0];
      pv[2 * bip + 1] = s2[0];
    }
    double uvp2_area = 0.0, uv2_area = 0.0;
    for (int i = 0; i < NB; i++) { uvp2_area += pv[2 * i]; uv2_area += pv[2 * i + 1]; }
    free(pv);
    uvp2_all += uvp2_area / ar->m;
    uv2_all += uv2_area / ar->m;
  }
  return sqrt(uvp2_all) / sqrt(uv2_all);
}

/* ---------------------------------------------------------------------------
 * Field access
 * ------------------------------------------------------------------------- */
void orc_get_fields(orc_sim *s, int a, double *rho, double *ux, double *uy, double *F, double *f, int *solid) {
  const size_t N = (size_t)s->geo.Areas[a].nx * s->geo.Areas[a].ny;
  const o_d2q9 *p = &s->pp[a];
  if (rho) memcpy(rho, p->rho, N * sizeof(double));
  if (ux) memcpy(ux, p->ux, N * sizeof(double));
  if (uy) memcpy(uy, p->uy, N * sizeof(double));
  if (solid) memcpy(solid, p->solid, N * sizeof(int));
  for (int k = 0; k < Q; k++) {
    if (F) memcpy(F + k * N, p->F[k], N * sizeof(double));
    if (f) memcpy(f + k * N, p->f[k], N * sizeof(double));
  }
}

void orc_set_fields(orc_sim *s, int a, const double *rho, const double *ux, const double *uy, const double *F,
                    const double *f) {
  const size_t N = (size_t)s->geo.Areas[a].nx * s->geo.Areas[a].ny;
  o_d2q9 *p = &s->pp[a];
  if (rho) memcpy(p->rho, rho, N * sizeof(double));
  if (ux) memcpy(p->ux, ux, N * sizeof(double));
  if (uy) memcpy(p->uy, uy, N * sizeof(double));
  for (int k = 0; k < Q; k++) {
    if (F) memcpy(p->F[k], F + k * N, N * sizeof(double));
    if (f) memcpy(p->f[k], f + k * N, N * sizeof(double));
  }
}

void orc_get_slots(orc_sim *s, int b, double *out) {
  const int N = s->t3[b].N;
  for (int t = 0; t < 3; t++)
    for (int k = 0; k < Q; k++) memcpy(out + ((size_t)t * Q + k) * N, s->t3[b].F[t][k], N * sizeof(double));
}

void orc_get_markers(orc_sim *s, int b, int *m3) {
  for (int p = 0; p < 3; p++) m3[p] = s->t3[b].marker[p];
}

/* output (output/output.h:2-38) */
int orc_write_tecplot(orc_sim *s, const char *path) {
  FILE *fp = fopen(path, "w");
  if (!fp) return MB_ERR_INVALID;
  fprintf(fp, "Title= \"LBM 2D\"\n");
  fprintf(fp, "VARIABLES= \"X\",\"Y\",\"solid\",\"rho\",\"U\",\"V\",\n");
  for (int a = 0; a < s->geo.layout.number_area; a++) {
    const mb_area *ar = &s->geo.Areas[a];
    const o_d2q9 *p = &s->pp[a];
    fprintf(fp, "ZONE T= \"zone_level%d\",I= %d,J= %d,F=POINT\n", a, ar->nx, ar->ny);
    for (int j = 0; j < ar->ny; j++)
      for (int i = 0; i < ar->nx; i++) {
        int ixy = i + j * ar->nx;
        fprintf(fp, "%g\t%g\t%d\t%g\t%g\t%g\n", p->x[ixy], p->y[ixy], p->solid[ixy], p->rho[ixy], p->ux[ixy],
                p->uy[ixy]);
      }
  }
  fclose(fp);
  return MB_OK;
}
