/*
 * oracle.h - FP64 CPU restatement of the reference multi-block D2Q9 step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg use it, as the checker.
 *
 * Every function restates one reference function (cited file:line within
 * zhangya9741/Multi-block-LBM-GPU) in plain C with the same FP64 arithmetic
 * order, the same data layout (structure of arrays, ixy = i + j*nx) and the
 * same quirks.  Where the reference has a race, the oracle takes the
 * race-free reading (documented at the function).
 */
#ifndef MBLBM_ORACLE_H
#define MBLBM_ORACLE_H
#include "../include/mblbm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

/* geo_init + Line_init (geo/init_geo.h:17-165) */
int orc_geo_init(const mb_layout *layout, const mb_config *cfg, mb_geometry *geo);
/* Allocation (Multi-block-LBM.cu:26-113) */
orc_sim *orc_create(const mb_geometry *geo);
void orc_destroy(orc_sim *s);
void orc_set_threads(int n);
/* init_General + init_Fstore + init_tri_A + sum_N_drag + fdrag_store
 * (Multi-block-LBM.cu:116-140) */
int orc_init(orc_sim *s);
void orc_sync_history(orc_sim *s);
/* evolution(level 0) (evolution.h:2-65), one coarse step */
void orc_evolution(orc_sim *s, int n);
/* error_L2 (lbm/error_L2.h:57-91); returns the value written to error_L2.dat */
double orc_error_L2(orc_sim *s);
/* getDrag_block (lbm/force_block.h:180-216) */
void orc_drag(orc_sim *s, double force[2], double *cd, double *cl);
int orc_drag_link_count(orc_sim *s);
/* links as (i, j, k) triples, i-outer j-inner (force_block.h:92-116) */
void orc_drag_links(orc_sim *s, int *ijk);

/* single kernels, for per-kernel checks */
void orc_block_step(orc_sim *s, int area);                     /* evolution_block.h:121 */
void orc_c_c(orc_sim *s, int line_cc);                         /* assit_multi.h:2       */
void orc_space_interpolation(orc_sim *s, int line);            /* assit_multi.h:187     */
void orc_temporal(orc_sim *s, int line, double xm);            /* assit_multi.h:213     */
void orc_c_f(orc_sim *s, int line);                            /* assit_multi.h:249     */
void orc_f_c(orc_sim *s, int line);                            /* assit_multi.h:273     */
void orc_rotate_markers(orc_sim *s, int line);                 /* evolution.h:41-46     */
/* tridiagonal solve of the spline system (cusparseDgtsv2 call, assit_multi.h:194-205) */
void orc_gtsv(int n, int nrhs, const double *l, const double *m, const double *u, double *B, int ldb);
/* one Spline3_S evaluation (assit_multi.h:118-134) */
double orc_spline3_s(double xx, double x_1, double h, double fi_1, double fi, double mi_1, double mi);
double orc_feq(int k, double rh, double ux, double uy);

/* options the reference declares but never uses (MRT, body force, free slip,
 * half-way bounce-back); semantics at their definitions in oracle.c */
int orc_set_collision(orc_sim *s, int kind, double s_e, double s_eps, double s_q);
void orc_set_body_force(orc_sim *s, double fx, double fy);
int orc_set_cell_types(orc_sim *s, int area, const int *types);

/* field access (FP64, ixy = i + j*nx; F and f are 9*nx*ny, plane-major) */
void orc_get_fields(orc_sim *s, int area, double *rho, double *ux, double *uy, double *F,
                    double *f, int *solid);
void orc_set_fields(orc_sim *s, int area, const double *rho, const double *ux, const double *uy,
                    const double *F, const double *f);
/* time slots of a coarse-fine line: 3 x 9 x Nf, slot order f_t1, f_t, f_t_1 */
void orc_get_slots(orc_sim *s, int line, double *out);
void orc_get_markers(orc_sim *s, int line, int *marker3);
/* Tecplot writer (output/output.h:2-38) */
int orc_write_tecplot(orc_sim *s, const char *path);

#ifdef __cplusplus
}
#endif
#endif
