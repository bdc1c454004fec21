/*
 * mblbm_run.c - C driver over the mblbm C ABI; the counterpart of main() in
 * Multi-block-LBM.cu:19-230 of zhangya9741/Multi-block-LBM-GPU.
 *
 * Same outputs as the reference program, in the working directory:
 *   fdrag_t.dat   "t\tCd\tCl\t"   every coarse step (force_block.h:212-215)
 *   error_L2.dat  "t\terr"        every coarse step (error_L2.h:85-88)
 *   time_t.dat    "steps seconds" every T steps (Multi-block-LBM.cu:160-167),
 *                 here device wall time, not CPU time
 *   steady_<n>.dat Tecplot fields at n = 0 and every T steps (output.h:2-38)
 *
 * usage: mblbm_run [-g 1_1|2_2|2_5|4_9|cfg1|cfg2] [-p f64|f32|f16s|f32u]
 *                  [-L loops] [-T steps] [-q]        (-q: no per-step diagnostics)
 * Physical parameters default to the reference's parameters.h (LX=768, LY=320,
 * R=10, centre (160,160), U0=(0.1,0), Re=10) for the built-in layouts.
 */
#define _POSIX_C_SOURCE 199309L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/mblbm.h"

static int die(const char *what, int code) {
  fprintf(stderr, "mblbm_run: %s: %s (%d)\n", what, mb_error_string(code), code);
  return 1;
}

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

int main(int argc, char **argv) {
  const char *geo_name = "2_5", *prec_name = "f32";
  int loops = 1, T = 1000, quiet = 0;
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "-g") && i + 1 < argc) geo_name = argv[++i];
    else if (!strcmp(argv[i], "-p") && i + 1 < argc) prec_name = argv[++i];
    else if (!strcmp(argv[i], "-L") && i + 1 < argc) loops = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-T") && i + 1 < argc) T = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-q")) quiet = 1;
    else {
      fprintf(stderr, "usage: %s [-g layout] [-p precision] [-L loops] [-T steps] [-q]\n", argv[0]);
      return 2;
    }
  }
  int prec = MB_PREC_F32;
  if (!strcmp(prec_name, "f64")) prec = MB_PREC_F64;
  else if (!strcmp(prec_name, "f16s")) prec = MB_PREC_F16S;
  else if (!strcmp(prec_name, "f32u")) prec = MB_PREC_F32U;

  mb_layout layout;
  mb_config cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.rho0 = 1.0;
  cfg.drag_area = -1;
  cfg.obstacle = MB_OBST_CIRCLE;
  int rc;
  if (!strcmp(geo_name, "cfg1")) {
    const int box[4] = {60, 140, 40, 120};
    rc = mb_layout_nested(400, 160, 2, box, &layout);
    cfg.LX = 400; cfg.LY = 160; cfg.R = 10; cfg.CX = 100; cfg.CY = 80; cfg.U0[0] = 0.05; cfg.Re = 40.0;
  } else if (!strcmp(geo_name, "cfg2")) {
    const int box[8] = {768, 1280, 384, 640, 896, 1152, 448, 576};
    rc = mb_layout_nested(4096, 1024, 3, box, &layout);
    cfg.LX = 4096; cfg.LY = 1024; cfg.R = 16; cfg.CX = 960; cfg.CY = 512; cfg.U0[0] = 0.04; cfg.Re = 100.0;
  } else {
    rc = mb_layout_builtin(geo_name, &layout);
    cfg.LX = 768; cfg.LY = 320; cfg.R = 10; cfg.CX = 160; cfg.CY = 160; cfg.U0[0] = 0.1; cfg.Re = 10.0;
  }
  if (rc) return die("layout", rc);

  mb_geometry *geo = (mb_geometry *)malloc(sizeof(mb_geometry));
  if ((rc = mb_geo_init(&layout, &cfg, geo))) return die("mb_geo_init", rc);
  mb_ctx *ctx = NULL;
  if ((rc = mb_create(geo, prec, &ctx))) return die("mb_create", rc);
  if ((rc = mb_init(ctx, NULL))) return die("mb_init", rc);
  if ((rc = mb_write_tecplot(ctx, "steady_0.dat"))) return die("output", rc);

  for (int k = 0; k < loops; k++) {
    const double t0 = now_s();
    if (quiet) {
      if ((rc = mb_step(ctx, T, NULL))) return die("mb_step", rc);
    } else {
      for (int n = 0; n < T; n++) {
        double e, force[2], cd, cl;
        if ((rc = mb_step(ctx, 1, NULL))) return die("mb_step", rc);
        if ((rc = mb_error_L2(ctx, &e, NULL))) return die("mb_error_L2", rc);
        if ((rc = mb_drag(ctx, force, &cd, &cl, NULL))) return die("mb_drag", rc);
        mb_append_error_L2("error_L2.dat", k * T + n, e);
        mb_append_drag("fdrag_t.dat", k * T + n, cd, cl);
      }
    }
    double force[2], cd, cl;
    if ((rc = mb_drag(ctx, force, &cd, &cl, NULL))) return die("mb_drag", rc);  /* synchronises */
    const double dt = now_s() - t0;
    printf("%f seconds\n", dt);
    FILE *fp = fopen("time_t.dat", "a");
    if (fp) {
      fprintf(fp, "%d %g\n", (k + 1) * T, dt);
      fclose(fp);
    }
    printf("%d\n", (k + 1) * T);
    char name[64];
    snprintf(name, sizeof name, "steady_%d.dat", (k + 1) * T);
    if ((rc = mb_write_tecplot(ctx, name))) return die("output", rc);
  }
  mb_destroy(ctx);
  free(geo);
  return 0;
}
