/*
 * mblbm.h - C ABI of the B200-native multi-block D2Q9 BGK lattice-Boltzmann step.
 *
 * The entry points replace the host call surface of the reference program
 * (zhangya9741/Multi-block-LBM-GPU): geometry set-up, block and interface
 * initialisation, the recursive level scheduler, momentum-exchange drag, the
 * relative L2 change and the Tecplot writer.  Each declaration cites the
 * reference function it replaces as file:line within that project.
 *
 * Conventions (differ from the reference, which has only void functions):
 *   - every function returns int: MB_OK (0) or a negative MB_ERR_* code;
 *   - no function writes a file except mb_write_tecplot / mb_append_*;
 *   - all device work is enqueued on the caller's stream (mb_stream is a
 *     cudaStream_t passed as void*; NULL = legacy default stream);
 *   - a context is used by one host thread at a time.
 *
 * Types mirror the reference structs field by field so that tables written
 * for the reference (geo/geometry.h) map one-to-one.
 */
#ifndef MBLBM_H
#define MBLBM_H

#ifdef __cplusplus
extern "C" {
#endif

#define MB_ABI_VERSION 1

/* ---- limits of the fixed-size tables ---------------------------------- */
#define MB_MAX_LEVEL 8
#define MB_MAX_AREA 64
#define MB_MAX_LINE 128  /* coarse-fine lines (number_line)            */
#define MB_MAX_LINE2 128 /* same-level lines (number_line2, even)      */

/* ---- error codes ------------------------------------------------------- */
#define MB_OK 0
#define MB_ERR_INVALID -1     /* bad argument or table                   */
#define MB_ERR_CUDA -2        /* a CUDA runtime call failed              */
#define MB_ERR_NOMEM -3       /* device or host allocation failed        */
#define MB_ERR_GEOMETRY -4    /* layout violates a geometry rule         */
#define MB_ERR_UNSUPPORTED -5 /* feature or size outside this build      */
#define MB_ERR_NUMERIC -6     /* NaN / Inf detected in the state         */
#define MB_ERR_TIMEOUT -7     /* a bounded device wait gave up           */
#define MB_ERR_STATE -8       /* call out of order (e.g. step before init)*/
#define MB_ERR_NODEVICE -9    /* no CUDA device / extension unusable     */

/* ---- storage precisions of the distributions -------------------------- */
#define MB_PREC_F64 0  /* FP64 storage and arithmetic (reference precision)     */
#define MB_PREC_F32 1  /* FP32 storage of f - s (shifted, mb_set_shift), FP32 arithmetic */
#define MB_PREC_F16S 2 /* FP16 storage of f - w (shifted), FP32 arithmetic      */
#define MB_PREC_F32U 3 /* FP32 storage of f (unshifted), FP32 arithmetic        */
/* 16-bit storage of the shifted distributions (default f - feq(rho0, U0))
 * with a 3-bit exponent and 12-bit fraction: magnitudes below 1/4, a quarter
 * of FP16's spacing there; FP32 arithmetic.  Out-of-range values saturate
 * and mb_check_finite counts them. */
#define MB_PREC_F16C 4

/* ---- shift of the stored distributions (shifted precisions) ------------- */
/* The shifted precisions store h = f - s with a constant vector s: the lattice
 * weights w (MB_SHIFT_W, MB_PREC_F16S's default), or the equilibrium of the
 * free stream feq(rho0, U0) (MB_SHIFT_FEQ0, the default of MB_PREC_F32 and
 * MB_PREC_F16C: the stored words are then small wherever the flow is close
 * to the free stream, and so are their rounding errors). */
#define MB_SHIFT_W 0
#define MB_SHIFT_FEQ0 1

/* ---- rounding of the stored words (mb_set_rounding) -------------------- */
/* MB_ROUND_NEAREST: round to nearest even (every precision; the default of
 * the FP64 and FP32 forms).
 * MB_ROUND_STOCHASTIC (the 16-bit forms, their default): the
 * collision rounds each output to one of its two neighbouring values of the
 * stored type, the upper one with probability equal to the distance from the
 * lower one over their spacing, so rounding errors have zero mean (FP16: the
 * hardware's stochastic-rounding conversion).  The random bits are a hash of
 * the cell and three of its inputs: every kernel variant and execution mode
 * gives the same words. */
#define MB_ROUND_NEAREST 0
#define MB_ROUND_STOCHASTIC 1

/* ---- cell type codes, values as in lbm/lbm.h:26-32 -------------------- */
#define MB_FLUID 0
#define MB_SOLID_SBB 1
#define MB_SOLID_SLIP 2 /* free-slip on-node wall, slip_gpu (lbm/lbm.h:51); no code in the reference */
#define MB_SOLID_HBB 3  /* half-way bounce-back, SOLID_HBB (lbm/lbm.h:28); declared, unused there */
#define MB_C_BOUNDARY 9

/* ---- collision operators -------------------------------------------------- */
#define MB_COLL_BGK 0 /* evolution_block.h:99-111 */
#define MB_COLL_MRT 1 /* M_gpu/InvM_gpu (lbm/lbm.h:53-75), Meq (lbm/assit_func.h:10-22) */

/* ---- obstacle kinds ---------------------------------------------------- */
#define MB_OBST_CIRCLE 0  /* (x-CX)^2+(y-CY)^2 < R^2, lbm/init_block.h:28    */
#define MB_OBST_ELLIPSE 1 /* rotated ellipse (batched cases; no reference)  */
#define MB_OBST_NONE 2    /* no obstacle (periodic flows; no reference)     */

/* ---- periodic level-0 domain (mb_config.periodic; no reference counterpart)
 * With MB_PERIODIC_X the level-0 nodes x = 0 and x = LX-1 become ghost cells
 * (MB_C_BOUNDARY) of x = LX-2 and x = 1: the period is LX-2 nodes.  Likewise
 * MB_PERIODIC_Y in y.  mb_geo_init adds same-level copy lines, direction code
 * MB_DIR_PERIODIC in NeborCC, that give every ghost the state of the level-0
 * cell computing its image node after each level-0 step, and drops the ghost
 * cells from the ends of the layout's own level-0 lines.  Blocks of finer
 * levels must not touch a periodic edge. */
#define MB_PERIODIC_X 1
#define MB_PERIODIC_Y 2
#define MB_DIR_PERIODIC 8

typedef void *mb_stream; /* cudaStream_t */

/* P4 (lbm/data_type_lbm.h:15-20) */
typedef struct {
  int xstart, xend, ystart, yend;
} mb_p4;
/* P4d (lbm/data_type_lbm.h:26-31) */
typedef struct {
  double xstart, xend, ystart, yend;
} mb_p4d;
/* P4d4i: fractional zone plus integer move (lbm/data_type_lbm.h:32-36) */
typedef struct {
  mb_p4d reduced;
  mb_p4 move;
} mb_zone;
/* P3i: (coarse block, fine block, direction) (lbm/data_type_lbm.h:21-25) */
typedef struct {
  int nc, nf, direction;
} mb_p3i;

/* Block layout: the tables of geo/geometry.h:55-100 as runtime data. */
typedef struct {
  int LEVEL;
  int mi[MB_MAX_LEVEL];
  int number_area, number_line, number_line2;
  int ASP[MB_MAX_LEVEL + 1];
  mb_zone AreaZone[MB_MAX_AREA];
  int LTCFFCP[MB_MAX_LEVEL + 1];
  int LS3CFFCP[MB_MAX_LEVEL + 1];
  int LCCP[MB_MAX_LEVEL + 1];
  mb_p3i NeborCF[MB_MAX_LINE];
  mb_p3i NeborCC[MB_MAX_LINE2];
} mb_layout;

/* Physical parameters: the globals of parameters.h:23-52 as runtime data. */
typedef struct {
  double Re;        /* parameters.h:24 */
  double rho0;      /* parameters.h:27 */
  int LX, LY;       /* parameters.h:32-33 */
  int R, CX, CY;    /* parameters.h:36-40 */
  double U0[2];     /* parameters.h:48 */
  int obstacle;     /* MB_OBST_* */
  double ell_cx, ell_cy, ell_a, ell_b, ell_angle; /* MB_OBST_ELLIPSE only */
  int drag_area;    /* block used for drag; -1 = last block (Multi-block-LBM.cu:127) */
  int periodic;     /* MB_PERIODIC_* bits; 0 = the reference's equilibrium edges */
} mb_config;

/* AREA (lbm/data_type_lbm.h:43-51) */
typedef struct {
  int m, nx, ny;
  double base_x, base_y, tau, rv_tau;
} mb_area;

/* Inf_Ff_store (multi/data_type_multi.h:15-22) */
typedef struct {
  int areac_n, Nc;
  mb_p4 line_C;
  int areaf_n, Nf;
  mb_p4 line_F;
} mb_line;

/* Everything geo_init() produces (geo/init_geo.h:10-14). */
typedef struct {
  mb_layout layout;
  mb_config config;
  mb_p4 AreaDefine[MB_MAX_AREA];
  mb_area Areas[MB_MAX_AREA];
  mb_line Line_Inf_C[MB_MAX_LINE];
  mb_line Line_Inf_F[MB_MAX_LINE];
  mb_line Line_Inf_CC[MB_MAX_LINE2];
} mb_geometry;

typedef struct mb_ctx mb_ctx;
typedef struct mb_batch mb_batch;

/* ---- library ------------------------------------------------------------ */
int mb_version(void);
const char *mb_error_string(int code);

/* ---- layouts and geometry (host only, no device needed) --------------- */
/* Built-in tables "1_1", "2_2", "2_5", "4_9" of geo/geometry.h:7-147. */
int mb_layout_builtin(const char *name, mb_layout *out);
/* Nested rectangular frames: level 0 covers [0,LX-1]x[0,LY-1]; level l>0
 * covers the integer box boxes[4(l-1)..] = {xs, xe, ys, ye} (coarse cells),
 * refined by ratio 2 per level.  Each non-finest level is split into four
 * blocks (top, bottom, left, right) that overlap their neighbours by one
 * coarse cell, the pattern of geo/geometry.h:55-100 (_GEO_2_5). */
int mb_layout_nested(int LX, int LY, int nlevels, const int *boxes, mb_layout *out);
/* geo_init() + Line_init() (geo/init_geo.h:17-165); with mb_config.periodic
 * also the periodic ghost lines (MB_PERIODIC_X above).  Entries of the
 * layout's NeborCC with direction MB_DIR_PERIODIC are dropped first, so the
 * layout of a geometry may be passed in again. */
int mb_geo_init(const mb_layout *layout, const mb_config *cfg, mb_geometry *geo);
/* Checks that every C_BOUNDARY cell is the target of some transfer line. */
int mb_geo_check_coverage(const mb_geometry *geo, int *n_uncovered);

/* ---- context ------------------------------------------------------------- */
/* Allocates all device state (Multi-block-LBM.cu:26-113). */
int mb_create(const mb_geometry *geo, int precision, mb_ctx **out);
int mb_destroy(mb_ctx *ctx);
/* init_General (lbm/init_block.h:2), init_Fstore / init_tri_A
 * (multi/init_multi.h:3,30), sum_N_drag + fdrag_store (lbm/force_block.h:50,78). */
int mb_init(mb_ctx *ctx, mb_stream stream);
/* After mb_set_fields has replaced the fields (a restart from outside data,
 * the learned warm start): re-derives the state the reference derives from
 * the initial fields, the ring slots of every coarse-fine line from the fine
 * edge F (init_Fstore, multi/init_multi.h:3-28) and u_prev from u. */
int mb_sync_history(mb_ctx *ctx, mb_stream stream);
/* n coarse steps of evolution(level 0) (evolution.h:2-65).  The last coarse
 * step of every call leaves rho/ux/uy of all cells up to date, as the
 * reference's stb2 does each step; earlier steps keep only the macroscopic
 * values that interface transfers read. */
int mb_step(mb_ctx *ctx, int n_coarse, mb_stream stream);
/* 0: launch the kernels one by one; 1: replay CUDA graphs of the dependency
 * DAG (default); 2: graphs whose kernel-to-kernel edges are programmatic, so a
 * consumer is scheduled while its producers drain; 3: one persistent
 * executor launch per plan, which tracks the DAG on the device (CTAs claim
 * work items of ready nodes; bulk interior work fills the fine-level chain's
 * waits); 4: hybrid graphs, whose bulk interior nodes (and drag and L2 nodes)
 * are kernel nodes and whose fine-level chain runs as persistent executor
 * launches between them, each capped at mb_set_hybrid_ctas CTAs per SM.
 * Results are identical in every mode. */
int mb_set_graph_mode(mb_ctx *ctx, int mode);
/* Executor CTAs per SM of the chain launches of graph mode 4 (default 2). */
int mb_set_hybrid_ctas(mb_ctx *ctx, int per_sm);
/* Mode 3: a CTA that finds no ready work for this long sets the context's
 * error word and the launch ends; the next synchronising call (mb_sync,
 * mb_drag, mb_error_L2, mb_check_finite, mb_copy_fields) returns
 * MB_ERR_TIMEOUT once.  Default 2 s; at most 600 s.  No reference counterpart. */
int mb_set_program_timeout(mb_ctx *ctx, double seconds);
/* Mode 3: cells per work item of interior (bulk) and of all other block-step
 * nodes (defaults 512 and 256); how many periods of the scheduler state (the
 * coarse-step cycle after which buffer parities and ring markers repeat) one
 * executor launch covers (default 2); at most how many CTAs execute bulk
 * items at once (default 0: no limit), which keeps memory latency low for
 * the fine-level chain.  No reference counterpart. */
int mb_set_program_shape(mb_ctx *ctx, int bulk_cells, int urgent_cells, int periods_per_launch, int bulk_ctas);
/* Mode 3 tracing: records one 48-byte entry per executed work item (global
 * timer at the claim scan, at the start and at the end of the work; plan
 * node, item, SM, CTA, launch number) into a device buffer of `capacity`
 * records (0 turns tracing off).  mb_program_trace copies up to max_records
 * of them to the host and empties the buffer.  No reference counterpart. */
int mb_set_program_trace(mb_ctx *ctx, long long capacity);
int mb_program_trace(mb_ctx *ctx, void *records, long long max_records, long long *n_records);
/* Waits for the stream and reports an executor timeout (MB_ERR_TIMEOUT) of
 * any earlier launch.  No reference counterpart. */
int mb_sync(mb_ctx *ctx, mb_stream stream);
/* One executor launch over a single empty node, for checking the timeout
 * path: stall = 0 completes (MB_OK); stall = 1 gives the node a dependency
 * that nothing satisfies, so the launch gives up after the timeout and the
 * call returns MB_ERR_TIMEOUT with the context still usable.  Synchronous.
 * No reference counterpart. */
int mb_program_selftest(mb_ctx *ctx, int stall, mb_stream stream);
/* Levels with at least `cells` cells update their interior (cells two or more
 * from a block edge) and their rim as separate DAG nodes, so that the interior
 * of the next coarse step overlaps the fine levels of this one.  Default 1e6,
 * no split for MB_PREC_F64; 0 splits every level. */
int mb_set_split_cells(mb_ctx *ctx, long long cells);
/* Work granularity of interface nodes: points per record CTA (graph modes)
 * or work item (mode 3), 32 (default) or 64; spline segments of 32 coarse
 * intervals per CTA or work item, 1 (default) to 4.  Interface lines across
 * rows touch one cache sector per value, so small units spread a node over
 * many SMs' load/store units.  Results are identical. */
int mb_set_interface_shape(mb_ctx *ctx, int rec_points, int spline_segments);
/* Unused shared memory (KB) reserved by every CTA of the bulk block-step
 * launches (the interiors of split levels): an SM then holds fewer of them at
 * once and keeps room for the latency-bound chain launches beside them.
 * Defaults: 80 KB in FP32 storage (two CTAs of the level-0 interior per SM),
 * 60 KB in the 16-bit forms (three), 0 in FP64.  Results are identical. */
int mb_set_bulk_spread(mb_ctx *ctx, int kb);
/* Sets aside up to mb MB of L2 (capped by the device's persisting maximum and
 * by the size of the fine levels' state) for persisting lines, and gives
 * every graph kernel except the bulk interiors an access-policy window over
 * one allocation that holds F and rho/u of the blocks with m > 1 and the
 * interface slots: the fine levels' chain then finds its lines in L2 while
 * the level-0 interior streams beside it.  0 (the default) releases it.  The
 * set-aside is a limit of the calling process's CUDA context, restored to 0
 * by mb_destroy.  Results are identical. */
int mb_set_l2_persist(mb_ctx *ctx, int mb);
/* Coarse steps per replayed CUDA graph (default 24, rounded up to a whole
 * number of scheduler periods; 1 to 4096): a call of n steps replays plans of
 * that length and one plan of the remaining steps.  Longer plans have fewer
 * graph boundaries, across which the next step's level-0 interior cannot
 * start beside the fine levels' chain, and cost more host time to compile
 * once (mb_prepare).  Results are identical. */
int mb_set_plan_steps(mb_ctx *ctx, int n);
/* MB_SHIFT_W or MB_SHIFT_FEQ0 for the stored distributions (no effect on
 * MB_PREC_F64 and MB_PREC_F32U, which store f).  Changing it discards the
 * state: mb_init, mb_set_fields or a checkpoint of the same shift must come
 * next (mb_step returns MB_ERR_STATE until then). */
int mb_set_shift(mb_ctx *ctx, int mode);
/* MB_ROUND_NEAREST or MB_ROUND_STOCHASTIC (MB_PREC_F16C and MB_PREC_F16S,
 * else MB_ERR_INVALID) for the words the collision stores.  The state is
 * kept. */
int mb_set_rounding(mb_ctx *ctx, int mode);
/* Minimum dynamic shared memory (KB, at most 200) per CTA of the spline and
 * the record kernels, which caps how many of their CTAs share one SM: a
 * latency-bound launch that starts while a block step still holds most SMs
 * then spreads over the SMs that free up instead of piling onto the first
 * ones.  Defaults: spline 48 KB in FP32 storage, 64 KB in the 16-bit forms,
 * 96 KB otherwise (at most 2 CTAs per SM); records 0.  Results are identical. */
int mb_set_cta_spread(mb_ctx *ctx, int spline_kb, int records_kb);
/* Splits exactly the levels whose bit is set in level_mask (bit l = level
 * l) into interior and rim nodes, overriding mb_set_split_cells; 0 returns
 * to the cell threshold.  Results are identical. */
int mb_set_split_levels(mb_ctx *ctx, unsigned level_mask);
/* Block-step nodes over at least `cells` cells (a whole level, or its
 * interior or rim) load and store with evict-first cache hints, so that the
 * streamed coarse level does not evict the fine levels' buffers from L2.
 * Default 2e6; 0 never hints.  bulk = 1 also schedules such whole-level
 * nodes as bulk work (lowest graph priority, executor bulk class), as the
 * interiors of split levels always are.  Results are identical. */
int mb_set_stream_cells(mb_ctx *ctx, long long cells, int bulk);
/* Block-step kernel of one level: 0 = one cell per thread (default),
 * 1 = four cells per thread with vector loads, 2 = two cells per thread with
 * the loads of both in flight together, 3 = cell ranges: a CTA steps 256
 * consecutive cells of one block with 32-bit offsets (whole levels and
 * interiors; rims use 0), 4 = cell pairs: a thread steps cells i, i+1 with
 * shared addresses and vector accesses, 256 pairs per CTA (same coverage as 3),
 * 5 = bulk asynchronous copies: persistent CTAs stage the nine input row
 * segments of 256 cells in shared memory with cp.async.bulk and mbarriers
 * (interiors of split levels; the other regions use 0), 6 = octets (16-bit
 * stored forms only; other precisions run 0): a lane steps eight cells of a
 * row with one 16-byte load and store per direction.
 * Default 0; every level uses 4 in MB_PREC_F16S and MB_PREC_F16C, level 0
 * uses 4 in MB_PREC_F32 and MB_PREC_F32U.  Results are identical. */
int mb_set_stb_variant(mb_ctx *ctx, int level, int variant);
/* Caps the grid of interior (bulk) block-step launches at ctas_per_sm CTAs of
 * 256 threads per SM (0 = uncapped), leaving CTA slots on every SM for the
 * fine-level kernels that run beside them. */
int mb_set_bulk_occupancy(mb_ctx *ctx, int ctas_per_sm);
/* Kernel fusions of the plan (bit mask; default 5: bits 0 and 2).  Bit 0: the same-level
 * copies (c_c_boundary_transfer, multi/FH/assit_multi.h:2-46) of a level run
 * inside its block-step launch: each target cell computes its source's new
 * values itself.  Bit 1: the spline of a coarse-fine line
 * (calculate_Spline3_gpu, assit_multi.h:136-185) also does the line's
 * temporal interpolation (assit_multi.h:213-247) of the fine level's next
 * substep, in place of a launch before that substep's block step; the spline
 * then waits for the fine level's current substep, which on the 3-level
 * cylinder costs more than the launch saves, so it is off by default.
 * Bit 2: the same at the spline's own place, on fine levels without
 * same-level copies: the spline writes the interpolated values into the
 * buffer the level's next block step reads, and the level's block step in
 * between leaves those edge cells alone; the spline then runs beside that
 * block step.  Bit 2 takes the lines it applies to before bit 1.  On the
 * 3-level cylinder bit 2 takes 2 of 20 launches per coarse step off the
 * fine levels' chain and the step 1 % shorter (103.1 against 104.3 us in
 * FP32, 93.3 against 93.8 in FP16 storage), so it is on by default.  Batches
 * and the persistent executor leave it out.  Bit 3: the f_c points
 * (f_c_boundary_transfer, multi/FH/assit_multi.h:273-314) whose fine cell the fine level's last
 * substep has just updated run in a small launch beside that block step,
 * which updates those fine cells itself (the step leaves them alone), when
 * no operation in between touches their cells: the coarse level's next
 * substep then waits for that launch, not for the fine step and a record
 * launch after it (levels stepped by the two-cell kernel, and MB_PREC_F32U,
 * keep the records).
 * Bit 4: consecutive record ops share a launch only when all or none of them
 * wait for the latest block step.  Bits 3 and 4 measured within run-to-run
 * noise on the 3-level cylinder and are off by default.  Results are
 * identical. */
int mb_set_fusion(mb_ctx *ctx, int flags);

/* ---- collision and boundary options ----------------------------------------
 * The reference declares these but never uses them: MRT (M_gpu, InvM_gpu,
 * lbm/lbm.h:53-75; Meq, lbm/assit_func.h:10-22), the body-force term of stb3
 * (multi/FH/evolution_block.h:97-108, forcex/forcey), free slip (slip_gpu,
 * lbm/lbm.h:51) and half-way bounce-back (SOLID_HBB, lbm/lbm.h:28).  While any
 * is on, every block step runs one general kernel; the persistent executor
 * (graph mode 3) and batches return MB_ERR_UNSUPPORTED. */
/* MB_COLL_BGK, or MB_COLL_MRT with S = diag(0, s_e, s_eps, 0, s_q, 0, s_q,
 * 1/tau, 1/tau); a rate <= 0 stands for the block's 1/tau (all three <= 0:
 * the BGK result up to rounding).  Rates must be below 2. */
int mb_set_collision(mb_ctx *ctx, int kind, double s_e, double s_eps, double s_q);
/* forcex, forcey of every cell (coarse lattice units), added as
 * dt (1 - 1/(2 tau)) w_k (v_k . F) on every FLUID cell, dt = 1/m. */
int mb_set_body_force(mb_ctx *ctx, double fx, double fy);
/* Cell types of one block, nx*ny codes (i + j*nx): MB_FLUID, MB_SOLID_SBB,
 * MB_SOLID_SLIP or MB_SOLID_HBB on cells that are FLUID or solid; C_BOUNDARY
 * cells must be passed unchanged.  A FLUID cell whose upstream neighbour
 * x - e_k is HBB takes f_k = F_opp(k) of itself; a slip cell returns
 * F_k = f_slip(k).  The drag sums SBB and HBB links.  Kept across mb_init. */
int mb_set_cell_types(mb_ctx *ctx, int area, const int *types);
/* Compiles the plans (and CUDA graphs, instantiated and uploaded) that
 * mb_step(ctx, n) will replay from the current state, so the step call itself
 * spends no host time on them.  Synchronous; the scheduler state is unchanged. */
int mb_prepare(mb_ctx *ctx, int n_coarse);
/* The same for mb_step_diag(ctx, n), whose per-step result buffers it also
 * sizes, so that the diagnostic call allocates nothing either. */
int mb_prepare_diag(mb_ctx *ctx, int n_coarse);
/* evolution_area_stb (multi/FH/evolution_block.h:121) on one block. */
int mb_block_step(mb_ctx *ctx, int area, mb_stream stream);
/* Single interface operations, for per-kernel checks. */
int mb_c_c_boundary_transfer(mb_ctx *ctx, int line_cc, mb_stream stream);       /* assit_multi.h:2   */
int mb_space_interpolation(mb_ctx *ctx, int line, mb_stream stream);            /* assit_multi.h:187 */
int mb_temporal_interpolation(mb_ctx *ctx, int line, double xm, mb_stream s);   /* assit_multi.h:213 */
int mb_c_f_boundary_transfer(mb_ctx *ctx, int line, mb_stream stream);          /* assit_multi.h:249 */
int mb_f_c_boundary_transfer(mb_ctx *ctx, int line, mb_stream stream);          /* assit_multi.h:273 */
int mb_rotate_markers(mb_ctx *ctx, int line);                                   /* evolution.h:41-46 */

/* ---- diagnostics ----------------------------------------------------------- */
/* getDrag_block (lbm/force_block.h:180-216) without the file: force[2], Cd, Cl.
 * Blocks until the value is on the host. */
int mb_drag(mb_ctx *ctx, double force[2], double *cd, double *cl, mb_stream stream);
int mb_drag_link_count(mb_ctx *ctx, int *n_links);
/* error_L2 (lbm/error_L2.h:57-91) without the file; updates u_prev. */
int mb_error_L2(mb_ctx *ctx, double *e, mb_stream stream);
/* The reference's main loop (Multi-block-LBM.cu:144-158): n coarse steps,
 * each followed by getDrag_block and error_L2 (the same values as calling
 * mb_step(1), mb_drag and mb_error_L2 in turn), without a host round trip per
 * step: every step's results are copied to host memory asynchronously and
 * the call returns once the last one has arrived.  cd, cl and err receive n
 * values each; any of them may be NULL. */
int mb_step_diag(mb_ctx *ctx, int n, double *cd, double *cl, double *err, mb_stream stream);
/* Scans every block for NaN / Inf; *bad = number of bad values. */
int mb_check_finite(mb_ctx *ctx, long long *bad, mb_stream stream);

/* ---- host field access (FP64 host buffers, row-major i + j*nx) ------------ */
/* Any pointer may be NULL.  F is 9*nx*ny (plane k at k*nx*ny).  Synchronous. */
int mb_copy_fields(mb_ctx *ctx, int area, double *rho, double *ux, double *uy, double *F,
                   int *solid, mb_stream stream);
int mb_set_fields(mb_ctx *ctx, int area, const double *rho, const double *ux,
                  const double *uy, const double *F, mb_stream stream);
/* Tecplot POINT file in the layout of output/output.h:2-38. */
int mb_write_tecplot(mb_ctx *ctx, const char *path);
/* Line "t\tCd\tCl\t" / "t\terr" appended as in force_block.h:212-215 / error_L2.h:85-88. */
int mb_append_drag(const char *path, int t, double cd, double cl);
int mb_append_error_L2(const char *path, int t, double e);

/* ---- checkpoint / restart (no counterpart in the reference) -------------- */
/* The raw device state (both distribution buffers, rho/u, u_prev, ring slots,
 * scheduler state) in a caller-provided host buffer of mb_checkpoint_size
 * bytes; loading it into a context built from the same geometry and precision
 * restarts bit-exactly.  Both calls synchronise the stream. */
int mb_checkpoint_size(mb_ctx *ctx, long long *bytes);
int mb_checkpoint_save(mb_ctx *ctx, void *host, long long bytes, mb_stream stream);
int mb_checkpoint_load(mb_ctx *ctx, const void *host, long long bytes, mb_stream stream);

/* ---- relative L2 change without any device allocation -------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory: an application that owns the device through its own memory pool,
 * or a time-stepping loop that must not pay the device-wide synchronisation
 * of cudaMalloc/cudaFree.  The caller passes its own device arrays (FP64,
 * dense) per segment and a device output of 3 doubles:
 *   out[0] = sum over segments of weight * sum |u - u_prev|^2,
 *   out[1] = sum of weight * sum |u|^2,   out[2] = sqrt(out[0]) / sqrt(out[1]),
 * and u_prev <- u: with weight 1/m per block these are the two sums of the
 * relative L2 change that mb_error_L2 reports.  With no cells at all (every
 * n zero) out[0] = out[1] = 0 and out[2] is 0/0, a NaN.  Scratch is a fixed array inside the library (one copy per
 * device, kept until exit); the first call on a device looks up its address
 * and should come before any stream capture.  Calls share that array, so
 * calls that overlap on the GPU race.  Returns MB_ERR_UNSUPPORTED beyond the
 * limits below.  Asynchronous on `stream`. */
#define MB_L2_NOALLOC_MAX_SEGMENTS 64
#define MB_L2_NOALLOC_MAX_CTAS 1184
#define MB_L2_NOALLOC_MAX_CELLS (1LL << 40)
typedef struct {
  const double *ux, *uy; /* current velocity, n values each (device) */
  double *upx, *upy;     /* previous velocity (device); overwritten with ux, uy */
  long long n;           /* cells in this segment */
  double weight;         /* factor of this segment's sums */
} mb_l2_segment;
int mb_error_L2_noalloc(const mb_l2_segment *segs, int nseg, double *d_out, mb_stream stream);

/* ---- introspection ------------------------------------------------------- */
/* Text description of the plan that mb_step(ctx, n) starts with from the
 * current state (n >= period + 1: the plan of `period` coarse steps; else a
 * single step): one line per launch with its kind, level, region, grid,
 * scheduling class, label and the launches it waits for.  Writes at most
 * cap - 1 characters and a terminating zero; *len receives the full length.
 * No counterpart in the reference (whose order is the call order). */
int mb_plan_describe(mb_ctx *ctx, int n_coarse, char *buf, long long cap, long long *len);
/* Number of kernels launched by the last mb_step call, and in one coarse step. */
int mb_stats(mb_ctx *ctx, long long *kernels_last_step_call, long long *kernels_per_coarse_step,
             long long *cell_updates_per_coarse_step);
/* Times the fused block-step kernel of one level alone: n launches captured as
 * one CUDA graph, replayed once to warm up and once between CUDA events on a
 * private stream (after the given stream drains); returns mean ms per launch
 * and algorithmic bytes per launch. */
int mb_time_block_step(mb_ctx *ctx, int level, int n, mb_stream stream, double *ms_per_launch,
                       double *alg_bytes_per_launch, long long *cells_per_launch);

/* ---- batches of independent cases (no reference counterpart) ------------- */
/* Groups n initialised cases of one precision, one number of levels and one
 * scheduler state (e.g. all freshly initialised) for batched stepping: each
 * node of their common plan runs as one launch over all cases, and the plan
 * is replayed as a CUDA graph.  Cases whose plans differ in structure cannot
 * share a batch (MB_ERR_UNSUPPORTED from the first mb_batch_step).  The
 * cases stay owned by the caller and usable one by one; they are switched to
 * graph mode 1 and block-step variant 0. */
int mb_batch_create(mb_ctx *const *cases, int n, mb_batch **out);
int mb_batch_destroy(mb_batch *batch);
/* n coarse steps of every case (the last one leaves all rho/u up to date, as
 * mb_step).  MB_ERR_STATE if a case was stepped on its own since. */
int mb_batch_step(mb_batch *batch, int n_coarse, mb_stream stream);
/* Compiles the plans and graphs mb_batch_step(n) will replay from the
 * current state (the cases' plans on all host cores). */
int mb_batch_prepare(mb_batch *batch, int n_coarse);
/* Cd and Cl of every case (n values each; either may be NULL), one
 * synchronisation for the whole batch. */
int mb_batch_drag(mb_batch *batch, double *cd, double *cl, mb_stream stream);
/* Cell updates of one coarse step of all cases, launches of the last step
 * call, and coarse steps taken through the batch so far (the autotuner's
 * timing steps included). */
int mb_batch_stats(mb_batch *batch, long long *cell_updates_per_coarse_step, long long *kernels_last_call,
                   long long *coarse_steps_done);
/* mb_set_interface_shape on every case of the batch. */
int mb_batch_set_interface_shape(mb_batch *batch, int rec_points, int spline_segments);
/* Block-step schedule of the batch: 0 launches one CTA per tile of 256
 * cells (cases in order); k = 1..8 (1..4 in FP64) launches a persistent grid
 * of k CTAs per SM, each CTA taking an equal share of the tiles, in order.
 * Results are identical. */
int mb_batch_set_schedule(mb_batch *batch, int stb_ctas_per_sm);
/* Block-step kernel of the batch: 0 one cell per thread (default), 1 cell
 * pairs (a thread steps cells i, i+1 of a row, the single-case variant 4),
 * tiles of 256 pairs under the same schedule; nodes where a case's launch
 * does not fit the pair form (block rims, 32-bit offsets exceeded) keep one
 * cell per thread.  Results are identical. */
int mb_batch_set_kernel(mb_batch *batch, int kernel);
/* Autotuner: times the block-step kernels and schedules (one cell per
 * thread at 0, 2, 4, 8 CTAs per SM; cell pairs at 0, 2, 4), then with the
 * fastest the interface shapes (points per record CTA, spline segments per
 * CTA), each over `steps` coarse steps, and keeps the fastest; reports the
 * choice and its time per coarse step (any pointer may be NULL).  The timing
 * steps advance the cases. */
int mb_batch_autotune(mb_batch *batch, int steps, mb_stream stream, int *rec_points, int *spline_segments,
                      int *stb_ctas_per_sm, double *ms_per_step, int *stb_kernel);

/* ---- learned warm start (no reference counterpart) ----------------------- */
/* A 4-level convolutional U-Net (3x3 convolutions with ReLU, 32, 64, 128,
 * 256 channels, 2x2 average pooling, nearest upsampling with skip
 * concatenation, a 1x1 head to 3 outputs) on an H x W grid (multiples of 8).
 * BF16 weights and activations, FP32 accumulation on the tensor cores, FP32
 * master weights updated by Adam.  Inputs are 4 FP32 channels per point
 * (NHWC, device memory): signed distance to the obstacle / D, Re / 100,
 * inside-obstacle flag, x / W.  Outputs are 3 FP32 channels: u / U0, v / U0,
 * 100 (rho - 1).  He-normal initialisation from `seed`. */
typedef struct mb_unet mb_unet;
int mb_unet_create(int H, int W, int max_batch, unsigned long long seed, mb_unet **out);
int mb_unet_destroy(mb_unet *net);
int mb_unet_param_count(mb_unet *net, long long *count);
/* which = 0: FP32 master weights; 1: gradients of the last train step. */
int mb_unet_get_params(mb_unet *net, float *host, long long count, int which);
int mb_unet_set_params(mb_unet *net, const float *host, long long count);
/* 3x3 convolutions (forward and input gradient) on the tcgen05 tensor cores
 * (kind 1, the default; layers whose shape does not fit fall back per layer)
 * or on mma.sync (kind 0). */
int mb_unet_set_gemm(mb_unet *net, int kind);
/* MB_ERR_TIMEOUT (once) when a tcgen05 kernel's bounded wait ran out since
 * the last call; synchronises the stream. */
int mb_unet_status(mb_unet *net, mb_stream stream);
/* d_in: [n][H][W][4], d_out: [n][H][W][3], FP32 device arrays. */
int mb_unet_forward(mb_unet *net, const float *d_in, int n, float *d_out, mb_stream stream);
/* Forward, masked squared error sum_p mask_p |y_p - t_p|^2 / (3 n H W)
 * against d_target ([n][H][W][3]) with d_mask ([n][H][W]), backward, and
 * (apply = 1) one Adam step with learning rate lr.  Synchronous; *loss is
 * the loss before the update. */
int mb_unet_train_step(mb_unet *net, const float *d_in, const float *d_target, const float *d_mask, int n, float lr,
                       int apply, float *loss, mb_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* MBLBM_H */
