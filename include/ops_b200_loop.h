/*
 * ops_b200_loop.h -- ABI between translator-generated par_loop stubs and the
 * host runtime.
 *
 * Replaces the per-loop host logic of the reference's generated CUDA stub
 * (ops_translator/resources/templates/cpp/cuda/loop_host.cpp.j2:13-780):
 * range/start computation, H->D dirty-bit exchange, reduction staging,
 * base-pointer computation, dirty-bit update and timing.  The stub calls
 * ob2_loop_begin, launches its own kernel with the views it gets back, and
 * calls ob2_loop_end.
 */
#ifndef OPS_B200_LOOP_H
#define OPS_B200_LOOP_H

#include "ops_lib_core.h"
#include "ops_b200_device.h"

#define OB2_MAX_ARGS 48

/* Where one dat argument lives for the loop:
 *   element of loop point (x,y,z) = base + x*wx + y*wy + z*wz   (elements)
 *   ACC strides ex/ey/ez/ed: neighbours along x/y/z and between components. */
typedef struct ob2_view {
  char *base;
  long long wx, wy, wz;
  int ex, ey, ez, ed;
  /* 4D / 5D blocks: the walk and the ACC strides along the 4th and 5th axes
   * (element of point (x,y,z,u,v) = base + x*wx + y*wy + z*wz + u*wu + v*wv) */
  long long wu, wv;
  int eu, ev;
} ob2_view;

/* reduction target of one ops_arg_reduce */
typedef struct ob2_red {
  void *acc;    /* device accumulator of the handle (dim values) */
  int first;    /* 1: this loop initialises the accumulator */
  int op;       /* OPS_INC / OPS_MIN / OPS_MAX */
} ob2_red;

/* A generated fused launcher (one per application): runs n (<= OB2_FUSE_MAX)
 * different loops of the application in one launch, loop k being the
 * application's loop ids[k] with parameter block params[k] (psize[k] bytes,
 * each rounded up to 16, together at most OB2_FUSE_BLOB) over its own grid
 * grids[3k..3k+2]; every loop takes the CTA shape `block`.  idx32: every
 * loop has 32-bit element offsets.  The runtime only passes loops that touch
 * no common point of a dat that one of them writes. */
#define OB2_FUSE_MAX 16
#define OB2_FUSE_BLOB 8192
typedef int (*ob2_flauncher)(int n, const int *ids, const void *const *params,
                             const size_t *psize, const unsigned *grids, const unsigned *block,
                             int idx32, void *stream);

/* A halo group folded into the launch of the loop that consumes it (the
 * multi-block case: ops_halo_transfer followed by a loop over the blocks
 * that reads the halos just filled).  Each CTA first copies the group's
 * cells that fall in its own footprint (its tile widened by the loop's
 * stencil reach), then runs the loop; the runtime folds a group only when
 * every cell of it lies in some footprint and the loop writes no dat the
 * group reads or fills, so the result equals running the transfer first.
 * Entry e: task task[e] of the group's device task table, whose destination
 * is read by instance inst[e] of the launch; org[e] is the loop coordinate
 * of the destination dat's storage index 0 along each axis. */
#define OB2_HFUSE_MAX 32
typedef struct ob2_hfuse {
  const ob2_halo_task *tasks;
  int n;
  int task[OB2_HFUSE_MAX];
  int inst[OB2_HFUSE_MAX];
  int org[OB2_HFUSE_MAX][3];
  int mlo[3], mhi[3];  /* stencil reach below / above along each axis (>= 0) */
} ob2_hfuse;
/* A generated halo-folding launcher: as ob2_mlauncher, with the folded
 * group h. */
typedef int (*ob2_hlauncher)(const void *const *params, int n, const unsigned *grid,
                             const unsigned *block, const ob2_hfuse *h, void *stream);

/* Shared-memory temporal blocking of a chain of sweeps (the GPU form of the
 * reference's loop-chain tiling, ops_lazy.cpp:380-1187): consecutive queued
 * instances of one 2D loop that ping-pong two dats -- sweep k reads dat X
 * through a stencil of reach at most 1 and writes dat Y at the centre,
 * sweep k+1 the other way round, everything else equal -- run `steps` sweeps
 * in one launch.  Each CTA loads its tile widened by `steps` into shared
 * memory (X, and Y outside the loop range), runs the sweeps there on
 * shrinking regions with the loop's own point function, and writes the
 * tile back: Y's new values in place, X's into X's spare buffer (`spare`:
 * the view base of arg s in it), which then becomes X's storage (no CTA
 * writes X while another may still read it).  The CTAs on the range edge
 * also copy X's points outside the range (storage box sx0..sx1 x sy0..sy1
 * in loop coordinates) into the spare.  Every point is computed by the same
 * code on the same values as sweep by sweep, so results are identical. */
#define OB2_TB_MAX 8
typedef struct ob2_tblock {
  int steps;       /* sweeps in this launch, 2..OB2_TB_MAX */
  int s;           /* argument index of X (the stencil-read dat of the first sweep) */
  char *spare;     /* view base of argument s in X's spare buffer */
  int sx0, sx1, sy0, sy1;
} ob2_tblock;
typedef int (*ob2_tlauncher)(const void *params, const ob2_tblock *t, void *stream);

typedef struct ob2_loop {
  const char *name;
  int kernel_index;  /* timing-table slot */
  int dim;
  int lo[3], hi[3];
  int n[3];          /* hi - lo (clamped at 0) */
  long long npoints;
  void *stream;
  int nargs;
  ops_arg *args;
  ob2_view view[OB2_MAX_ARGS];
  ob2_red red[OB2_MAX_ARGS];
  void *partials;           /* device scratch: per-CTA reduction partials */
  size_t partials_bytes;
  unsigned int *counter;    /* device: CTAs finished (last-CTA combine) */
  void *ev_start, *ev_end;  /* timing events (diagnostics level > 1) */
  double host_t0;
  int block[3];             /* suggested CTA shape */
  int grid[3];              /* suggested grid: x covers the range, y/z capped
                               at about one full wave of resident CTAs; the
                               kernel loops over the remaining y/z */
  int idx32;                /* 1: every dat has < 2^31 elements, so element
                               offsets fit 32-bit arithmetic */
  int tune;                 /* >= 0: this launch times block-shape candidate
                               `tune` of the autotuner (OPS_B200_AUTOTUNE) */
  unsigned prolong_mask;    /* set by the stub BEFORE ob2_loop_begin: bit i =
                               argument i has a prolong stencil and the
                               generated code divides the loop index by its
                               multigrid stride */
  int fuse_id;              /* the loop's id in the fused launcher, -1: none */
  ob2_flauncher ffn;        /* the application's fused launcher (set by the
                               stub before ob2_launch; NULL: none) */
  ob2_hlauncher hfn;        /* the loop's halo-folding launcher (set by the
                               stub before ob2_launch; NULL: none) */
  ob2_tlauncher tfn;        /* the loop's temporal-blocking launcher (2D loops
                               with one written dat; NULL: none) */
  const size_t *tb_off;     /* byte offset of each dat argument's view base
                               in the parameter block (tfn != NULL) */
  const int *tb_role;       /* per argument: 1 a read dat the chain may
                               ping-pong, 2 the written dat, 0 other */
  int lo4[2], hi4[2];       /* 4D / 5D blocks: the range along the 4th and
                               5th axes (0 / 1 for fewer dimensions); the
                               suggested grid's z extent covers the product
                               of the extents along the 3rd to 5th axes */
} ob2_loop;

/* A generated launcher: launches one kernel variant with the parameter block
 * `params` (which starts with int lo[3], hi[3]: the loop range) on `stream`. */
typedef int (*ob2_launcher)(const void *params, const unsigned *grid, const unsigned *block,
                            void *stream);
/* A generated multi-instance launcher: runs n (<= OB2_MULTI_MAX) instances
 * of one loop in one launch, instance k with params[k]; grid is the largest
 * instance grid (the launch's z extent is n times grid[2]). */
#define OB2_MULTI_MAX 8
typedef int (*ob2_mlauncher)(const void *const *params, int n, const unsigned *grid,
                             const unsigned *block, void *stream);

/* Launch or queue one par_loop kernel.  Eager mode (OPS_B200_LAZY=0)
 * launches now.  In lazy mode (the default) loops without reductions are
 * queued with a copy of their parameters, halo transfers are queued with
 * them, and the queue runs at the next flush point: a reduction loop,
 * ops_reduction_result's loop, a constant, a solve, any call that moves data
 * between host and device or hands out a raw pointer, ops_execute, ops_timers,
 * or 64 queued items (OPS_B200_MAX_CHAIN).  A flushed chain is captured as a
 * CUDA graph and replayed when the same chain recurs (OPS_B200_GRAPHS=0:
 * plain launches).  With OPS_TILING (or OPS_B200_TILING=1) the chain runs
 * tile by tile: skewed tiles along the slowest axis sized for the L2 budget
 * OPS_CACHE_SIZE (MB), the GPU form of the reference's loop-chain tiling,
 * ops_lazy.cpp:380-1187.  Consecutive queued instances of one loop with
 * no data shared between them (the blocks of a multi-block program) run as
 * one launch of mfn (may be NULL: loops with reductions).  Consecutive
 * queued small loops (up to OPS_B200_FUSE_PTS points each, default 65536)
 * that share no point of a dat that one of them writes -- each loop writes
 * its range and reads its range shifted by every stencil point -- run as one
 * launch of the application's fused launcher L->ffn (OPS_B200_FUSE=0: off);
 * the boundary loops of a halo update are the typical case.  A queued halo
 * transfer followed by a run of instances whose loop reads the halos it
 * fills is folded into that run's launch (L->hfn, ob2_hfuse;
 * OPS_B200_HFUSE=0: off).  A run of sweeps at the end of the queue that
 * ping-pong two dats runs through L->tfn in launches of up to
 * OPS_B200_TB_DEPTH sweeps (ob2_tblock; OPS_B200_TB=0: off).
 * rows_per_thread: points each thread covers along y (the grid's y extent
 * is derived from it per tile). */
OPS_API void ob2_launch(ob2_loop *L, ob2_launcher fn, ob2_mlauncher mfn, const void *params,
                        size_t psize, const unsigned *grid, const unsigned *block,
                        int rows_per_thread);

/* Runs everything the lazy queue holds (no-op in eager mode). */
OPS_API void ob2_flush(void);

/* Returns 0 when the range is empty (nothing to launch, ob2_loop_end not
 * needed), 1 otherwise. */
OPS_API int ob2_loop_begin(ob2_loop *L, const char *name, ops_block block, int dim,
                           const int *range, ops_arg *args, int nargs);
OPS_API void ob2_loop_end(ob2_loop *L);
/* 1 when some dat is passed more than once and written through one of the
 * arguments: the loop's kernel must then not assume its dat pointers are
 * unaliased. */
OPS_API int ob2_args_alias(const ops_arg *args, int nargs);
/* Checks the launch just issued; throws OPSException on error. */
OPS_API void ob2_loop_check_launch(ob2_loop *L);

/* Per-kernel device timing.  While enabled, every launch (par_loops, halo
 * transfers, tridiagonal solves) is bracketed by CUDA events on the work
 * stream without any host synchronisation.  ob2_ktime_report resolves them
 * and writes one line per kernel: "name launches device_ms algorithmic_bytes"
 * (bytes by the OPS transfer model, ops_lib_core.cpp:1687-1697), returning
 * the full length.  ob2_ktime_reset clears the counters of every kernel. */
OPS_API void ob2_ktime_enable(int on);
OPS_API void ob2_ktime_reset(void);
OPS_API size_t ob2_ktime_report(char *buf, size_t n);
/* Kernels launched by the runtime since ops_init. */
OPS_API long long ob2_launch_count(void);

/* Constant registry: the generated kernels file registers one callback that
 * copies a named constant into its __constant__ symbol. */
typedef int (*ob2_const_fn)(const char *name, int dim, int type_size, const char *data,
                            void *stream);
OPS_API void ob2_register_const_handler(ob2_const_fn fn);

#endif /* OPS_B200_LOOP_H */
