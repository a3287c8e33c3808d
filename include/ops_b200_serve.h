/*
 * ops_b200_serve.h -- solve-serving engine (no counterpart in the reference;
 * an added form of the backend).
 *
 * Requests are independent solves that arrive over time:
 *   OB2S_POISSON2D  -lap(u) = f on an n x n grid (5-point, zero Dirichlet
 *                   boundary), f ~ U(-1,1) from the request's seed; solved by
 *                   conjugate gradients to a relative residual tolerance
 *                   ||h^2 f - A u|| / ||h^2 f|| <= tol;
 *   OB2S_HEAT2D     `steps` backward-Euler steps of the 2D heat equation on
 *                   an n x n grid with dt = h^2: each step solves
 *                   5 u' - (sum of the 4 neighbours of u') = u by conjugate
 *                   gradients to `tol` relative to that step's right-hand
 *                   side, from u0 ~ U(-1,1) (the seed), zero Dirichlet
 *                   boundary;
 *   OB2S_ADI3D      `steps` steps of the 3D ADI heat scheme on an n^3 grid
 *                   (the reference's adi app: preproc_kernel.h, then
 *                   tridiagonal solves along x, y and z with the z solution
 *                   added to u), u0 ~ U(-1,1) from the seed.
 *
 * Every admitted request keeps its arrays resident in HBM until released.
 * All active requests advance together: one engine iteration is one launch
 * of each batched kernel over a device-side work list that spans every
 * active request (ragged sizes share the launch), and the CG scalars live on
 * the device, so an iteration needs no host round trip.  `ob2s_run` replays
 * one CUDA graph of K iterations; the graph reads the work list from device
 * memory, so it stays valid when requests join or leave (continuous
 * batching: new requests join at the next ob2s_run, finished ones stop
 * consuming work immediately).
 *
 * Precision modes (conjugate gradients, FP64 iterate x):
 *   OB2S_FP64   CG in FP64 (the plain form);
 *   OB2S_MIXED  FP32 CG vectors r, w, p and their arithmetic (dot
 *               products accumulated in FP64), FP64 iterate x updated in
 *               FP64; whenever the recursive residual has dropped by
 *               `inner_tol` since the last true residual (or meets `tol`),
 *               the residual is replaced by b - A x computed in FP64
 *               (iterative refinement that keeps the Krylov directions);
 *               convergence is tested on that FP64 residual.
 * Both modes use the same replacement schedule; `max_inner` caps the CG
 * iterations of a request.
 * ADI requests run in FP64 in both modes (constant coefficients: only u and
 * the right-hand side are stored, 16 B per point per solve).
 *
 * Each request's arithmetic depends only on its own data and its own tile
 * decomposition, with partial sums combined in a fixed order, so a request's
 * result is bit-identical alone and in any mix.
 *
 * All functions return 0 or a cudaError_t value (OB2S_ERR_* for engine
 * errors); ob2_error_string (ops_b200_device.h) names CUDA codes.
 */
#ifndef OPS_B200_SERVE_H
#define OPS_B200_SERVE_H

#include <stddef.h>

#include "ops_b200_device.h"

enum { OB2S_POISSON2D = 0, OB2S_ADI3D = 1, OB2S_HEAT2D = 2 };
enum { OB2S_FP64 = 0, OB2S_MIXED = 1 };

#define OB2S_MAX_ACTIVE 128
#define OB2S_ERR_FULL 200001     /* no free request slot */
#define OB2S_ERR_BADARG 200002   /* kind / size / id out of range */
#define OB2S_ERR_NOTDONE 200003  /* result asked for an unfinished request */

typedef struct ob2s_engine ob2s_engine;

typedef struct ob2s_result {
  int kind, n, done;
  int iterations;      /* CG iterations (all time steps of a heat request) / ADI steps */
  int outer;           /* residual evaluations in FP64 (refinement passes) */
  double rel_residual; /* final FP64 relative residual (Poisson) */
  double checksum;     /* sum of the interior solution */
} ob2s_result;

/* tile_y: rows of a Poisson tile (8, 16 or 32 = 1, 2 or 4 rows per thread of
 * a 32 x 8 CTA; 0 = 32). */
OB2_API int ob2s_create(ob2s_engine **e, int mode, double tol, double inner_tol, int max_inner,
                        int tile_y);
OB2_API void ob2s_destroy(ob2s_engine *e);
/* grows the engine's memory pool to `bytes` once (a server's start-up: the
 * requests admitted later are carved from memory already mapped instead of
 * mapping their own); the pool keeps freed memory for the engine's life */
OB2_API int ob2s_reserve(ob2s_engine *e, size_t bytes);
/* device bytes a request holds while admitted */
OB2_API size_t ob2s_request_bytes(int mode, int kind, int n);
/* Allocates and initialises a request (stream-ordered); it joins the active
 * set at the next ob2s_run.  steps: ADI or heat time steps (ignored for
 * Poisson). */
OB2_API int ob2s_submit(ob2s_engine *e, int kind, int n, int seed, int steps, int *id);
/* Runs `iters` engine iterations (a graph of that many is captured once per
 * value and replayed) and waits for them; *n_done: requests finished since
 * the last call, their ids in ids[0..cap). */
OB2_API int ob2s_run(ob2s_engine *e, int iters, int *ids, int cap, int *n_done);
OB2_API int ob2s_active(ob2s_engine *e);
OB2_API int ob2s_result_of(ob2s_engine *e, int id, ob2s_result *res);
/* interior solution of a finished request into host memory (n^2 or n^3) */
OB2_API int ob2s_fetch(ob2s_engine *e, int id, double *host, size_t count);
/* frees the request's device memory and its slot */
OB2_API int ob2s_release(ob2s_engine *e, int id);
/* kernel launches issued by the engine (graph replays count their kernels) */
OB2_API long long ob2s_launches(ob2s_engine *e);

#endif /* OPS_B200_SERVE_H */
