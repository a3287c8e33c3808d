/*
 * ops_tridiag.h -- batched tridiagonal solves over ops_dats.
 *
 * Replaces ops/c/include/ops_tridiag.h:45-83 of the reference.  The reference
 * forwards these calls to the external tridsolver library
 * (ops/c/src/tridiag/ops_tridiag.cpp:78-249, ops_tridiag_cuda.cpp:96-251);
 * this backend solves them with its own sm_100a kernels.
 *
 * Semantics (reference doc/opsapi.md:882-912):
 *   ops_tridMultiDimBatch     a x_{i-1} + b x_i + c x_{i+1} = d along
 *                             `solvedim` for every line inside `range`;
 *                             the solution overwrites d.
 *   ops_tridMultiDimBatch_Inc same system; the solution is added to u and d
 *                             is left unchanged.
 * a[first] and c[last] of every line are ignored.  a, b, c, d (and u) must
 * have the same sizes and type ("double" or "float").
 */
#ifndef OPS_B200_TRIDIAG_H
#define OPS_B200_TRIDIAG_H

#include "ops_lib_core.h"

#ifdef __cplusplus
class ops_tridsolver_params {
 public:
  enum SolveStrategy {
    GATHER_SCATTER = 0,
    ALLGATHER,
    JACOBI,
    PCR,
    LATENCY_HIDING_INTERLEAVED,
    LATENCY_HIDING_TWO_STEP
  };
  ops_tridsolver_params(ops_block block) : block_(block), strategy_(PCR) {}
  ops_tridsolver_params(ops_block block, SolveStrategy s) : block_(block), strategy_(s) {}
  ~ops_tridsolver_params() {}
  /* distributed-solve knobs of the reference; single GPU: recorded, unused */
  void set_jacobi_params(double rtol, double atol, int maxiter) {
    rtol_ = rtol; atol_ = atol; maxiter_ = maxiter;
  }
  void set_batch_size(int b) { batch_ = b; }
  void set_cuda_opts(int x, int y, int z) { opts_[0] = x; opts_[1] = y; opts_[2] = z; }
  void set_cuda_sync(int s) { sync_ = s; }
  void *tridsolver_params = nullptr;

 private:
  ops_block block_;
  SolveStrategy strategy_;
  double rtol_ = 0, atol_ = 0;
  int maxiter_ = 0, batch_ = 0, sync_ = 0;
  int opts_[3] = {0, 0, 0};
};
#else
typedef struct ops_tridsolver_params ops_tridsolver_params;
#endif

/* ops_tridiag.h:75-77 */
OPS_API void ops_tridMultiDimBatch(int ndim, int solvedim, int *range, ops_dat a, ops_dat b,
                                   ops_dat c, ops_dat d, ops_tridsolver_params *ctx);
/* ops_tridiag.h:80-83 */
OPS_API void ops_tridMultiDimBatch_Inc(int ndim, int solvedim, int *range, ops_dat a,
                                       ops_dat b, ops_dat c, ops_dat d, ops_dat u,
                                       ops_tridsolver_params *ctx);

#endif /* OPS_B200_TRIDIAG_H */
