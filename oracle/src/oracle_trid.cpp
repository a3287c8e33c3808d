/*
 * ORACLE -- test infrastructure only.
 *
 * CPU restatement of the batched tridiagonal solve behind
 * ops_tridMultiDimBatch(_Inc).  The reference wrapper
 * (ops/c/src/tridiag/ops_tridiag.cpp:78-249) checks sizes/types, forms the
 * line box from `range` and calls the external tridsolver library
 * (tridDmtsvStridedBatch / tridDmtsvStridedBatchInc, github.com/OP-DSL/
 * tridsolver, not vendored and not version-pinned by the reference).  This
 * restates the published scalar Thomas algorithm that library applies per
 * line (forward elimination c'_i = c_i / (b_i - a_i c'_{i-1}),
 * d'_i = (d_i - a_i d'_{i-1}) / (b_i - a_i c'_{i-1}), back substitution
 * x_i = d'_i - c'_i x_{i+1}) in FP64, for double and float dats.
 *
 * Parity of this solve is unpinned by the reference (no vendored solver, no
 * golden output); it is pinned here by residual checks in the tests.
 */
#include <vector>

#include "ops_lib_core.h"
#include "ops_tridiag.h"

namespace {

template <typename T>
void solve_all(int ndim, int solvedim, const int *range, ops_dat a, ops_dat b, ops_dat c,
               ops_dat d, ops_dat u) {
  long long str[3] = {1, a->size[0], (long long)a->size[0] * a->size[1]};
  int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  for (int i = 0; i < ndim; i++) {
    lo[i] = range[2 * i];
    hi[i] = range[2 * i + 1];
  }
  /* origin of interior point (0,0,0) in storage, as ops_dat_get_raw_pointer */
  long long org = 0;
  for (int i = 0; i < ndim; i++) org += (long long)(-a->d_m[i] - a->base[i]) * str[i];
  const T *A = (const T *)a->data, *B = (const T *)b->data, *C = (const T *)c->data;
  T *D = (T *)d->data;
  T *U = u ? (T *)u->data : nullptr;
  int n = hi[solvedim] - lo[solvedim];
  if (n <= 0) return;
  std::vector<double> cp(n), dp(n);
  int o1 = (solvedim + 1) % 3, o2 = (solvedim + 2) % 3;
  for (int j = lo[o2]; j < hi[o2]; j++)
    for (int i = lo[o1]; i < hi[o1]; i++) {
      int idx[3];
      idx[o1] = i;
      idx[o2] = j;
      idx[solvedim] = lo[solvedim];
      long long p0 = org + idx[0] * str[0] + idx[1] * str[1] + idx[2] * str[2];
      long long s = str[solvedim];
      double m = 1.0 / (double)B[p0];
      cp[0] = (double)C[p0] * m;
      dp[0] = (double)D[p0] * m;
      for (int k = 1; k < n; k++) {
        long long p = p0 + k * s;
        m = 1.0 / ((double)B[p] - (double)A[p] * cp[k - 1]);
        cp[k] = (double)C[p] * m;
        dp[k] = ((double)D[p] - (double)A[p] * dp[k - 1]) * m;
      }
      for (int k = n - 2; k >= 0; k--) dp[k] = dp[k] - cp[k] * dp[k + 1];
      for (int k = 0; k < n; k++) {
        long long p = p0 + k * s;
        if (U)
          U[p] = (T)((double)U[p] + dp[k]);
        else
          D[p] = (T)dp[k];
      }
    }
}

void check(int ndim, ops_dat a, ops_dat b, ops_dat c, ops_dat d, ops_dat u) {
  for (int i = 0; i < ndim; i++)
    if (a->size[i] != b->size[i] || b->size[i] != c->size[i] || c->size[i] != d->size[i] ||
        (u && u->size[i] != d->size[i]))
      throw OPSException(OPS_RUNTIME_ERROR,
                         "Tridsolver error: the a,b,c,d datasets all need to be the same size");
  if (strcmp(a->type, b->type) || strcmp(b->type, c->type) || strcmp(c->type, d->type) ||
      (u && strcmp(d->type, u->type)))
    throw OPSException(OPS_RUNTIME_ERROR,
                       "Tridsolver error: the a,b,c,d datasets must all be of the same type");
}

void dispatch(int ndim, int solvedim, int *range, ops_dat a, ops_dat b, ops_dat c, ops_dat d,
              ops_dat u) {
  if (ndim < 1 || ndim > 3 || solvedim < 0 || solvedim >= ndim)
    throw OPSException(OPS_INVALID_ARGUMENT, "Tridsolver error: bad ndim/solvedim");
  check(ndim, a, b, c, d, u);
  if (!strcmp(a->type, "double"))
    solve_all<double>(ndim, solvedim, range, a, b, c, d, u);
  else if (!strcmp(a->type, "float"))
    solve_all<float>(ndim, solvedim, range, a, b, c, d, u);
  else
    throw OPSException(OPS_RUNTIME_ERROR,
                       "Tridsolver error: unsupported type. Dataset type must either be "
                       "\"double\" or \"float\"");
}

} // namespace

OPS_API void ops_tridMultiDimBatch(int ndim, int solvedim, int *range, ops_dat a, ops_dat b,
                                   ops_dat c, ops_dat d, ops_tridsolver_params *) {
  dispatch(ndim, solvedim, range, a, b, c, d, nullptr);
}

OPS_API void ops_tridMultiDimBatch_Inc(int ndim, int solvedim, int *range, ops_dat a,
                                       ops_dat b, ops_dat c, ops_dat d, ops_dat u,
                                       ops_tridsolver_params *) {
  dispatch(ndim, solvedim, range, a, b, c, d, u);
}
