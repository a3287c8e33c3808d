/*
 * ORACLE -- test infrastructure only.  Not part of the product, never linked
 * into libops_b200.so; only tests/, the smoke check and the CPU-baseline leg
 * of bench.py build against it.
 *
 * CPU restatement of the OPS sequential par_loop (the "dev_seq" path):
 *   ops/c/include/ops_seq_v2.h:211-334   ops_par_loop_impl / ops_par_loop
 *   ops/c/include/ops_seq_v2.h:55-62     address(): byte offset of a point
 *   ops/c/include/ops_seq_v2.h:156-195   param_handler: what each kernel
 *                                         parameter receives (ACC, gbl, idx)
 *
 * Semantics restated:
 *   - the kernel runs once per point of the half-open range, x fastest;
 *   - an ACC argument points at element
 *       sum_i (idx_i*stride_i - base_i - d_m_i) * prod_{j<i} size_j
 *     (times the component count for AoS dats), offsets inside the kernel are
 *     raw element offsets along each axis;
 *   - an OPS_READ global gets the caller's pointer, a reduction gets the
 *     handle's own buffer (so the kernel accumulates in place, sequentially);
 *   - ops_arg_idx gets the global index of the current point.
 * Apps include this header exactly like the reference's dev_seq header.
 */
#ifndef OPS_ORACLE_SEQ_V2_H
#define OPS_ORACLE_SEQ_V2_H

#include <tuple>
#include <type_traits>
#include <utility>

#include "ops_lib_core.h"
#include "ops_tridiag.h"

/* oracle runtime hooks (oracle/src/oracle_core.cpp) */
OPS_API void oracle_loop_prologue(const char *name, ops_block block, int dim, const int *range,
                                  ops_arg *args, int nargs);
OPS_API void oracle_loop_epilogue(const char *name, ops_block block, int dim, const int *range,
                                  ops_arg *args, int nargs);
OPS_API int oracle_soa(void);
/* slab decomposition over ranks (ops_b200_dist.h): halo exchanges before the
 * loop and its range clipped to this rank's rows along the slowest axis */
OPS_API void oracle_dist_loop(const char *name, ops_block block, int dim, int *lo, int *hi,
                              ops_arg *args, int nargs);

namespace ops_oracle {

template <typename P> struct holder {
  /* pointer parameters: ops_arg_gbl / ops_arg_reduce / ops_arg_idx */
  typedef typename std::decay<P>::type PT;
  PT v;
  void set(const ops_arg &a, const int *gidx, const int *, ops_block) {
    if (a.argtype == OPS_ARG_GBL)
      v = (a.acc == OPS_READ) ? (PT)a.data : (PT)((ops_reduction)a.data)->data;
    else if (a.argtype == OPS_ARG_IDX)
      v = (PT)gidx;
    else
      v = (PT)0;
  }
  PT get() { return v; }
};

template <typename T> struct acc_holder {
  ACC<T> a;
  void set(const ops_arg &arg, const int *, const int *pt, ops_block block) {
    // a disabled optional argument still points at its dat, as in the
    // reference's sequential backend (the flag only matters to halo exchanges)
    if (arg.argtype != OPS_ARG_DAT || arg.dat == NULL) {
      a = ACC<T>();
      return;
    }
    ops_dat d = arg.dat;
    const int nd = block->dims;
    const int soa = oracle_soa();
    long long off = 0, cum = 1;
    for (int i = 0; i < nd; i++) {
      off += cum * (long long)(pt[i] * arg.stencil->stride[i] - d->base[i] - d->d_m[i]);
      cum *= d->size[i];
    }
    const int md = d->dim;
    int sx, sy, sz, sd;
    // points before the 4th and 5th axes (4D / 5D blocks)
    const long long c3 = (long long)d->size[0] * d->size[1] * d->size[2];
    const long long c4 = c3 * d->size[3];
    int su, sv;
    if (soa) {
      sx = 1; sy = d->size[0]; sz = d->size[0] * d->size[1];
      su = (int)c3; sv = (int)c4;
      sd = (int)cum;
    } else {
      off *= md;
      sx = md; sy = d->size[0] * md; sz = d->size[0] * d->size[1] * md;
      su = (int)(c3 * md); sv = (int)(c4 * md);
      sd = 1;
    }
    a = ACC<T>((T *)d->data + off, sx, sy, sz, su, sv, sd);
  }
  ACC<T> &get() { return a; }
};

template <typename P> struct pick {
  typedef holder<P> type;
};
template <typename T> struct pick<ACC<T> &> {
  typedef acc_holder<T> type;
};
template <typename T> struct pick<const ACC<T> &> {
  typedef acc_holder<T> type;
};
template <typename T> struct pick<ACC<T>> {  // ACC taken by value
  typedef acc_holder<T> type;
};
template <typename T> struct pick<const ACC<T>> {
  typedef acc_holder<T> type;
};

template <typename... P, size_t... I>
void run(void (*kernel)(P...), std::index_sequence<I...>, const char *name, ops_block block,
         int dim, int *range, ops_arg *args) {
  constexpr int N = sizeof...(P);
  oracle_loop_prologue(name, block, dim, range, args, N);
  std::tuple<typename pick<P>::type...> h;
  int lo[OPS_MAX_DIM] = {0, 0, 0, 0, 0}, hi[OPS_MAX_DIM] = {1, 1, 1, 1, 1};
  for (int i = 0; i < dim && i < OPS_MAX_DIM; i++) {
    lo[i] = range[2 * i];
    hi[i] = range[2 * i + 1];
  }
  oracle_dist_loop(name, block, dim, lo, hi, args, N);
  int pt[OPS_MAX_DIM] = {0, 0, 0, 0, 0};
  int gidx[OPS_MAX_DIM] = {0, 0, 0, 0, 0};
  for (int v = lo[4]; v < hi[4]; v++)
    for (int u = lo[3]; u < hi[3]; u++)
      for (int z = lo[2]; z < hi[2]; z++)
        for (int y = lo[1]; y < hi[1]; y++)
          for (int x = lo[0]; x < hi[0]; x++) {
            pt[0] = x; pt[1] = y; pt[2] = z; pt[3] = u; pt[4] = v;
            gidx[0] = x; gidx[1] = y; gidx[2] = z; gidx[3] = u; gidx[4] = v;
            (void)std::initializer_list<int>{
                (std::get<I>(h).set(args[I], gidx, pt, block), 0)...};
            kernel(std::get<I>(h).get()...);
          }
  oracle_loop_epilogue(name, block, dim, range, args, N);
}

} /* namespace ops_oracle */

template <typename... P, typename... A>
void ops_par_loop(void (*kernel)(P...), char const *name, ops_block block, int dim, int *range,
                  A... arguments) {
  static_assert(sizeof...(P) == sizeof...(A), "kernel parameter / argument count mismatch");
  ops_arg args[sizeof...(A)] = {arguments...};
  ops_oracle::run(kernel, std::index_sequence_for<P...>{}, name, block, dim, range, args);
}

#endif /* OPS_ORACLE_SEQ_V2_H */
