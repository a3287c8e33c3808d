/*
 * ops_b200_dist.h -- slab decomposition of an OPS program over ranks (one
 * process per GPU), no counterpart as a header in the reference: it takes
 * the place of the reference's MPI layer for single-block programs
 * (ops/c/src/mpi/ops_mpi_partition.cpp: the decomposition;
 * ops_mpi_rt_support.cpp:836 ops_exchange_halo and its Isend/Irecv pairs,
 * :1122-1136; the MPI_Allreduce of reduction results in
 * ops_mpi_rt_support.cpp).
 *
 * Every block is cut along its slowest axis (y in 2D, z in 3D) into
 * contiguous slabs, rank r owning block rows [r G / R, (r + 1) G / R) of the
 * block's extent G (the interior extent of the first dat declared on it);
 * the first rank also owns the rows below the interior, the last rank those
 * above.  Each rank allocates, for every dat, only its owned rows plus H
 * rows on each inner side (H = the dat's halo depth along that axis, at
 * least 1), and keeps the dat's global metadata (size, d_m, d_p, base):
 * the device pointer is offset so that global storage indices address the
 * local rows.  A par_loop runs over its range clipped to the owned rows; a
 * dat read through a stencil that reaches along the split axis has its H
 * inner halo rows refreshed from the neighbouring ranks first when it was
 * written since its last exchange (rows along the slowest axis are
 * contiguous in memory: one message per neighbour and component); a
 * reduction result is combined over the ranks (sum, min, max) when the
 * program asks for it.  Supported: declarations, par_loops (stencil reach
 * along the split axis at most H), reductions, ops_dat_fetch_data /
 * ops_dat_get_extents of the local rows, the exit dump.  Calls that need
 * the whole dat on one rank (halo transfers between blocks, raw pointers,
 * slab access, tridiagonal solves along the split axis, edge dats of extent
 * 1 along it) raise OPS_NOT_IMPLEMENTED.
 *
 * Transport: the caller registers a communicator before ops_init.  With
 * device == 0 the buffers are host memory (the runtime stages the rows
 * through pinned host buffers; any host transport works, e.g. a gloo
 * process group); with device == 1 they are device memory ordered on the
 * runtime's work stream (the NCCL transport the runtime builds itself when
 * OPS_B200_DIST=nccl: ncclSend / ncclRecv of the rows straight between the
 * GPUs and ncclAllReduce of the reduction results).
 */
#ifndef OPS_B200_DIST_H
#define OPS_B200_DIST_H

#include <stddef.h>

#include "ops_lib_core.h"

typedef struct ob2_dist_comm {
  int rank, size;
  int device; /* 1: buffers are device memory (stream-ordered), 0: host memory */
  void *ctx;
  /* sends sbytes from sbuf to rank speer and receives rbytes into rbuf from
   * rank rpeer (a peer of -1 skips that side); returns 0 on success */
  int (*sendrecv)(void *ctx, const void *sbuf, size_t sbytes, int speer, void *rbuf,
                  size_t rbytes, int rpeer);
  /* combines count values of kind type (0 double, 1 float, 2 int, 3 long
   * long) over all ranks in place with op OPS_INC (sum), OPS_MIN or OPS_MAX */
  int (*allreduce)(void *ctx, void *buf, int count, int type, int op);
} ob2_dist_comm;

/* Registers the communicator; call before ops_init (size 1: no split).
 * Returns 0, or OPS_INVALID_ARGUMENT for an inconsistent communicator. */
OPS_API int ob2_dist_init(const ob2_dist_comm *comm);
/* rank and size of the registered communicator (0 / 1 without one) */
OPS_API int ob2_dist_rank(void);
OPS_API int ob2_dist_size(void);

#ifdef __cplusplus
/* The decomposition arithmetic, shared by the runtime and its CPU check. */
namespace ob2dist {

/* owned rows [lo, hi) of rank r among R ranks over extent G */
inline void slab(int G, int R, int r, int *lo, int *hi) {
  *lo = (int)((long long)G * r / R);
  *hi = (int)((long long)G * (r + 1) / R);
}

/* rows a rank holds for a dat: [alo, ahi) in block coordinates along the
 * split axis, given the owned rows and the dat's interior extent n and halo
 * depths dm (<= 0) and dp (>= 0) along that axis */
inline void held_rows(int lo, int hi, int first, int last, int n, int dm, int dp, int H,
                      int *alo, int *ahi) {
  *alo = first ? dm : lo - H;
  *ahi = last ? n + dp : hi + H;
}

/* clips [a, b) along the split axis to the rows this rank computes */
inline void clip(int lo, int hi, int first, int last, int *a, int *b) {
  const int ca = first ? *a : (*a > lo ? *a : lo);
  const int cb = last ? *b : (*b < hi ? *b : hi);
  *a = ca;
  *b = cb > ca ? cb : ca;
}

}  // namespace ob2dist
#endif

#endif /* OPS_B200_DIST_H */
