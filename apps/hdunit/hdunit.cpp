/*
 * hdunit: the 5D par_loop, reduction and halo paths that the parity tests
 * compare between this backend and the oracle -- a 5D block with halo depth
 * 1, a fill from ops_arg_idx, a stencil reaching one point along every axis,
 * OPS_INC and OPS_MAX reductions over the 5D range, and a halo group whose
 * boxes are flipped along the 4th and 5th axes.
 *
 * Options: -n= (extent along the first three axes, default 6)
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OPS_5D
#include "ops_seq_v2.h"

#include "hdunit_kernels.h"

static int opt(int argc, char **argv, const char *key, int def) {
  size_t n = strlen(key);
  for (int i = 1; i < argc; i++)
    if (!strncmp(argv[i], key, n)) return atoi(argv[i] + n);
  return def;
}

int main(int argc, char **argv) {
  ops_init(argc, argv, 1);
  const int n = opt(argc, argv, "-n=", 6);
  ops_block g = ops_decl_block(5, "g5");
  int size[5] = {n, n - 1, n - 2, 4, 3}, base[5] = {0, 0, 0, 0, 0};
  int d_m[5] = {-1, -1, -1, -1, -1}, d_p[5] = {1, 1, 1, 1, 1};
  double *none = NULL;
  ops_dat a = ops_decl_dat(g, 1, size, base, d_m, d_p, none, "double", "a");
  ops_dat b = ops_decl_dat(g, 1, size, base, d_m, d_p, none, "double", "b");
  ops_dat c = ops_decl_dat(g, 1, size, base, d_m, d_p, none, "double", "c");
  int s0[5] = {0, 0, 0, 0, 0};
  int s11[55] = {0, 0, 0, 0, 0,  1, 0, 0, 0, 0,  -1, 0, 0, 0, 0,  0, 1, 0, 0, 0,  0, -1, 0, 0, 0,
                 0, 0, 1, 0, 0,  0, 0, -1, 0, 0,  0, 0, 0, 1, 0,  0, 0, 0, -1, 0,
                 0, 0, 0, 0, 1,  0, 0, 0, 0, -1};
  ops_stencil S0 = ops_decl_stencil(5, 1, s0, "0");
  ops_stencil S11 = ops_decl_stencil(5, 11, s11, "star11");
  ops_reduction rs = ops_decl_reduction_handle(sizeof(double), "double", "sum");
  ops_reduction rm = ops_decl_reduction_handle(sizeof(double), "double", "max");

  // every point including the halo ring
  int all[10] = {-1, size[0] + 1, -1, size[1] + 1, -1, size[2] + 1, -1, size[3] + 1, -1, size[4] + 1};
  int in[10] = {0, size[0], 0, size[1], 0, size[2], 0, size[3], 0, size[4]};
  ops_par_loop(hd_fill, "hd_fill", g, 5, all, ops_arg_dat(a, 1, S0, "double", OPS_WRITE),
               ops_arg_idx());
  ops_par_loop(hd_stencil, "hd_stencil", g, 5, in, ops_arg_dat(a, 1, S11, "double", OPS_READ),
               ops_arg_dat(b, 1, S0, "double", OPS_WRITE));
  ops_par_loop(hd_reduce, "hd_reduce", g, 5, in, ops_arg_dat(b, 1, S0, "double", OPS_READ),
               ops_arg_reduce(rs, 1, "double", OPS_INC), ops_arg_reduce(rm, 1, "double", OPS_MAX));
  double sum = 0.0, mx = 0.0;
  ops_reduction_result(rs, &sum);
  ops_reduction_result(rm, &mx);
  ops_printf("hdunit sums %.17g max %.17g\n", sum, mx);

  // halo: the interior of b into c shifted by one along x, flipped along
  // the 4th and 5th axes (a box of the full extent along those)
  int iter[5] = {size[0] - 1, size[1], size[2], size[3], size[4]};
  int from_base[5] = {0, 0, 0, 0, 0}, to_base[5] = {1, 0, 0, 0, 0};
  int from_dir[5] = {1, 2, 3, 4, 5}, to_dir[5] = {1, 2, 3, -4, -5};
  ops_halo h = ops_decl_halo(b, c, iter, from_base, to_base, from_dir, to_dir);
  ops_halo_group grp = ops_decl_halo_group(1, &h);
  ops_halo_transfer(grp);
  ops_par_loop(hd_reduce, "hd_reduce", g, 5, in, ops_arg_dat(c, 1, S0, "double", OPS_READ),
               ops_arg_reduce(rs, 1, "double", OPS_INC), ops_arg_reduce(rm, 1, "double", OPS_MAX));
  ops_reduction_result(rs, &sum);
  ops_reduction_result(rm, &mx);
  ops_printf("hdunit halo sums %.17g max %.17g\n", sum, mx);
  ops_exit();
  return 0;
}
