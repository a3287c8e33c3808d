/*
 * opsunit: one OPS program that exercises the par_loop features the parity
 * tests compare between this backend and the oracle -- ops_arg_idx, global
 * arrays, multi-component AoS dats with (d,x,y) access, int and float dats,
 * 9-point stencils into 2-deep halos, strided stencils over row / column
 * dats, INC (2-vector) / MIN / MAX / integer reductions accumulated over two
 * loops, optional arguments (enabled and disabled), RW access with a global
 * constant, an empty range, and low-dim accumulation with combine_inc.
 *
 * Options: -nx= -ny= (default 37 x 23), -soa=1 (SoA storage of multi-component
 * dats)
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OPS_2D
#include "ops_seq_v2.h"
#include "user_types.h"

double ou_scale;

#include "opsunit_kernels.h"

static int opt(int argc, char **argv, const char *key, int def) {
  size_t n = strlen(key);
  for (int i = 1; i < argc; i++)
    if (!strncmp(argv[i], key, n)) return atoi(argv[i] + n);
  return def;
}

int main(int argc, char **argv) {
  ops_init(argc, argv, 1);
  // -soa=1: multi-component dats stored component-major (ops_set_soa)
  if (opt(argc, argv, "-soa=", 0)) ops_set_soa(1);
  const int nx = opt(argc, argv, "-nx=", 37), ny = opt(argc, argv, "-ny=", 23);
  ou_scale = 0.75;
  ops_decl_const("ou_scale", 1, "double", &ou_scale);
  ops_block g = ops_decl_block(2, "grid");

  int size[] = {nx, ny}, base[] = {0, 0}, m2[] = {-2, -2}, p2[] = {2, 2}, z0[] = {0, 0};
  double *dn = NULL;
  int *in = NULL;
  float *fn = NULL;
  ops_dat a = ops_decl_dat(g, 1, size, base, m2, p2, dn, "double", "a");
  ops_dat ia = ops_decl_dat(g, 1, size, base, m2, p2, in, "int", "ia");
  ops_dat v = ops_decl_dat(g, 3, size, base, z0, z0, dn, "double", "v");
  ops_dat f = ops_decl_dat(g, 1, size, base, z0, z0, fn, "float", "f");
  ops_dat b = ops_decl_dat(g, 1, size, base, z0, z0, dn, "double", "b");
  ops_dat c = ops_decl_dat(g, 1, size, base, z0, z0, dn, "double", "c");
  ops_dat o = ops_decl_dat(g, 1, size, base, z0, z0, dn, "double", "o");
  int rsz[] = {nx, 1}, rm[] = {-1, 0}, rp[] = {1, 0};
  ops_dat rowx = ops_decl_dat(g, 1, rsz, base, rm, rp, dn, "double", "rowx");
  int csz[] = {1, ny}, cm[] = {0, -1}, cp[] = {0, 1};
  ops_dat coly = ops_decl_dat(g, 1, csz, base, cm, cp, dn, "double", "coly");
  ops_dat rowsum = ops_decl_dat(g, 1, rsz, base, z0, z0, dn, "double", "rowsum");

  int s00[] = {0, 0};
  ops_stencil S00 = ops_decl_stencil(2, 1, s00, "00");
  int s9[] = {-1, -1, 0, -1, 1, -1, -1, 0, 0, 0, 1, 0, -1, 1, 0, 1, 1, 1};
  ops_stencil S9 = ops_decl_stencil(2, 9, s9, "9pt");
  int strx[] = {1, 0}, stry[] = {0, 1};
  int sx2[] = {0, 0, 1, 0};
  ops_stencil SX = ops_decl_strided_stencil(2, 2, sx2, strx, "rowx");
  ops_stencil SX1 = ops_decl_strided_stencil(2, 1, s00, strx, "rowx1");
  int sy2[] = {0, 0, 0, -1};
  ops_stencil SY = ops_decl_strided_stencil(2, 2, sy2, stry, "coly");
  ops_stencil SY1 = ops_decl_strided_stencil(2, 1, s00, stry, "coly1");

  ops_reduction r_sum = ops_decl_reduction_handle(2 * sizeof(double), "double", "sums");
  ops_reduction r_min = ops_decl_reduction_handle(sizeof(double), "double", "min");
  ops_reduction r_max = ops_decl_reduction_handle(sizeof(double), "double", "max");
  ops_reduction r_cnt = ops_decl_reduction_handle(sizeof(int), "int", "count");
  ops_partition("");

  double w[3] = {0.5, -1.25, 3.0};
  int whole[] = {-2, nx + 2, -2, ny + 2};
  ops_par_loop(ou_fill, "ou_fill", g, 2, whole, ops_arg_idx(), ops_arg_gbl(w, 3, "double", OPS_READ),
               ops_arg_dat(a, 1, S00, "double", OPS_WRITE), ops_arg_dat(ia, 1, S00, "int", OPS_WRITE));
  int in_r[] = {0, nx, 0, ny};
  ops_par_loop(ou_vec, "ou_vec", g, 2, in_r, ops_arg_dat(a, 1, S00, "double", OPS_READ),
               ops_arg_dat(v, 3, S00, "double", OPS_WRITE), ops_arg_dat(f, 1, S00, "float", OPS_WRITE));
  ops_par_loop(ou_stencil, "ou_stencil", g, 2, in_r, ops_arg_dat(a, 1, S9, "double", OPS_READ),
               ops_arg_dat(b, 1, S00, "double", OPS_WRITE));
  int rowr[] = {-1, nx + 1, 0, 1};
  ops_par_loop(ou_rowfill, "ou_rowfill", g, 2, rowr, ops_arg_idx(),
               ops_arg_dat(rowx, 1, SX1, "double", OPS_WRITE));
  int colr[] = {0, 1, -1, ny + 1};
  ops_par_loop(ou_colfill, "ou_colfill", g, 2, colr, ops_arg_idx(),
               ops_arg_dat(coly, 1, SY1, "double", OPS_WRITE));
  ops_par_loop(ou_strided, "ou_strided", g, 2, in_r, ops_arg_dat(rowx, 1, SX, "double", OPS_READ),
               ops_arg_dat(coly, 1, SY, "double", OPS_READ), ops_arg_dat(c, 1, S00, "double", OPS_WRITE));
  /* reductions accumulated over two loops covering the two halves */
  int lo_r[] = {0, nx, 0, ny / 2}, hi_r[] = {0, nx, ny / 2, ny};
  int *halves[2] = {lo_r, hi_r};
  for (int h = 0; h < 2; h++)
    ops_par_loop(ou_reduce, "ou_reduce", g, 2, halves[h], ops_arg_dat(a, 1, S00, "double", OPS_READ),
                 ops_arg_dat(v, 3, S00, "double", OPS_READ), ops_arg_reduce(r_sum, 2, "double", OPS_INC),
                 ops_arg_reduce(r_min, 1, "double", OPS_MIN), ops_arg_reduce(r_max, 1, "double", OPS_MAX),
                 ops_arg_reduce(r_cnt, 1, "int", OPS_INC));
  int on = 1, off = 0;
  ops_par_loop(ou_opt, "ou_opt", g, 2, in_r, ops_arg_gbl(&on, 1, "int", OPS_READ),
               ops_arg_dat(a, 1, S00, "double", OPS_READ),
               ops_arg_dat_opt(o, 1, S00, "double", OPS_WRITE, 1));
  int half_r[] = {0, nx / 2, 0, ny};
  ops_par_loop(ou_opt, "ou_opt", g, 2, half_r, ops_arg_gbl(&off, 1, "int", OPS_READ),
               ops_arg_dat(b, 1, S00, "double", OPS_READ),
               ops_arg_dat_opt(o, 1, S00, "double", OPS_WRITE, 0));
  ops_par_loop(ou_rw, "ou_rw", g, 2, in_r, ops_arg_dat(b, 1, S00, "double", OPS_RW));
  int empty[] = {5, 5, 0, ny};
  ops_par_loop(ou_rw, "ou_rw", g, 2, empty, ops_arg_dat(b, 1, S00, "double", OPS_RW));
  ops_par_loop(ou_colsum, "ou_colsum", g, 2, in_r, ops_arg_dat(a, 1, S00, "double", OPS_READ),
               ops_arg_dat(rowsum, 1, SX1, "double", OPS_INC));

  double sums[2], mn, mx;
  int cnt;
  ops_reduction_result(r_sum, sums);
  ops_reduction_result(r_min, &mn);
  ops_reduction_result(r_max, &mx);
  ops_reduction_result(r_cnt, &cnt);
  printf("sums %.17g %.17g\nmin %.17g\nmax %.17g\ncount %d\n", sums[0], sums[1], mn, mx, cnt);
  /* fetch through the external-access API */
  double *buf = (double *)malloc(sizeof(double) * nx * ny);
  ops_dat_fetch_data(b, 0, (char *)buf);
  double s = 0.0;
  for (int i = 0; i < nx * ny; i++) s += buf[i] * (1.0 + (i % 7));
  printf("fetch_b %.17g\n", s);
  free(buf);
  ops_exit();
  return 0;
}
