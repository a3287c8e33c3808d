/*
 * Multi-block Poisson / Jacobi driver on the OPS API.
 *
 *   -lap(u) = f on the unit square, u = sin(pi x) sin(pi y) on the boundary,
 *   f ~ U(-1,1) (seeded), NB x NB blocks of N x N cells joined by 1-cell
 *   halos exchanged with ops_halo_transfer, Jacobi sweeps ping-ponging
 *   between u and u2, max-abs residual (OPS_MAX reduction) every CHECK sweeps.
 *
 * Defaults are the configuration 2 x 2 blocks of 256 x 256, 1000 sweeps,
 * residual every 100.  Options: -nb= -n= -sweeps= -check= -seed=
 * Prints the residual history, a checksum of u and the sweep rate.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OPS_2D
#include "ops_seq_v2.h"
#include "user_types.h"

double h_grid;
int rng_seed;

#include "poisson_mb_kernels.h"

static int opt(int argc, char **argv, const char *key, int def) {
  size_t n = strlen(key);
  for (int i = 1; i < argc; i++)
    if (!strncmp(argv[i], key, n)) return atoi(argv[i] + n);
  return def;
}

int main(int argc, char **argv) {
  ops_init(argc, argv, 1);
  const int NB = opt(argc, argv, "-nb=", 2);
  const int N = opt(argc, argv, "-n=", 256);
  const int SWEEPS = opt(argc, argv, "-sweeps=", 1000);
  const int CHECK = opt(argc, argv, "-check=", 100);
  rng_seed = opt(argc, argv, "-seed=", 1);
  const int G = NB * N; /* global interior points per direction */
  h_grid = 1.0 / (double)(G + 1);
  ops_decl_const("h_grid", 1, "double", &h_grid);
  ops_decl_const("rng_seed", 1, "int", &rng_seed);

  const int nblk = NB * NB;
  ops_block *blk = (ops_block *)malloc(sizeof(ops_block) * nblk);
  ops_dat *u = (ops_dat *)malloc(sizeof(ops_dat) * nblk);
  ops_dat *u2 = (ops_dat *)malloc(sizeof(ops_dat) * nblk);
  ops_dat *f = (ops_dat *)malloc(sizeof(ops_dat) * nblk);
  int *disp = (int *)malloc(sizeof(int) * 2 * nblk);
  int size[2] = {N, N}, base[2] = {0, 0}, d_m[2] = {-1, -1}, d_p[2] = {1, 1};
  char nm[64];
  for (int j = 0; j < NB; j++)
    for (int i = 0; i < NB; i++) {
      int b = i + NB * j;
      snprintf(nm, sizeof nm, "block %d,%d", i, j);
      blk[b] = ops_decl_block(2, nm);
      double *none = NULL;
      snprintf(nm, sizeof nm, "u %d,%d", i, j);
      u[b] = ops_decl_dat(blk[b], 1, size, base, d_m, d_p, none, "double", nm);
      snprintf(nm, sizeof nm, "u2 %d,%d", i, j);
      u2[b] = ops_decl_dat(blk[b], 1, size, base, d_m, d_p, none, "double", nm);
      snprintf(nm, sizeof nm, "f %d,%d", i, j);
      f[b] = ops_decl_dat(blk[b], 1, size, base, d_m, d_p, none, "double", nm);
      disp[2 * b] = i * N;
      disp[2 * b + 1] = j * N;
    }

  int s00[] = {0, 0};
  ops_stencil S00 = ops_decl_stencil(2, 1, s00, "00");
  int s5[] = {0, 0, 1, 0, -1, 0, 0, 1, 0, -1};
  ops_stencil S5 = ops_decl_stencil(2, 5, s5, "5pt");

  /* inner halos: both directions across every block face */
  const int nh = 2 * 2 * NB * (NB - 1);
  ops_halo *hu = (ops_halo *)malloc(sizeof(ops_halo) * (nh > 0 ? nh : 1));
  ops_halo *hu2 = (ops_halo *)malloc(sizeof(ops_halo) * (nh > 0 ? nh : 1));
  int k = 0;
  int dir[] = {1, 2};
  for (int j = 0; j < NB; j++)
    for (int i = 0; i < NB; i++) {
      int b = i + NB * j;
      if (i > 0) {
        int a = b - 1, it[] = {1, N};
        int fb1[] = {N - 1, 0}, tb1[] = {-1, 0}; /* left neighbour's last column -> my left halo */
        int fb2[] = {0, 0}, tb2[] = {N, 0};      /* my first column -> its right halo */
        hu[k] = ops_decl_halo(u[a], u[b], it, fb1, tb1, dir, dir);
        hu2[k++] = ops_decl_halo(u2[a], u2[b], it, fb1, tb1, dir, dir);
        hu[k] = ops_decl_halo(u[b], u[a], it, fb2, tb2, dir, dir);
        hu2[k++] = ops_decl_halo(u2[b], u2[a], it, fb2, tb2, dir, dir);
      }
      if (j > 0) {
        int a = b - NB, it[] = {N, 1};
        int fb1[] = {0, N - 1}, tb1[] = {0, -1};
        int fb2[] = {0, 0}, tb2[] = {0, N};
        hu[k] = ops_decl_halo(u[a], u[b], it, fb1, tb1, dir, dir);
        hu2[k++] = ops_decl_halo(u2[a], u2[b], it, fb1, tb1, dir, dir);
        hu[k] = ops_decl_halo(u[b], u[a], it, fb2, tb2, dir, dir);
        hu2[k++] = ops_decl_halo(u2[b], u2[a], it, fb2, tb2, dir, dir);
      }
    }
  ops_halo_group gu = ops_decl_halo_group(k, hu);
  ops_halo_group gu2 = ops_decl_halo_group(k, hu2);
  ops_reduction red = ops_decl_reduction_handle(sizeof(double), "double", "residual");
  ops_reduction rsum = ops_decl_reduction_handle(sizeof(double), "double", "checksum");
  ops_partition("");

  int gsize[2] = {G, G};
  for (int b = 0; b < nblk; b++) {
    int r[] = {-1, N + 1, -1, N + 1};
    ops_par_loop(pmb_init_kernel, "pmb_init_kernel", blk[b], 2, r,
                 ops_arg_gbl(&disp[2 * b], 2, "int", OPS_READ),
                 ops_arg_gbl(gsize, 2, "int", OPS_READ), ops_arg_idx(),
                 ops_arg_dat(u[b], 1, S00, "double", OPS_WRITE),
                 ops_arg_dat(u2[b], 1, S00, "double", OPS_WRITE),
                 ops_arg_dat(f[b], 1, S00, "double", OPS_WRITE));
  }

  double ct0, et0, ct1, et1;
  ops_timers(&ct0, &et0);
  ops_dat *cur = u, *nxt = u2;
  ops_halo_group gcur = gu, gnxt = gu2;
  int r_in[] = {0, N, 0, N};
  for (int s = 1; s <= SWEEPS; s++) {
    if (NB > 1) ops_halo_transfer(gcur);
    for (int b = 0; b < nblk; b++)
      ops_par_loop(pmb_jacobi_kernel, "pmb_jacobi_kernel", blk[b], 2, r_in,
                   ops_arg_dat(cur[b], 1, S5, "double", OPS_READ),
                   ops_arg_dat(f[b], 1, S00, "double", OPS_READ),
                   ops_arg_dat(nxt[b], 1, S00, "double", OPS_WRITE));
    ops_dat *t = cur; cur = nxt; nxt = t;
    ops_halo_group tg = gcur; gcur = gnxt; gnxt = tg;
    if (CHECK > 0 && s % CHECK == 0) {
      if (NB > 1) ops_halo_transfer(gcur);
      for (int b = 0; b < nblk; b++)
        ops_par_loop(pmb_residual_kernel, "pmb_residual_kernel", blk[b], 2, r_in,
                     ops_arg_dat(cur[b], 1, S5, "double", OPS_READ),
                     ops_arg_dat(f[b], 1, S00, "double", OPS_READ),
                     ops_arg_reduce(red, 1, "double", OPS_MAX));
      double res = 0.0;
      ops_reduction_result(red, &res);
      ops_printf("sweep %6d  max|residual| %.15e\n", s, res);
    }
  }
  ops_timers(&ct1, &et1);
  for (int b = 0; b < nblk; b++)
    ops_par_loop(pmb_sum_kernel, "pmb_sum_kernel", blk[b], 2, r_in,
                 ops_arg_dat(cur[b], 1, S00, "double", OPS_READ),
                 ops_arg_reduce(rsum, 1, "double", OPS_INC));
  double sum = 0.0;
  ops_reduction_result(rsum, &sum);
  double glups = (double)G * G * SWEEPS / (et1 - et0) / 1e9;
  ops_printf("checksum %.15e\n", sum);
  ops_printf("sweeps %d  time %.6f s  %.3f GLUPS\n", SWEEPS, et1 - et0, glups);
  ops_timing_output(std::cout);
  ops_exit();
  free(blk); free(u); free(u2); free(f); free(disp); free(hu); free(hu2);
  return 0;
}
