/*
 * Implicit heat conduction by conjugate gradients on the OPS API.
 *
 *   (I + dt K) u = u0 on the unit square, K the 5-point variable-coefficient
 *   operator of TeaLeaf (conductivity = density: 100 inside a seeded circle
 *   of radius 0.2, 0.1 outside), no flux through the boundary, u0 ~ U(0,1).
 *
 * Two solvers on the same system:
 *   fp64   plain FP64 CG (TeaLeaf's unpreconditioned CG, tea_leaf_cg.cpp) to a
 *          relative residual tol;
 *   mixed  CG with r, w, p stored and computed in FP32 (dot products
 *          accumulated in FP64) and the iterate x in FP64; the residual is
 *          replaced by b - A x computed in FP64 whenever it has dropped by
 *          the factor -inner= since the last such evaluation (iterative
 *          refinement that keeps the search direction), and convergence is
 *          tested on that FP64 residual.
 *
 * Options: -n= (cells per side, default 4096) -prec=64|32|both (default both)
 *          -tol= (default 1e-10) -inner= (residual drop between FP64
 *          residual replacements, default 1e-2)
 *          -maxit= (iteration cap per CG, default 20000) -dt= (default 4e-6)
 *          -dump=FILE (every dat's interior at the end, apps/dumpdats.h)
 *          -seed= (circle centre, default 4) -useed= (u0, default 5)
 * Prints per solver: iterations, recursive and true relative residuals and a
 * checksum ("fp64 ...", "mixed ..."), for both the relative difference of the
 * two solutions ("compare ..."), and on "timing ..." lines the solve times,
 * the bytes-model bandwidth and the time ratio.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OPS_2D
#include "ops_seq_v2.h"
#include "user_types.h"

double hc_rx, hc_ry, hc_cell, hc_cx, hc_cy, hc_r2;
float hc_rx32, hc_ry32;
int hc_seed;

#include "heat_cg_kernels.h"
#include "dumpdats.h"

static const char *sopt(int argc, char **argv, const char *key) {
  size_t n = strlen(key);
  for (int i = 1; i < argc; i++)
    if (!strncmp(argv[i], key, n)) return argv[i] + n;
  return nullptr;
}
static int iopt(int argc, char **argv, const char *key, int def) {
  const char *v = sopt(argc, argv, key);
  return v ? atoi(v) : def;
}
static double dopt(int argc, char **argv, const char *key, double def) {
  const char *v = sopt(argc, argv, key);
  return v ? atof(v) : def;
}

/* circle centre drawn from the seed, inside [0.2, 0.8]^2 so the circle lies
 * in the domain */
static void circle_centre(int seed, double *cx, double *cy) {
  *cx = 0.2 + 0.6 * hc_uniform(seed, 7, 11);
  *cy = 0.2 + 0.6 * hc_uniform(seed, 13, 17);
}

struct Grid {
  ops_block blk;
  int N;
  ops_stencil S00, S5, SK, SKX, SKY;
  ops_reduction red;
  int in[4];
};

static double reduce_result(Grid &g) {
  double v = 0.0;
  ops_reduction_result(g.red, &v);
  return v;
}

static double true_residual(Grid &g, ops_dat Kx, ops_dat Ky, ops_dat u, ops_dat b) {
  ops_par_loop(hc_true_res_kernel, "hc_true_res_kernel", g.blk, 2, g.in,
               ops_arg_dat(Kx, 1, g.SKX, "double", OPS_READ),
               ops_arg_dat(Ky, 1, g.SKY, "double", OPS_READ),
               ops_arg_dat(u, 1, g.S5, "double", OPS_READ),
               ops_arg_dat(b, 1, g.S00, "double", OPS_READ),
               ops_arg_reduce(g.red, 1, "double", OPS_INC));
  return sqrt(reduce_result(g));
}

static double checksum(Grid &g, ops_dat u) {
  ops_par_loop(hc_sum_kernel, "hc_sum_kernel", g.blk, 2, g.in,
               ops_arg_dat(u, 1, g.S00, "double", OPS_READ),
               ops_arg_reduce(g.red, 1, "double", OPS_INC));
  return reduce_result(g);
}

/* plain FP64 CG from u = b; returns iterations */
static int cg64(Grid &g, ops_dat u, ops_dat b, ops_dat r, ops_dat p, ops_dat w, ops_dat Kx,
                ops_dat Ky, double tol, int maxit, double *rel) {
  ops_par_loop(hc_res_kernel, "hc_res_kernel", g.blk, 2, g.in,
               ops_arg_dat(r, 1, g.S00, "double", OPS_WRITE),
               ops_arg_dat(p, 1, g.S00, "double", OPS_WRITE),
               ops_arg_dat(Kx, 1, g.SKX, "double", OPS_READ),
               ops_arg_dat(Ky, 1, g.SKY, "double", OPS_READ),
               ops_arg_dat(u, 1, g.S5, "double", OPS_READ),
               ops_arg_dat(b, 1, g.S00, "double", OPS_READ),
               ops_arg_reduce(g.red, 1, "double", OPS_INC));
  double rro = reduce_result(g);
  const double rr0 = rro;
  int it = 0;
  *rel = 1.0;
  while (it < maxit && rro > 0.0 && sqrt(rro / rr0) > tol) {
    ops_par_loop(hc_w_kernel, "hc_w_kernel", g.blk, 2, g.in,
                 ops_arg_dat(w, 1, g.S00, "double", OPS_WRITE),
                 ops_arg_dat(Kx, 1, g.SKX, "double", OPS_READ),
                 ops_arg_dat(Ky, 1, g.SKY, "double", OPS_READ),
                 ops_arg_dat(p, 1, g.S5, "double", OPS_READ),
                 ops_arg_reduce(g.red, 1, "double", OPS_INC));
    const double pw = reduce_result(g);
    const double alpha = rro / pw;
    ops_par_loop(hc_ur_kernel, "hc_ur_kernel", g.blk, 2, g.in,
                 ops_arg_dat(u, 1, g.S00, "double", OPS_RW),
                 ops_arg_dat(r, 1, g.S00, "double", OPS_RW),
                 ops_arg_dat(p, 1, g.S00, "double", OPS_READ),
                 ops_arg_dat(w, 1, g.S00, "double", OPS_READ),
                 ops_arg_gbl(&alpha, 1, "double", OPS_READ),
                 ops_arg_reduce(g.red, 1, "double", OPS_INC));
    const double rnn = reduce_result(g);
    const double beta = rnn / rro;
    ops_par_loop(hc_p_kernel, "hc_p_kernel", g.blk, 2, g.in,
                 ops_arg_dat(p, 1, g.S00, "double", OPS_RW),
                 ops_arg_dat(r, 1, g.S00, "double", OPS_READ),
                 ops_arg_gbl(&beta, 1, "double", OPS_READ));
    rro = rnn;
    it++;
  }
  *rel = rr0 > 0.0 ? sqrt(rro / rr0) : 0.0;
  return it;
}

/* Mixed precision CG: r, w, p in FP32 (FP32 arithmetic, dot products
 * accumulated in FP64), the iterate x in FP64 and updated in FP64 every
 * iteration.  When the recursive residual has dropped by `drop` since the
 * last true residual, or meets tol, the residual is replaced by b - A x
 * computed in FP64 (reliable updates: the search direction p is kept, so CG
 * keeps its FP64 convergence) and convergence is tested on that residual.
 * Returns the CG iterations; *repl counts the FP64 residual evaluations,
 * *rel the final true relative residual. */
static int cg_mixed(Grid &g, ops_dat x, ops_dat b, ops_dat r, ops_dat p, ops_dat w,
                    ops_dat Kx, ops_dat Ky, ops_dat Kx32, ops_dat Ky32, double tol, double drop,
                    int maxit, int *repl, double *rel) {
  auto true_res = [&]() {  // r = b - A x in FP64, stored in FP32
    ops_par_loop(hc_res32_kernel, "hc_res32_kernel", g.blk, 2, g.in,
                 ops_arg_dat(r, 1, g.S00, "float", OPS_WRITE),
                 ops_arg_dat(Kx, 1, g.SKX, "double", OPS_READ),
                 ops_arg_dat(Ky, 1, g.SKY, "double", OPS_READ),
                 ops_arg_dat(x, 1, g.S5, "double", OPS_READ),
                 ops_arg_dat(b, 1, g.S00, "double", OPS_READ),
                 ops_arg_reduce(g.red, 1, "double", OPS_INC));
    return reduce_result(g);
  };
  double rro = true_res();
  const double rr0 = rro;
  double rr_true = rro;
  *repl = 1;
  *rel = rr0 > 0.0 ? 1.0 : 0.0;
  ops_par_loop(hc_copy32_kernel, "hc_copy32_kernel", g.blk, 2, g.in,
               ops_arg_dat(p, 1, g.S00, "float", OPS_WRITE),
               ops_arg_dat(r, 1, g.S00, "float", OPS_READ));
  int it = 0;
  while (it < maxit && rro > 0.0 && *rel > tol) {
    ops_par_loop(hc_w32_kernel, "hc_w32_kernel", g.blk, 2, g.in,
                 ops_arg_dat(w, 1, g.S00, "float", OPS_WRITE),
                 ops_arg_dat(Kx32, 1, g.SKX, "float", OPS_READ),
                 ops_arg_dat(Ky32, 1, g.SKY, "float", OPS_READ),
                 ops_arg_dat(p, 1, g.S5, "float", OPS_READ),
                 ops_arg_reduce(g.red, 1, "double", OPS_INC));
    const double pw = reduce_result(g);
    const double alpha = rro / pw;
    ops_par_loop(hc_xr32_kernel, "hc_xr32_kernel", g.blk, 2, g.in,
                 ops_arg_dat(x, 1, g.S00, "double", OPS_RW),
                 ops_arg_dat(r, 1, g.S00, "float", OPS_RW),
                 ops_arg_dat(p, 1, g.S00, "float", OPS_READ),
                 ops_arg_dat(w, 1, g.S00, "float", OPS_READ),
                 ops_arg_gbl(&alpha, 1, "double", OPS_READ),
                 ops_arg_reduce(g.red, 1, "double", OPS_INC));
    double rnn = reduce_result(g);
    it++;
    if (sqrt(rnn / rr_true) <= drop || sqrt(rnn / rr0) <= tol) {
      rnn = true_res();
      rr_true = rnn;
      (*repl)++;
      *rel = sqrt(rnn / rr0);
      if (*rel <= tol) break;
    }
    const float beta = (float)(rnn / rro);
    ops_par_loop(hc_p32_kernel, "hc_p32_kernel", g.blk, 2, g.in,
                 ops_arg_dat(p, 1, g.S00, "float", OPS_RW),
                 ops_arg_dat(r, 1, g.S00, "float", OPS_READ),
                 ops_arg_gbl(&beta, 1, "float", OPS_READ));
    rro = rnn;
  }
  if (it >= maxit) *rel = sqrt(true_res() / rr0);
  return it;
}

int main(int argc, char **argv) {
  ops_init(argc, argv, 1);
  const int N = iopt(argc, argv, "-n=", 4096);
  const double tol = dopt(argc, argv, "-tol=", 1e-10);
  const double inner = dopt(argc, argv, "-inner=", 1e-2);
  const int maxit = iopt(argc, argv, "-maxit=", 20000);
  const double dt = dopt(argc, argv, "-dt=", 4e-6);
  const char *prec = sopt(argc, argv, "-prec=");
  const bool do64 = !prec || !strcmp(prec, "64") || !strcmp(prec, "both");
  const bool do32 = !prec || !strcmp(prec, "32") || !strcmp(prec, "both");
  hc_seed = iopt(argc, argv, "-useed=", 5);
  circle_centre(iopt(argc, argv, "-seed=", 4), &hc_cx, &hc_cy);
  hc_r2 = 0.2 * 0.2;
  hc_cell = 1.0 / N;
  hc_rx = dt / (hc_cell * hc_cell);
  hc_ry = hc_rx;
  hc_rx32 = (float)hc_rx;
  hc_ry32 = (float)hc_ry;
  ops_decl_const("hc_rx", 1, "double", &hc_rx);
  ops_decl_const("hc_ry", 1, "double", &hc_ry);
  ops_decl_const("hc_rx32", 1, "float", &hc_rx32);
  ops_decl_const("hc_ry32", 1, "float", &hc_ry32);
  ops_decl_const("hc_cell", 1, "double", &hc_cell);
  ops_decl_const("hc_cx", 1, "double", &hc_cx);
  ops_decl_const("hc_cy", 1, "double", &hc_cy);
  ops_decl_const("hc_r2", 1, "double", &hc_r2);
  ops_decl_const("hc_seed", 1, "int", &hc_seed);

  Grid g;
  g.N = N;
  g.blk = ops_decl_block(2, "heat");
  int size[2] = {N, N}, base[2] = {0, 0}, d_m[2] = {-1, -1}, d_p[2] = {1, 1};
  double *nulld = nullptr;
  float *nullf = nullptr;
  ops_dat den = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "density");
  ops_dat b = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "u0");
  ops_dat Kx = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "Kx");
  ops_dat Ky = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "Ky");
  int s00[] = {0, 0};
  int s5[] = {0, 0, -1, 0, 1, 0, 0, -1, 0, 1};
  int skx[] = {0, 0, 1, 0};
  int sky[] = {0, 0, 0, 1};
  int sk[] = {0, 0, -1, 0, 0, -1};
  g.S00 = ops_decl_stencil(2, 1, s00, "00");
  g.S5 = ops_decl_stencil(2, 5, s5, "5pt");
  g.SKX = ops_decl_stencil(2, 2, skx, "00_P10");
  g.SKY = ops_decl_stencil(2, 2, sky, "00_0P1");
  g.SK = ops_decl_stencil(2, 3, sk, "00_M10_0M1");
  g.red = ops_decl_reduction_handle(sizeof(double), "double", "dot");
  g.in[0] = 0; g.in[1] = N; g.in[2] = 0; g.in[3] = N;

  ops_dat u64 = nullptr, x64 = nullptr;
  ops_dat r = nullptr, p = nullptr, w = nullptr;
  if (do64) {
    u64 = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "u");
    r = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "r");
    p = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "p");
    w = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "w");
  }
  if (do32) x64 = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nulld, "double", "x");

  int full[] = {-1, N + 1, -1, N + 1};
  ops_par_loop(hc_init_kernel, "hc_init_kernel", g.blk, 2, full, ops_arg_idx(),
               ops_arg_dat(den, 1, g.S00, "double", OPS_WRITE),
               ops_arg_dat(b, 1, g.S00, "double", OPS_WRITE),
               ops_arg_dat(do64 ? u64 : x64, 1, g.S00, "double", OPS_WRITE));
  int faces[] = {0, N + 1, 0, N + 1};
  ops_par_loop(hc_coef_kernel, "hc_coef_kernel", g.blk, 2, faces,
               ops_arg_dat(Kx, 1, g.S00, "double", OPS_WRITE),
               ops_arg_dat(Ky, 1, g.S00, "double", OPS_WRITE),
               ops_arg_dat(den, 1, g.SK, "double", OPS_READ));
  int fx0[] = {0, 1, 0, N}, fx1[] = {N, N + 1, 0, N}, fy0[] = {0, N, 0, 1}, fy1[] = {0, N, N, N + 1};
  ops_par_loop(hc_zero_kernel, "hc_zero_kernel", g.blk, 2, fx0,
               ops_arg_dat(Kx, 1, g.S00, "double", OPS_WRITE));
  ops_par_loop(hc_zero_kernel, "hc_zero_kernel", g.blk, 2, fx1,
               ops_arg_dat(Kx, 1, g.S00, "double", OPS_WRITE));
  ops_par_loop(hc_zero_kernel, "hc_zero_kernel", g.blk, 2, fy0,
               ops_arg_dat(Ky, 1, g.S00, "double", OPS_WRITE));
  ops_par_loop(hc_zero_kernel, "hc_zero_kernel", g.blk, 2, fy1,
               ops_arg_dat(Ky, 1, g.S00, "double", OPS_WRITE));
  if (do64 && do32) ops_dat_deep_copy(x64, u64);
  ops_dat Kx32 = nullptr, Ky32 = nullptr, r32 = nullptr, p32 = nullptr, w32 = nullptr;
  const double cells = (double)N * N;
  double t64 = 0.0, t32 = 0.0;

  if (do64) {
    double c0, e0, c1, e1, rel = 0.0;
    const double res0 = true_residual(g, Kx, Ky, u64, b);  // u starts at b
    ops_timers(&c0, &e0);
    int it = cg64(g, u64, b, r, p, w, Kx, Ky, tol, maxit, &rel);
    ops_timers(&c1, &e1);
    t64 = e1 - e0;
    const double tres = true_residual(g, Kx, Ky, u64, b) / res0;
    const double bytes = cells * (104.0 * it + 48.0);
    ops_printf("fp64 iterations %d  resid %.15e  true_resid %.15e\n", it, rel, tres);
    ops_printf("timing fp64 %.6f s  %.1f GB/s\n", t64, bytes / t64 / 1e9);
    ops_printf("fp64 checksum %.15e\n", checksum(g, u64));
  }

  if (do32) {
    Kx32 = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nullf, "float", "Kx32");
    Ky32 = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nullf, "float", "Ky32");
    r32 = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nullf, "float", "r32");
    p32 = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nullf, "float", "p32");
    w32 = ops_decl_dat(g.blk, 1, size, base, d_m, d_p, nullf, "float", "w32");
    int all[] = {0, N + 1, 0, N + 1};
    ops_par_loop(hc_coef32_kernel, "hc_coef32_kernel", g.blk, 2, all,
                 ops_arg_dat(Kx32, 1, g.S00, "float", OPS_WRITE),
                 ops_arg_dat(Ky32, 1, g.S00, "float", OPS_WRITE),
                 ops_arg_dat(Kx, 1, g.S00, "double", OPS_READ),
                 ops_arg_dat(Ky, 1, g.S00, "double", OPS_READ));
    double c0, e0, c1, e1, rel = 1.0;
    int repl = 0;
    ops_timers(&c0, &e0);
    const int it = cg_mixed(g, x64, b, r32, p32, w32, Kx, Ky, Kx32, Ky32, tol, inner, maxit,
                            &repl, &rel);
    ops_timers(&c1, &e1);
    t32 = e1 - e0;
    // bytes model per iteration: w = A p reads Kx, Ky, p (FP32) and writes w
    // (16 B); x += alpha p, r -= alpha w read p, w and update x (FP64) and r
    // (32 B); p = r + beta p (12 B); each FP64 residual reads Kx, Ky, x, b
    // and writes r (36 B)
    const double bytes = cells * (60.0 * it + 36.0 * repl);
    ops_printf("mixed iterations %d  replacements %d  true_resid %.15e\n", it, repl, rel);
    ops_printf("timing mixed %.6f s  %.1f GB/s\n", t32, bytes / t32 / 1e9);
    ops_printf("mixed checksum %.15e\n", checksum(g, x64));
  }
  if (do64 && do32) {
    // max |x - u| / max |u| over the interior, through host copies
    ops_get_data(u64);
    ops_get_data(x64);
    int disp[2], sz[2];
    ops_dat_get_extents(u64, 0, disp, sz);
    size_t n = (size_t)sz[0] * sz[1];
    double *hu = (double *)malloc(n * sizeof(double)), *hx = (double *)malloc(n * sizeof(double));
    int rng[] = {0, N, 0, N};
    ops_dat_fetch_data_slab_memspace(u64, 0, (char *)hu, rng, OPS_HOST);
    ops_dat_fetch_data_slab_memspace(x64, 0, (char *)hx, rng, OPS_HOST);
    double dmax = 0.0, umax = 0.0;
    for (size_t i = 0; i < (size_t)N * N; i++) {
      dmax = fmax(dmax, fabs(hx[i] - hu[i]));
      umax = fmax(umax, fabs(hu[i]));
    }
    free(hu);
    free(hx);
    ops_printf("compare max_rel_diff %.15e\n", dmax / umax);
    ops_printf("timing ratio_fp64_over_mixed %.3f\n", t64 / t32);
  }
  const char *dump = sopt(argc, argv, "-dump=");
  if (dump) {  // every dat through the public fetch call (apps/dumpdats.h)
    ops_dat all[] = {den, b, Kx, Ky, u64, r, p, w, x64, Kx32, Ky32, r32, p32, w32};
    if (dump_dats(dump, all, (int)(sizeof(all) / sizeof(all[0]))) != 0)
      ops_printf("dump to %s failed\n", dump);
  }
  ops_timing_output(std::cout);
  ops_exit();
  return 0;
}
