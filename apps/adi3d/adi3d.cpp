/*
 * 3D ADI heat driver on the OPS API (ops_par_loop + ops_tridMultiDimBatch).
 *
 * Per step: the preprocessing par_loop builds the right-hand side
 * du = lambda * lap7(u) and the three sets of tridiagonal coefficients, then
 * three batched solves run along x and y (solution in du) and along z with
 * the solution added to u (ops_tridMultiDimBatch_Inc).
 *
 * Defaults are the configuration 256^3, u0 ~ U(0,1) (seed 3), lambda = 1,
 * 50 steps.  -prec=64 (FP64 storage), -prec=32 (FP32 storage, FP64
 * arithmetic and elimination) or -prec=both (both, and the FP32 error
 * against FP64 is printed).  Options: -n= (cube) or -nx= -ny= -nz=, -steps=,
 * -seed=, -lambda=
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OPS_3D
#include "ops_seq_v2.h"
#include "ops_tridiag.h"
#include "user_types.h"

int adi_n[3];
double adi_lambda;
int adi_seed;

#include "adi3d_kernels.h"

static int iopt(int argc, char **argv, const char *key, int def) {
  size_t n = strlen(key);
  for (int i = 1; i < argc; i++)
    if (!strncmp(argv[i], key, n)) return atoi(argv[i] + n);
  return def;
}
static const char *sopt(int argc, char **argv, const char *key, const char *def) {
  size_t n = strlen(key);
  for (int i = 1; i < argc; i++)
    if (!strncmp(argv[i], key, n)) return argv[i] + n;
  return def;
}

struct Set {
  ops_dat u, du, ax, bx, cx, ay, by, cy, az, bz, cz;
};

template <typename T>
static Set decl_set(ops_block blk, const char *tag, const char *type) {
  int size[3] = {adi_n[0], adi_n[1], adi_n[2]};
  int base[3] = {0, 0, 0}, d_m[3] = {-1, -1, -1}, d_p[3] = {1, 1, 1};
  T *none = NULL;
  char nm[64];
  Set s;
  ops_dat *slots[11] = {&s.u, &s.du, &s.ax, &s.bx, &s.cx, &s.ay, &s.by, &s.cy, &s.az, &s.bz, &s.cz};
  const char *names[11] = {"u", "du", "ax", "bx", "cx", "ay", "by", "cy", "az", "bz", "cz"};
  for (int i = 0; i < 11; i++) {
    snprintf(nm, sizeof nm, "%s_%s", names[i], tag);
    *slots[i] = ops_decl_dat(blk, 1, size, base, d_m, d_p, none, type, nm);
  }
  return s;
}

int main(int argc, char **argv) {
  ops_init(argc, argv, 1);
  int n = iopt(argc, argv, "-n=", 256);
  adi_n[0] = iopt(argc, argv, "-nx=", n);
  adi_n[1] = iopt(argc, argv, "-ny=", n);
  adi_n[2] = iopt(argc, argv, "-nz=", n);
  const int STEPS = iopt(argc, argv, "-steps=", 50);
  adi_seed = iopt(argc, argv, "-seed=", 3);
  adi_lambda = atof(sopt(argc, argv, "-lambda=", "1.0"));
  const char *prec = sopt(argc, argv, "-prec=", "64");
  const bool do64 = strcmp(prec, "32") != 0;
  const bool do32 = strcmp(prec, "64") != 0;
  ops_decl_const("adi_n", 3, "int", adi_n);
  ops_decl_const("adi_lambda", 1, "double", &adi_lambda);
  ops_decl_const("adi_seed", 1, "int", &adi_seed);

  ops_block blk = ops_decl_block(3, "heat3D");
  int s000[] = {0, 0, 0};
  ops_stencil S000 = ops_decl_stencil(3, 1, s000, "000");
  int s7[] = {0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1};
  ops_stencil S7 = ops_decl_stencil(3, 7, s7, "7pt");
  Set d64, d32;
  if (do64) d64 = decl_set<double>(blk, "f64", "double");
  if (do32) d32 = decl_set<float>(blk, "f32", "float");
  ops_reduction r_s = ops_decl_reduction_handle(sizeof(double), "double", "sum");
  ops_reduction r_s2 = ops_decl_reduction_handle(sizeof(double), "double", "sum2");
  ops_reduction r_e2 = ops_decl_reduction_handle(sizeof(double), "double", "err2");
  ops_reduction r_em = ops_decl_reduction_handle(sizeof(double), "double", "errmax");
  ops_partition("");
  ops_tridsolver_params *ctx_x = new ops_tridsolver_params(blk);
  ops_tridsolver_params *ctx_y = new ops_tridsolver_params(blk);
  ops_tridsolver_params *ctx_z = new ops_tridsolver_params(blk);

  int all[] = {0, adi_n[0], 0, adi_n[1], 0, adi_n[2]};
  if (do64)
    ops_par_loop(adi_init_f64, "adi_init_f64", blk, 3, all, ops_arg_idx(),
                 ops_arg_dat(d64.u, 1, S000, "double", OPS_WRITE));
  if (do32)
    ops_par_loop(adi_init_f32, "adi_init_f32", blk, 3, all, ops_arg_idx(),
                 ops_arg_dat(d32.u, 1, S000, "float", OPS_WRITE));

  double ct0, et0, ct1, et1, t64 = 0.0, t32 = 0.0;
  if (do64) {
    ops_timers(&ct0, &et0);
    for (int it = 0; it < STEPS; it++) {
      Set &s = d64;
      ops_par_loop(adi_preproc_f64, "adi_preproc_f64", blk, 3, all,
                   ops_arg_dat(s.u, 1, S7, "double", OPS_READ),
                   ops_arg_dat(s.du, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.ax, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.bx, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.cx, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.ay, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.by, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.cy, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.az, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.bz, 1, S000, "double", OPS_WRITE),
                   ops_arg_dat(s.cz, 1, S000, "double", OPS_WRITE), ops_arg_idx());
      ops_tridMultiDimBatch(3, 0, all, s.ax, s.bx, s.cx, s.du, ctx_x);
      ops_tridMultiDimBatch(3, 1, all, s.ay, s.by, s.cy, s.du, ctx_y);
      ops_tridMultiDimBatch_Inc(3, 2, all, s.az, s.bz, s.cz, s.du, s.u, ctx_z);
    }
    ops_timers(&ct1, &et1);
    t64 = et1 - et0;
    double sum = 0.0, sum2 = 0.0;
    ops_par_loop(adi_sum_f64, "adi_sum_f64", blk, 3, all,
                 ops_arg_dat(d64.u, 1, S000, "double", OPS_READ),
                 ops_arg_reduce(r_s, 1, "double", OPS_INC),
                 ops_arg_reduce(r_s2, 1, "double", OPS_INC));
    ops_reduction_result(r_s, &sum);
    ops_reduction_result(r_s2, &sum2);
    ops_printf("fp64 checksum sum %.15e sum2 %.15e\n", sum, sum2);
    ops_printf("fp64 %d steps %.6f s  %.3f ms/step\n", STEPS, t64, 1e3 * t64 / STEPS);
  }
  if (do32) {
    ops_timers(&ct0, &et0);
    for (int it = 0; it < STEPS; it++) {
      Set &s = d32;
      ops_par_loop(adi_preproc_f32, "adi_preproc_f32", blk, 3, all,
                   ops_arg_dat(s.u, 1, S7, "float", OPS_READ),
                   ops_arg_dat(s.du, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.ax, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.bx, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.cx, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.ay, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.by, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.cy, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.az, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.bz, 1, S000, "float", OPS_WRITE),
                   ops_arg_dat(s.cz, 1, S000, "float", OPS_WRITE), ops_arg_idx());
      ops_tridMultiDimBatch(3, 0, all, s.ax, s.bx, s.cx, s.du, ctx_x);
      ops_tridMultiDimBatch(3, 1, all, s.ay, s.by, s.cy, s.du, ctx_y);
      ops_tridMultiDimBatch_Inc(3, 2, all, s.az, s.bz, s.cz, s.du, s.u, ctx_z);
    }
    ops_timers(&ct1, &et1);
    t32 = et1 - et0;
    double sum = 0.0, sum2 = 0.0;
    ops_par_loop(adi_sum_f32, "adi_sum_f32", blk, 3, all,
                 ops_arg_dat(d32.u, 1, S000, "float", OPS_READ),
                 ops_arg_reduce(r_s, 1, "double", OPS_INC),
                 ops_arg_reduce(r_s2, 1, "double", OPS_INC));
    ops_reduction_result(r_s, &sum);
    ops_reduction_result(r_s2, &sum2);
    ops_printf("fp32 checksum sum %.15e sum2 %.15e\n", sum, sum2);
    ops_printf("fp32 %d steps %.6f s  %.3f ms/step\n", STEPS, t32, 1e3 * t32 / STEPS);
  }
  if (do64 && do32) {
    double e2 = 0.0, em = 0.0, s2 = 0.0, s = 0.0;
    ops_par_loop(adi_diff, "adi_diff", blk, 3, all, ops_arg_dat(d64.u, 1, S000, "double", OPS_READ),
                 ops_arg_dat(d32.u, 1, S000, "float", OPS_READ),
                 ops_arg_reduce(r_e2, 1, "double", OPS_INC),
                 ops_arg_reduce(r_em, 1, "double", OPS_MAX));
    ops_reduction_result(r_e2, &e2);
    ops_reduction_result(r_em, &em);
    ops_par_loop(adi_sum_f64, "adi_sum_f64", blk, 3, all,
                 ops_arg_dat(d64.u, 1, S000, "double", OPS_READ),
                 ops_arg_reduce(r_s, 1, "double", OPS_INC),
                 ops_arg_reduce(r_s2, 1, "double", OPS_INC));
    ops_reduction_result(r_s, &s);
    ops_reduction_result(r_s2, &s2);
    ops_printf("fp32 vs fp64: relative L2 error %.6e  max abs error %.6e\n", sqrt(e2 / s2), em);
  }
  delete ctx_x;
  delete ctx_y;
  delete ctx_z;
  ops_timing_output(std::cout);
  ops_exit();
  return 0;
}
