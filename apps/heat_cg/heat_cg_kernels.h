/*
 * Kernels of the CG heat-conduction driver, written against the unchanged
 * OPS API.  The operator and the CG steps follow TeaLeaf's unpreconditioned
 * CG (apps/c/TeaLeaf/tea_leaf_common_kernels.h:11-32 for the coefficients and
 * the operator, tea_leaf_cg_kernels.h:8-20 and tea_leaf_cg.cpp for the
 * iteration): A u = (1 + rx (Kx(1,0)+Kx) + ry (Ky(0,1)+Ky)) u
 *                   - rx (Kx(1,0) u(1,0) + Kx u(-1,0)) - ry (Ky(0,1) u(0,1) + Ky u(0,-1)),
 * Kx = (w(-1,0)+w) / (2 w(-1,0) w) with w the density (conductivity), and
 * Kx, Ky zero on the domain faces (no flux through the boundary).
 *
 * The *32 kernels are the mixed-precision form: FP32 storage and arithmetic
 * for the CG vectors, dot products accumulated in FP64, the iterate and the
 * replacement residual in FP64.
 */
#ifndef HEAT_CG_KERNELS_H
#define HEAT_CG_KERNELS_H

/* density (100 inside the circle, 0.1 outside) and the initial temperature
 * u0 ~ U(0,1), which is also the right-hand side and the first iterate */
void hc_init_kernel(const int *idx, ACC<double> &den, ACC<double> &u0, ACC<double> &u) {
  const double x = (idx[0] + 0.5) * hc_cell, y = (idx[1] + 0.5) * hc_cell;
  const double dx = x - hc_cx, dy = y - hc_cy;
  den(0, 0) = (dx * dx + dy * dy <= hc_r2) ? 100.0 : 0.1;
  const double t = hc_uniform(hc_seed, idx[0] + 1, idx[1] + 1);
  u0(0, 0) = t;
  u(0, 0) = t;
}

/* face coefficients from the density (harmonic-mean form) */
void hc_coef_kernel(ACC<double> &Kx, ACC<double> &Ky, const ACC<double> &w) {
  Kx(0, 0) = (w(-1, 0) + w(0, 0)) / (2.0 * w(-1, 0) * w(0, 0));
  Ky(0, 0) = (w(0, -1) + w(0, 0)) / (2.0 * w(0, -1) * w(0, 0));
}

void hc_zero_kernel(ACC<double> &K) { K(0, 0) = 0.0; }

/* ---- FP64 CG ---- */

/* r = b - A u, p = r, rr += r.r */
void hc_res_kernel(ACC<double> &r, ACC<double> &p, const ACC<double> &Kx, const ACC<double> &Ky,
                   const ACC<double> &u, const ACC<double> &b, double *rr) {
  const double au = (1.0 + hc_ry * (Ky(0, 1) + Ky(0, 0)) + hc_rx * (Kx(1, 0) + Kx(0, 0))) * u(0, 0) -
                    hc_ry * (Ky(0, 1) * u(0, 1) + Ky(0, 0) * u(0, -1)) -
                    hc_rx * (Kx(1, 0) * u(1, 0) + Kx(0, 0) * u(-1, 0));
  const double rv = b(0, 0) - au;
  r(0, 0) = rv;
  p(0, 0) = rv;
  *rr = *rr + rv * rv;
}

/* true residual norm only: rr += (b - A u)^2 */
void hc_true_res_kernel(const ACC<double> &Kx, const ACC<double> &Ky, const ACC<double> &u,
                        const ACC<double> &b, double *rr) {
  const double au = (1.0 + hc_ry * (Ky(0, 1) + Ky(0, 0)) + hc_rx * (Kx(1, 0) + Kx(0, 0))) * u(0, 0) -
                    hc_ry * (Ky(0, 1) * u(0, 1) + Ky(0, 0) * u(0, -1)) -
                    hc_rx * (Kx(1, 0) * u(1, 0) + Kx(0, 0) * u(-1, 0));
  const double rv = b(0, 0) - au;
  *rr = *rr + rv * rv;
}

/* w = A p, pw += p.w */
void hc_w_kernel(ACC<double> &w, const ACC<double> &Kx, const ACC<double> &Ky,
                 const ACC<double> &p, double *pw) {
  const double ap = (1.0 + hc_ry * (Ky(0, 1) + Ky(0, 0)) + hc_rx * (Kx(1, 0) + Kx(0, 0))) * p(0, 0) -
                    hc_ry * (Ky(0, 1) * p(0, 1) + Ky(0, 0) * p(0, -1)) -
                    hc_rx * (Kx(1, 0) * p(1, 0) + Kx(0, 0) * p(-1, 0));
  w(0, 0) = ap;
  *pw = *pw + ap * p(0, 0);
}

/* u += alpha p, r -= alpha w, rnn += r.r */
void hc_ur_kernel(ACC<double> &u, ACC<double> &r, const ACC<double> &p, const ACC<double> &w,
                  const double *alpha, double *rnn) {
  u(0, 0) = u(0, 0) + (*alpha) * p(0, 0);
  const double rv = r(0, 0) - (*alpha) * w(0, 0);
  r(0, 0) = rv;
  *rnn = *rnn + rv * rv;
}

/* p = r + beta p */
void hc_p_kernel(ACC<double> &p, const ACC<double> &r, const double *beta) {
  p(0, 0) = r(0, 0) + (*beta) * p(0, 0);
}

void hc_sum_kernel(const ACC<double> &u, double *s) { *s = *s + u(0, 0); }

/* ---- mixed precision: FP32 inner CG inside FP64 refinement ---- */

void hc_coef32_kernel(ACC<float> &Kx32, ACC<float> &Ky32, const ACC<double> &Kx,
                      const ACC<double> &Ky) {
  Kx32(0, 0) = (float)Kx(0, 0);
  Ky32(0, 0) = (float)Ky(0, 0);
}

/* FP64 residual of the FP64 iterate, stored in FP32: r32 = b - A x,
 * rr += r.r (FP64) */
void hc_res32_kernel(ACC<float> &r32, const ACC<double> &Kx, const ACC<double> &Ky,
                     const ACC<double> &x, const ACC<double> &b, double *rr) {
  const double ax = (1.0 + hc_ry * (Ky(0, 1) + Ky(0, 0)) + hc_rx * (Kx(1, 0) + Kx(0, 0))) * x(0, 0) -
                    hc_ry * (Ky(0, 1) * x(0, 1) + Ky(0, 0) * x(0, -1)) -
                    hc_rx * (Kx(1, 0) * x(1, 0) + Kx(0, 0) * x(-1, 0));
  const double rv = b(0, 0) - ax;
  r32(0, 0) = (float)rv;
  *rr = *rr + rv * rv;
}

void hc_copy32_kernel(ACC<float> &p, const ACC<float> &r) { p(0, 0) = r(0, 0); }

/* w = A p in FP32, pw += p.w accumulated in FP64 */
void hc_w32_kernel(ACC<float> &w, const ACC<float> &Kx, const ACC<float> &Ky,
                   const ACC<float> &p, double *pw) {
  const float ap = (1.0f + hc_ry32 * (Ky(0, 1) + Ky(0, 0)) + hc_rx32 * (Kx(1, 0) + Kx(0, 0))) * p(0, 0) -
                   hc_ry32 * (Ky(0, 1) * p(0, 1) + Ky(0, 0) * p(0, -1)) -
                   hc_rx32 * (Kx(1, 0) * p(1, 0) + Kx(0, 0) * p(-1, 0));
  w(0, 0) = ap;
  *pw = *pw + (double)ap * (double)p(0, 0);
}

/* x += alpha p in FP64, r -= alpha w in FP32, rnn += r.r (FP64) */
void hc_xr32_kernel(ACC<double> &x, ACC<float> &r, const ACC<float> &p, const ACC<float> &w,
                    const double *alpha, double *rnn) {
  x(0, 0) = x(0, 0) + (*alpha) * (double)p(0, 0);
  const float rv = r(0, 0) - (float)(*alpha) * w(0, 0);
  r(0, 0) = rv;
  *rnn = *rnn + (double)rv * (double)rv;
}

void hc_p32_kernel(ACC<float> &p, const ACC<float> &r, const float *beta) {
  p(0, 0) = r(0, 0) + (*beta) * p(0, 0);
}

#endif
