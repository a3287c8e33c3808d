/*
 * Kernels of the 3D ADI heat driver: one implicit step of the heat equation
 * split into x, y and z tridiagonal solves (a = c = -lambda/2, b = 1 + lambda
 * inside, identity rows on the boundary), with the right-hand side
 * lambda * (7-point Laplacian of u).  The same kernels exist for FP64 storage
 * and for FP32 storage with FP64 arithmetic.
 */
#ifndef ADI3D_KERNELS_H
#define ADI3D_KERNELS_H

void adi_init_f64(const int *idx, ACC<double> &u) { u(0, 0, 0) = adi_uniform(adi_seed, idx); }
void adi_init_f32(const int *idx, ACC<float> &u) { u(0, 0, 0) = (float)adi_uniform(adi_seed, idx); }

void adi_preproc_f64(const ACC<double> &u, ACC<double> &du, ACC<double> &ax, ACC<double> &bx,
                     ACC<double> &cx, ACC<double> &ay, ACC<double> &by, ACC<double> &cy,
                     ACC<double> &az, ACC<double> &bz, ACC<double> &cz, const int *idx) {
  double a, b, c, d;
  if (idx[0] == 0 || idx[0] == adi_n[0] - 1 || idx[1] == 0 || idx[1] == adi_n[1] - 1 ||
      idx[2] == 0 || idx[2] == adi_n[2] - 1) {
    a = 0.0; b = 1.0; c = 0.0; d = 0.0;
  } else {
    d = adi_lambda * (u(-1, 0, 0) + u(1, 0, 0) + u(0, -1, 0) + u(0, 1, 0) + u(0, 0, -1) +
                      u(0, 0, 1) - 6.0 * u(0, 0, 0));
    a = -0.5 * adi_lambda;
    b = 1.0 + adi_lambda;
    c = -0.5 * adi_lambda;
  }
  du(0, 0, 0) = d;
  ax(0, 0, 0) = a; bx(0, 0, 0) = b; cx(0, 0, 0) = c;
  ay(0, 0, 0) = a; by(0, 0, 0) = b; cy(0, 0, 0) = c;
  az(0, 0, 0) = a; bz(0, 0, 0) = b; cz(0, 0, 0) = c;
}

void adi_preproc_f32(const ACC<float> &u, ACC<float> &du, ACC<float> &ax, ACC<float> &bx,
                     ACC<float> &cx, ACC<float> &ay, ACC<float> &by, ACC<float> &cy,
                     ACC<float> &az, ACC<float> &bz, ACC<float> &cz, const int *idx) {
  double a, b, c, d;
  if (idx[0] == 0 || idx[0] == adi_n[0] - 1 || idx[1] == 0 || idx[1] == adi_n[1] - 1 ||
      idx[2] == 0 || idx[2] == adi_n[2] - 1) {
    a = 0.0; b = 1.0; c = 0.0; d = 0.0;
  } else {
    d = adi_lambda * ((double)u(-1, 0, 0) + (double)u(1, 0, 0) + (double)u(0, -1, 0) +
                      (double)u(0, 1, 0) + (double)u(0, 0, -1) + (double)u(0, 0, 1) -
                      6.0 * (double)u(0, 0, 0));
    a = -0.5 * adi_lambda;
    b = 1.0 + adi_lambda;
    c = -0.5 * adi_lambda;
  }
  du(0, 0, 0) = (float)d;
  ax(0, 0, 0) = (float)a; bx(0, 0, 0) = (float)b; cx(0, 0, 0) = (float)c;
  ay(0, 0, 0) = (float)a; by(0, 0, 0) = (float)b; cy(0, 0, 0) = (float)c;
  az(0, 0, 0) = (float)a; bz(0, 0, 0) = (float)b; cz(0, 0, 0) = (float)c;
}

/* sums for checksums and the FP32-vs-FP64 error */
void adi_sum_f64(const ACC<double> &u, double *s, double *s2) {
  *s = *s + u(0, 0, 0);
  *s2 = *s2 + u(0, 0, 0) * u(0, 0, 0);
}
void adi_diff(const ACC<double> &u, const ACC<float> &v, double *e2, double *emax) {
  const double e = (double)v(0, 0, 0) - u(0, 0, 0);
  *e2 = *e2 + e * e;
  *emax = MAX(*emax, fabs(e));
}
void adi_sum_f32(const ACC<float> &u, double *s, double *s2) {
  *s = *s + (double)u(0, 0, 0);
  *s2 = *s2 + (double)u(0, 0, 0) * (double)u(0, 0, 0);
}

#endif
