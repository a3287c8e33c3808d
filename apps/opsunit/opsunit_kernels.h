/* Kernels of the opsunit application: one kernel per OPS feature. */
#ifndef OPSUNIT_KERNELS_H
#define OPSUNIT_KERNELS_H

/* ops_arg_idx + ops_arg_gbl array: a(x,y) = w0*x + w1*y + w2 */
void ou_fill(const int *idx, const double *w, ACC<double> &a, ACC<int> &ia) {
  a(0, 0) = w[0] * idx[0] + w[1] * idx[1] + w[2] + ou_hash(idx[0], idx[1]);
  ia(0, 0) = idx[0] * 1000 + idx[1];
}

/* multi-component (AoS) dat with (d,x,y) access, float dat */
void ou_vec(const ACC<double> &a, ACC<double> &v, ACC<float> &f) {
  v(0, 0, 0) = a(0, 0) * 2.0;
  v(1, 0, 0) = a(0, 0) - 1.0;
  v(2, 0, 0) = a(0, 0) * a(0, 0);
  f(0, 0) = (float)(a(0, 0) / 3.0);
}

/* 9-point stencil reading halos written by ou_fill */
void ou_stencil(const ACC<double> &a, ACC<double> &b) {
  b(0, 0) = a(-1, -1) + 2.0 * a(0, -1) + a(1, -1) + 2.0 * a(-1, 0) - 12.0 * a(0, 0) +
            2.0 * a(1, 0) + a(-1, 1) + 2.0 * a(0, 1) + a(1, 1);
}

/* strided stencils: row / column dats (sizes {nx,1} and {1,ny}) in a 2D loop */
void ou_strided(const ACC<double> &rowx, const ACC<double> &coly, ACC<double> &c) {
  c(0, 0) = rowx(0, 0) * 10.0 + coly(0, 0) + rowx(1, 0) - coly(0, -1);
}
void ou_rowfill(const int *idx, ACC<double> &rowx) { rowx(0, 0) = 0.5 * idx[0] + 1.0; }
void ou_colfill(const int *idx, ACC<double> &coly) { coly(0, 0) = -0.25 * idx[1] + 2.0; }

/* reductions: INC of a 2-vector, MIN, MAX, integer INC */
void ou_reduce(const ACC<double> &a, const ACC<double> &v, double *sums, double *mn, double *mx,
               int *cnt) {
  sums[0] = sums[0] + a(0, 0);
  sums[1] = sums[1] + v(2, 0, 0);
  *mn = MIN(*mn, a(0, 0));
  *mx = MAX(*mx, v(1, 0, 0));
  *cnt = *cnt + 1;
}

/* optional argument: written only when enabled */
void ou_opt(const int *flag, const ACC<double> &a, ACC<double> &o) {
  if (*flag) o(0, 0) = a(0, 0) + 100.0;
}

/* RW access and a global read scalar from the constant table */
void ou_rw(ACC<double> &b) { b(0, 0) = b(0, 0) * ou_scale + 1.0; }

/* low-dim accumulation: column sums of a into a row dat through
 * combine_inc (the row dat is written by every y) */
void ou_colsum(const ACC<double> &a, ACC<double> &rowsum) { rowsum.combine_inc(0, 0, a(0, 0)); }

#endif
