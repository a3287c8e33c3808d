/*
 * Kernels of the 4D / 5D unit program: a fill from the point index, a
 * stencil reaching one point along each of the five axes, a copy into a
 * 4D dat, and sum / max reductions over the 5D range.
 */
#ifndef HDUNIT_KERNELS_H
#define HDUNIT_KERNELS_H

void hd_fill(ACC<double> &a, const int *idx) {
  a(0, 0, 0, 0, 0) = 1.0 + idx[0] + 3.0 * idx[1] + 0.5 * idx[2] - 2.0 * idx[3] + 7.0 * idx[4] +
                     0.125 * idx[0] * idx[4];
}

void hd_stencil(const ACC<double> &a, ACC<double> &b) {
  b(0, 0, 0, 0, 0) = 2.0 * a(0, 0, 0, 0, 0) - 0.25 * (a(1, 0, 0, 0, 0) + a(-1, 0, 0, 0, 0)) +
                     0.125 * (a(0, 1, 0, 0, 0) - a(0, -1, 0, 0, 0)) +
                     0.0625 * (a(0, 0, 1, 0, 0) + a(0, 0, -1, 0, 0)) +
                     0.5 * (a(0, 0, 0, 1, 0) - a(0, 0, 0, -1, 0)) +
                     0.75 * (a(0, 0, 0, 0, 1) + a(0, 0, 0, 0, -1));
}

void hd_reduce(const ACC<double> &b, double *sum, double *mx) {
  *sum += b(0, 0, 0, 0, 0);
  *mx = MAX(*mx, b(0, 0, 0, 0, 0));
}

#endif
