/*
 * Kernels of the multi-block Poisson/Jacobi driver (config: 2x2 blocks of
 * 256x256 cells, 1-cell halos joined by ops_halo_transfer, 5-point Jacobi,
 * max-abs residual reduction).  Written against the unchanged OPS API.
 */
#ifndef POISSON_MB_KERNELS_H
#define POISSON_MB_KERNELS_H

/* initial state: u = 0 inside, Dirichlet sin(pi x) sin(pi y) in the outer
 * halo, f ~ U(-1,1) from a counter-based hash of (seed, global index) */
void pmb_init_kernel(const int *disp, const int *gsize, const int *idx, ACC<double> &u,
                     ACC<double> &u2, ACC<double> &f) {
  const int gi = idx[0] + disp[0] + 1;  /* global node index, boundary at 0 and n+1 */
  const int gj = idx[1] + disp[1] + 1;
  const double x = gi * h_grid, y = gj * h_grid;
  const bool boundary = gi == 0 || gj == 0 || gi == gsize[0] + 1 || gj == gsize[1] + 1;
  const double bc = boundary ? sin(M_PI * x) * sin(M_PI * y) : 0.0;
  u(0, 0) = bc;
  u2(0, 0) = bc;
  f(0, 0) = pmb_uniform(rng_seed, gi, gj) * 2.0 - 1.0;
}

/* one Jacobi sweep of -lap(u) = f on a uniform grid of spacing h */
void pmb_jacobi_kernel(const ACC<double> &u, const ACC<double> &f, ACC<double> &un) {
  un(0, 0) = 0.25 * (u(-1, 0) + u(1, 0) + u(0, -1) + u(0, 1) + h_grid * h_grid * f(0, 0));
}

/* max-abs residual of -lap(u) = f */
void pmb_residual_kernel(const ACC<double> &u, const ACC<double> &f, double *res) {
  const double r = f(0, 0) - (4.0 * u(0, 0) - u(-1, 0) - u(1, 0) - u(0, -1) - u(0, 1)) /
                                 (h_grid * h_grid);
  *res = MAX(*res, fabs(r));
}

/* sum of u over the block interior (checksum) */
void pmb_sum_kernel(const ACC<double> &u, double *s) { *s = *s + u(0, 0); }

#endif
