// ob2_serve.cu -- the solve-serving engine (include/ops_b200_serve.h).
//
// Device state: an array of request slots (struct Req, FP64 CG scalars
// included) and a work list (struct Work) naming the active requests with
// prefix sums of their work units.  Every batched kernel is persistent: a
// grid of a few CTAs per SM walks the global unit index over all active
// requests, finds the request by binary search in the prefix table, and works
// on that request's tile.  One engine iteration:
//   pois_pass     one pass of the single-reduction CG over every Poisson /
//                 heat request: the iteration (p, s, x, r and w = A r with
//                 per-tile (r, r), (w, r)), or the FP64 residual b - A x and
//                 w = A r of a residual replacement
//   adi_pre       right-hand side of the ADI step (adi/preproc_kernel.h)
//   adi_x/y/z     constant-coefficient Thomas solves (z adds into u)
//   scalars_b     per request: fixed-order sum of its tile partials, alpha,
//                 beta, residual replacement and convergence; heat time
//                 steps; ADI step count
// All kernels read the work list from device memory, so one captured graph
// of K iterations serves every batch composition.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "ops_b200_serve.h"

namespace {

constexpr int TX = 32;
constexpr int MAXA = OB2S_MAX_ACTIVE;
constexpr int ADI_MAX_N = 192;  // x-solve tile: 32 lines x n points in shared memory
constexpr int ADI_XL = 32;      // lines per x-solve unit
constexpr int ADI_YZ = 4;       // planes per y/z-solve unit (CTA 32 x 4 lines)
constexpr double kHeatRho = 1.0;  // heat requests: dt / h^2 of the implicit step

struct Req {
  int kind, n, pitch, tiles_x, tiles;
  int phase, done, outer, inner_it, iters;
  int max_inner, max_outer, steps, step;
  int par;  // p buffer parity
  int newstep;  // heat: the next pass starts a time step (b = x)
  double tol, inner_tol;
  double alpha, beta, gamma, gamma_in0, rr0, rel;
  double diag, off;  // operator: diag x - off (sum of the 4 neighbours)
  double *x, *b, *part;
  void *r[2], *w[2], *s[2], *p;
  void *y;  // mixed mode: FP32 correction accumulator (NULL in FP64 mode)
  double *u, *du, *cp, *mm;
  double a_coef, lambda;
};

struct Work {
  int npois, nadi;
  int pois_slot[MAXA];
  int adi_slot[MAXA];
  long long pois_pref[MAXA + 1];
  long long pre_pref[MAXA + 1];
  long long x_pref[MAXA + 1];
  long long yz_pref[MAXA + 1];
};

__device__ __forceinline__ int find_req(const long long *pref, int n, long long u) {
  int lo = 0, hi = n;  // pref[lo] <= u < pref[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pref[mid] <= u)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ double hash_uniform(int seed, int i, int j, int k) {
  unsigned long long z = ((unsigned long long)(unsigned)seed << 42) ^
                         ((unsigned long long)(unsigned)i << 21) ^ (unsigned long long)(unsigned)j ^
                         ((unsigned long long)(unsigned)k << 52);
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// ---------------------------------------------------------------- Poisson
// CTA 32 x 8 threads; each thread handles RY consecutive rows, so a tile is
// 32 x (8 RY) points.  Loads of out-of-range rows are clamped to the zero
// halo row below the grid (always valid memory) and only the stores are
// guarded, so the loads of all rows are issued before any store.
//
// Poisson and heat requests: A x = diag x - off (sum of the 4 neighbours)
// with a zero Dirichlet boundary (Poisson: diag 4, off 1; a backward-Euler
// heat step: diag 1 + 4 rho, off rho), solved by conjugate gradients in the
// single-reduction form of Chronopoulos and Gear ("s-step iterative methods
// for symmetric linear systems", J. Comput. Appl. Math. 25, 1989): with
// w = A r and s = A p carried along,
//   p_i = r_i + beta_i p_{i-1}      s_i = w_i + beta_i s_{i-1}
//   x_{i+1} = x_i + alpha_i p_i     r_{i+1} = r_i - alpha_i s_i
//   w_{i+1} = A r_{i+1}             gamma = (r, r), delta = (w, r) at i+1
//   beta_{i+1} = gamma_{i+1} / gamma_i
//   alpha_{i+1} = gamma_{i+1} / (delta_{i+1} - beta_{i+1} gamma_{i+1} / alpha_i)
// so that one pass over the vectors and one scalar kernel make an
// iteration (the two-reduction form needs two passes and two scalar
// kernels).  w_{i+1} needs r_{i+1} at the four neighbours: each thread forms
// r_{i+1} = r_i - alpha (w_i + beta s_{i-1}) of its rows and of the rows above
// and below itself, the warp's lanes exchange theirs by shuffles and the edge
// lanes form their outer neighbours from memory with the same arithmetic, so
// every value of r_{i+1} is computed identically wherever it is used.
// r, w and s are double-buffered (read [par], written [par ^ 1]); p and the
// iterate are updated in place (read only at their own point).
//
// Precision: the vectors r, w, s, p are stored in TI (FP32 in the mixed mode,
// FP64 otherwise); every value is formed in FP64 from its stored inputs and
// rounded once to TI; dot products accumulate in FP64.  The FP64 mode updates
// the FP64 iterate x every iteration.  The mixed mode accumulates alpha p into
// an FP32 correction y instead and folds y into the FP64 x at each residual
// replacement (reliable updates with a low-precision accumulator, as in
// mixed-precision Krylov solvers since Sleijpen and van der Vorst,
// Computing 56, 1996): between replacements y holds only the correction since
// the last fold, so its rounding shrinks with the error it corrects.  Per
// point per iteration the mixed mode moves 40 bytes (r, w, s, p, y read and
// written in FP32), the FP64 mode 80.
// The recursive residual is replaced by b - A x computed in FP64 whenever it
// has dropped by inner_tol since the last true residual or meets the
// tolerance; the search directions p, s are kept.
// Phases:
//   0  start (and restart after a breakdown; for heat requests also the start
//      of each time step, which first sets b = x): r = b - A (x + y) [pois_pass]
//   4  w = A r, fold x += y, y = 0, (r, r), (w, r)   [pois_pass]; alpha_0
//   2  CG iteration                                  [pois_pass]; alpha, beta
//   3  replacement: r = b - A (x + y) in FP64        [pois_pass]
//   5  as 4, then beta from the true (r, r), p and s kept
// The scalar kernel (scalars_b) moves every request to its next phase.

constexpr int CTA_Y = 8;
constexpr int NPART = 2;  // partial sums per tile: (r, r) and (w, r)

// resident CTAs per SM the Poisson kernels are compiled for (register cap)
#ifndef OB2S_MINB
#define OB2S_MINB 4
#endif
#define POIS_BOUNDS __launch_bounds__(256, OB2S_MINB)

// fixed-order CTA sum of NV values per thread; result in thread 0
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*sh)[32]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int c = 0; c < NV; c++) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  const int nw = (blockDim.x * blockDim.y + 31) >> 5;
  if ((t & 31) == 0)
#pragma unroll
    for (int c = 0; c < NV; c++) sh[c][t >> 5] = v[c];
  __syncthreads();
  if (t == 0)
#pragma unroll
    for (int c = 0; c < NV; c++) {
      double a = 0.0;
      for (int k = 0; k < nw; k++) a += sh[c][k];
      v[c] = a;
    }
  __syncthreads();
}

// r_{i+1} at one point from the stored r_i, w_i, s_{i-1}: the one expression
// every thread uses for it
template <typename TI>
__device__ __forceinline__ TI next_r(TI r, TI w, TI s, double alpha, double beta, TI &s_new) {
  s_new = (TI)((double)w + beta * (double)s);
  return (TI)((double)r - alpha * (double)s_new);
}

// one pass of a Poisson / heat request's current phase over the tile
template <typename TI, int RY>
__global__ void POIS_BOUNDS pois_pass(const Work *__restrict__ W, Req *R) {
  __shared__ double sh[NPART][32];
  const long long total = W->pois_pref[W->npois];
  const unsigned full = 0xffffffffu;
  for (long long un = blockIdx.x; un < total; un += gridDim.x) {
    const int k = find_req(W->pois_pref, W->npois, un);
    const Req &q = R[W->pois_slot[k]];
    const int ph = q.phase;
    if (q.done) continue;  // uniform over the CTA
    const int t = (int)(un - W->pois_pref[k]);
    const int n = q.n, P = q.pitch;
    const int lane = threadIdx.x;
    const int i = (t % q.tiles_x) * TX + lane;
    const int j0 = (t / q.tiles_x) * (CTA_Y * RY) + threadIdx.y * RY;
    const bool inx = i < n;
    const int ic = inx ? i : n - 1;  // lanes past the edge load valid memory
    const double diag = q.diag, off = q.off;
    const int cur = q.par, nxt = q.par ^ 1;
    const bool mixed = q.y != nullptr;
    double v[NPART] = {0.0, 0.0};
    if (j0 < n) {  // uniform over the warp (one threadIdx.y per warp)
      // storage offsets of rows j0-1 .. j0+RY of column i, clamped into the
      // array ((n + 2)^2 < 2^31 for n <= 32768)
      int o[RY + 2];
#pragma unroll
      for (int m = 0; m < RY + 2; m++) o[m] = (min(j0 + m - 1, n) + 1) * P + (ic + 1);
      if (ph == 2) {
        const TI *r = (const TI *)q.r[cur], *w = (const TI *)q.w[cur];
        const TI *s = (const TI *)q.s[cur];
        TI *r1 = (TI *)q.r[nxt], *w1 = (TI *)q.w[nxt], *s1 = (TI *)q.s[nxt];
        TI *pp = (TI *)q.p;
        const double alpha = q.alpha, beta = q.beta;
        TI rn[RY + 2], sn[RY + 2];
#pragma unroll
        for (int m = 0; m < RY + 2; m++) {
          rn[m] = (TI)0;
          sn[m] = (TI)0;
          if (inx) rn[m] = next_r<TI>(r[o[m]], w[o[m]], s[o[m]], alpha, beta, sn[m]);
        }
#pragma unroll
        for (int m = 0; m < RY; m++) {
          const int oc = o[m + 1];
          TI rw = __shfl_up_sync(full, rn[m + 1], 1);
          TI re = __shfl_down_sync(full, rn[m + 1], 1);
          TI dummy;
          if (lane == 0) rw = next_r<TI>(r[oc - 1], w[oc - 1], s[oc - 1], alpha, beta, dummy);
          if (lane == TX - 1 && inx)
            re = next_r<TI>(r[oc + 1], w[oc + 1], s[oc + 1], alpha, beta, dummy);
          if (!inx || j0 + m >= n) continue;
          const TI rc = rn[m + 1];
          const TI wn = (TI)(diag * (double)rc -
                             off * ((double)rw + (double)re + (double)rn[m] + (double)rn[m + 2]));
          const TI pn = (TI)((double)r[oc] + beta * (double)pp[oc]);
          if (mixed) {
            TI *y = (TI *)q.y;
            y[oc] = (TI)((double)y[oc] + alpha * (double)pn);
          } else {
            q.x[oc] = q.x[oc] + alpha * (double)pn;
          }
          pp[oc] = pn;
          r1[oc] = rc;
          s1[oc] = sn[m + 1];
          w1[oc] = wn;
          v[0] += (double)rc * (double)rc;
          v[1] += (double)wn * (double)rc;
        }
      } else if (ph == 0 || ph == 3) {
        // r = b - A (x + y) in FP64 (heat: b = x first at a new time step)
        const double *x = q.x;
        const TI *y = (const TI *)q.y;
        double xs[RY + 2];
#pragma unroll
        for (int m = 0; m < RY + 2; m++)
          xs[m] = inx ? x[o[m]] + (mixed ? (double)y[o[m]] : 0.0) : 0.0;
        TI *r = (TI *)q.r[cur];
#pragma unroll
        for (int m = 0; m < RY; m++) {
          const int oc = o[m + 1];
          double xw = __shfl_up_sync(full, xs[m + 1], 1);
          double xe = __shfl_down_sync(full, xs[m + 1], 1);
          if (lane == 0) xw = x[oc - 1] + (mixed ? (double)y[oc - 1] : 0.0);
          if (lane == TX - 1 && inx) xe = x[oc + 1] + (mixed ? (double)y[oc + 1] : 0.0);
          if (!inx || j0 + m >= n) continue;
          double bv = q.b[oc];
          if (q.newstep) {
            bv = xs[m + 1];
            q.b[oc] = bv;
          }
          const double ax = diag * xs[m + 1] - off * (xw + xe + xs[m] + xs[m + 2]);
          r[oc] = (TI)(bv - ax);
        }
      } else {  // phases 4, 5: w = A r, fold the correction, (r, r), (w, r)
        const TI *r = (const TI *)q.r[cur];
        TI *w = (TI *)q.w[cur];
        TI rs[RY + 2];
#pragma unroll
        for (int m = 0; m < RY + 2; m++) rs[m] = inx ? r[o[m]] : (TI)0;
#pragma unroll
        for (int m = 0; m < RY; m++) {
          const int oc = o[m + 1];
          TI rw = __shfl_up_sync(full, rs[m + 1], 1);
          TI re = __shfl_down_sync(full, rs[m + 1], 1);
          if (lane == 0) rw = r[oc - 1];
          if (lane == TX - 1 && inx) re = r[oc + 1];
          if (!inx || j0 + m >= n) continue;
          const TI rc = rs[m + 1];
          const TI wn = (TI)(diag * (double)rc -
                             off * ((double)rw + (double)re + (double)rs[m] + (double)rs[m + 2]));
          w[oc] = wn;
          if (mixed) {
            TI *y = (TI *)q.y;
            q.x[oc] = q.x[oc] + (double)y[oc];
            y[oc] = (TI)0;
          }
          v[0] += (double)rc * (double)rc;
          v[1] += (double)wn * (double)rc;
        }
      }
    }
    if (ph == 2 || ph == 4 || ph == 5) {  // uniform over the CTA
      block_sum<NPART>(v, sh);
      if (threadIdx.x == 0 && threadIdx.y == 0) {
        q.part[NPART * t] = v[0];
        q.part[NPART * t + 1] = v[1];
      }
    }
  }
}

// per-request fixed-order sums of the two partial columns
__device__ __forceinline__ void request_sums(const Req &q, double (*sh)[32], double &g,
                                             double &d) {
  double v[NPART] = {0.0, 0.0};
  for (int t = threadIdx.x; t < q.tiles; t += blockDim.x) {
    v[0] += q.part[NPART * t];
    v[1] += q.part[NPART * t + 1];
  }
  block_sum<NPART>(v, sh);
  g = v[0];
  d = v[1];
}

// after a converged solve: the next heat time step, or done
__device__ __forceinline__ void finish_solve(Req &q) {
  if (q.kind == OB2S_HEAT2D && q.step + 1 < q.steps) {
    q.step++;
    q.newstep = 1;
    q.outer = 0;
    q.phase = 0;
    return;
  }
  q.done = 1;
}

// Every request's next phase (thread 0 of one CTA per request slot; CTAs
// [MAXA, MAXA + nadi) advance the ADI requests' step counts).
__global__ void __launch_bounds__(256) scalars_b(const Work *__restrict__ W, Req *R) {
  __shared__ double sh[NPART][32];
  const int b = blockIdx.x;
  if (b >= MAXA) {
    const int k = b - MAXA;
    if (k >= W->nadi || threadIdx.x != 0) return;
    Req &q = R[W->adi_slot[k]];
    if (q.done) return;
    q.step++;
    q.iters = q.step;
    if (q.step >= q.steps) q.done = 1;
    return;
  }
  if (b >= W->npois) return;
  Req &q = R[W->pois_slot[b]];
  if (q.done) return;
  const int ph = q.phase;
  if (ph == 0 || ph == 3) {  // r written; w, the fold and the dots next
    if (threadIdx.x == 0) {
      q.newstep = 0;
      q.phase = ph == 0 ? 4 : 5;
    }
    return;
  }
  double g, dl;
  request_sums(q, sh, g, dl);
  if (threadIdx.x != 0) return;
  if (ph == 4 || ph == 5) {  // true residual: g = (r, r), dl = (w, r)
    if (q.outer == 0) q.rr0 = g;
    q.outer++;
    q.rel = q.rr0 > 0.0 ? sqrt(g / q.rr0) : 0.0;
    if (q.rel <= q.tol || q.outer > q.max_outer || q.iters >= q.max_inner || g == 0.0) {
      finish_solve(q);
      return;
    }
    double beta = 0.0, den = dl;
    if (ph == 5) {
      beta = g / q.gamma;
      den = dl - beta * g / q.alpha;
    }
    if (!(den > 0.0)) {  // breakdown: start again from the true residual
      q.phase = 0;
      return;
    }
    q.beta = beta;
    q.alpha = g / den;
    q.gamma = g;
    q.gamma_in0 = g;
    q.phase = 2;
    return;
  }
  // phase 2: recursive (r, r) and (w, r) of the new residual
  q.iters++;
  q.par ^= 1;
  const double drop = sqrt(g / q.gamma_in0);
  const double relr = q.rr0 > 0.0 ? sqrt(g / q.rr0) : 0.0;
  if (drop <= q.inner_tol || relr <= q.tol || q.iters >= q.max_inner || g == 0.0) {
    q.phase = 3;  // gamma and alpha stay those of the step just taken
    return;
  }
  const double beta = g / q.gamma;
  const double den = dl - beta * g / q.alpha;
  if (!(den > 0.0)) {
    q.phase = 3;  // loss of positivity: replace the residual and go on from it
    return;
  }
  q.beta = beta;
  q.alpha = g / den;
  q.gamma = g;
}

// ---------------------------------------------------------------- ADI
// grid of n^3 points including the Dirichlet boundary (adi/preproc_kernel.h)

__global__ void __launch_bounds__(256) adi_pre(const Work *__restrict__ W, Req *R) {
  const long long total = W->pre_pref[W->nadi];
  for (long long un = blockIdx.x; un < total; un += gridDim.x) {
    const int k = find_req(W->pre_pref, W->nadi, un);
    const Req &q = R[W->adi_slot[k]];
    if (q.done) continue;
    const int n = q.n;
    const int t = (int)(un - W->pre_pref[k]);
    const int tx = (n + 31) / 32, ty = (n + 7) / 8;
    const int i = (t % tx) * 32 + threadIdx.x;
    const int j = ((t / tx) % ty) * 8 + threadIdx.y;
    const int z = t / (tx * ty);
    if (i >= n || j >= n) continue;
    const long long o = ((long long)z * n + j) * n + i;
    const double *u = q.u;
    double d = 0.0;
    if (!(i == 0 || i == n - 1 || j == 0 || j == n - 1 || z == 0 || z == n - 1)) {
      const long long sy = n, sz = (long long)n * n;
      d = q.lambda * (u[o - 1] + u[o + 1] + u[o - sy] + u[o + sy] + u[o - sz] + u[o + sz] -
                      6.0 * u[o]);
    }
    q.du[o] = d;
  }
}

// x solve: 32 lines of one z plane staged through shared memory
__global__ void __launch_bounds__(128) adi_x(const Work *__restrict__ W, Req *R) {
  extern __shared__ double sm[];  // [ADI_XL][n + 1]
  const long long total = W->x_pref[W->nadi];
  for (long long un = blockIdx.x; un < total; un += gridDim.x) {
    const int k = find_req(W->x_pref, W->nadi, un);
    const Req &q = R[W->adi_slot[k]];
    if (q.done) continue;  // uniform over the CTA
    const int n = q.n, ld = n + 1;
    const int t = (int)(un - W->x_pref[k]);
    const int nyb = (n + ADI_XL - 1) / ADI_XL;
    const int y0 = (t % nyb) * ADI_XL, z = t / nyb;
    double *du = q.du + (long long)z * n * n;
    for (int e = threadIdx.x; e < ADI_XL * n; e += blockDim.x) {
      const int l = e / n, xi = e - l * n;
      if (y0 + l < n) sm[l * ld + xi] = du[(long long)(y0 + l) * n + xi];
    }
    __syncthreads();
    if (threadIdx.x < ADI_XL && y0 + threadIdx.x < n) {
      double *v = sm + threadIdx.x * ld;
      const double a = q.a_coef;
      double prev = v[0] * q.mm[0];
      v[0] = prev;
      for (int xi = 1; xi < n - 1; xi++) {
        prev = (v[xi] - a * prev) * q.mm[xi];
        v[xi] = prev;
      }
      v[n - 1] = v[n - 1] * q.mm[n - 1];  // Dirichlet row: a = 0
      double nxt = v[n - 1];
      for (int xi = n - 2; xi >= 0; xi--) {
        nxt = v[xi] - q.cp[xi] * nxt;
        v[xi] = nxt;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ADI_XL * n; e += blockDim.x) {
      const int l = e / n, xi = e - l * n;
      if (y0 + l < n) du[(long long)(y0 + l) * n + xi] = sm[l * ld + xi];
    }
    __syncthreads();
  }
}

// y (dir 1) or z (dir 2) solve: one thread per line, neighbouring threads on
// neighbouring x (coalesced); the z solve adds its solution into u
template <int DIR>
__global__ void __launch_bounds__(32 * ADI_YZ) adi_yz(const Work *__restrict__ W, Req *R) {
  const long long total = W->yz_pref[W->nadi];
  for (long long un = blockIdx.x; un < total; un += gridDim.x) {
    const int k = find_req(W->yz_pref, W->nadi, un);
    const Req &q = R[W->adi_slot[k]];
    if (q.done) continue;
    const int n = q.n;
    const int t = (int)(un - W->yz_pref[k]);
    const int nxb = (n + 31) / 32;
    const int i = (t % nxb) * 32 + threadIdx.x;
    const int c = (t / nxb) * ADI_YZ + threadIdx.y;  // the other coordinate
    if (i >= n || c >= n) continue;
    const long long s = DIR == 1 ? (long long)n : (long long)n * n;
    const long long base = DIR == 1 ? (long long)c * n * n + i : (long long)c * n + i;
    double *v = q.du + base;
    const double a = q.a_coef;
    double prev = v[0] * q.mm[0];
    v[0] = prev;
    for (int m = 1; m < n - 1; m++) {
      prev = (v[m * s] - a * prev) * q.mm[m];
      v[m * s] = prev;
    }
    v[(n - 1) * s] = v[(n - 1) * s] * q.mm[n - 1];  // Dirichlet row: a = 0
    double nxt = v[(n - 1) * s];
    if (DIR == 2) {
      double *u = q.u + base;
      u[(n - 1) * s] = u[(n - 1) * s] + nxt;
      for (int m = n - 2; m >= 0; m--) {
        nxt = v[m * s] - q.cp[m] * nxt;
        u[m * s] = u[m * s] + nxt;
      }
    } else {
      for (int m = n - 2; m >= 0; m--) {
        nxt = v[m * s] - q.cp[m] * nxt;
        v[m * s] = nxt;
      }
    }
  }
}

// ---------------------------------------------------------------- init

__global__ void pois_init(double *b, int n, int pitch, int seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= n) return;
  const double h = 1.0 / (n + 1);
  b[(long long)(j + 1) * pitch + i + 1] = h * h * (2.0 * hash_uniform(seed, i, j, 0) - 1.0);
}

// heat request: u0 ~ U(-1,1) into b and x
__global__ void heat_init(double *b, double *x, int n, int pitch, int seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= n) return;
  const double v = 2.0 * hash_uniform(seed, i, j, 3) - 1.0;
  b[(long long)(j + 1) * pitch + i + 1] = v;
  x[(long long)(j + 1) * pitch + i + 1] = v;
}

__global__ void adi_init(double *u, int n, int seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, z = blockIdx.z;
  if (i >= n) return;
  u[((long long)z * n + j) * n + i] = 2.0 * hash_uniform(seed, i, j, z + 1) - 1.0;
}

__global__ void interior_copy(const double *src, double *dst, int n, int pitch, int off) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= n) return;
  dst[(long long)j * n + i] = src[(long long)(j + off) * pitch + i + off];
}

}  // namespace

// ---------------------------------------------------------------- host side

struct ob2s_engine {
  int mode, tile_y;
  double tol, inner_tol;
  int max_inner;
  cudaStream_t st;
  int sms;
  Req *R_d;
  Work *W_d;
  std::vector<Req> R;       // host copy (refreshed after every run)
  std::vector<int> used;    // slot in use
  std::vector<int> active;  // slot is in the work list
  std::vector<int> reported;
  std::vector<void *> mem;  // per slot allocation
  std::vector<size_t> bytes;
  bool work_dirty;
  int pois_ctas_per_sm;  // resident CTAs per SM of the Poisson kernels
  struct Graph {
    int iters, variant, kernels;
    cudaGraphExec_t exec;
  };
  std::vector<Graph> graphs;
  long long launches;
};

static int rc(cudaError_t e) { return (int)e; }

static size_t elem_inner(int mode) { return mode == OB2S_MIXED ? 4 : 8; }

OB2_API size_t ob2s_request_bytes(int mode, int kind, int n) {
  if (kind == OB2S_POISSON2D || kind == OB2S_HEAT2D) {
    const size_t p = (size_t)(n + 2) * (n + 2);
    const size_t tiles = (size_t)((n + 31) / 32) * (size_t)((n + 7) / 8);  // at the smallest tile
    // x, b (FP64); r, w, s (two buffers each) and p; y in the mixed mode
    const size_t vec = 7 + (mode == OB2S_MIXED ? 1 : 0);
    return p * (16 + vec * elem_inner(mode)) + 8 * NPART * tiles + 4096;
  }
  return (size_t)n * n * n * 16 + (size_t)n * 16 + 4096;
}

// one engine iteration; the kernels of a request kind with no active
// request are left out (variant bit 0: Poisson, bit 1: ADI)
template <typename TI, int RY>
static int launch_iteration(ob2s_engine *e, int variant) {
  int k = 0;
  if (variant & 1) {
    const int g = e->sms * e->pois_ctas_per_sm;
    pois_pass<TI, RY><<<g, dim3(TX, CTA_Y), 0, e->st>>>(e->W_d, e->R_d);
    k += 1;
  }
  if (variant & 2) {
    adi_pre<<<e->sms * 8, dim3(32, 8), 0, e->st>>>(e->W_d, e->R_d);
    const size_t xsm = (size_t)ADI_XL * (ADI_MAX_N + 1) * sizeof(double);
    adi_x<<<e->sms * 4, 128, xsm, e->st>>>(e->W_d, e->R_d);
    adi_yz<1><<<e->sms * 16, dim3(32, ADI_YZ), 0, e->st>>>(e->W_d, e->R_d);
    adi_yz<2><<<e->sms * 16, dim3(32, ADI_YZ), 0, e->st>>>(e->W_d, e->R_d);
    k += 4;
  }
  scalars_b<<<2 * MAXA, 256, 0, e->st>>>(e->W_d, e->R_d);
  return k + 1;
}

static int launch_iteration_any(ob2s_engine *e, int variant) {
  const bool mixed = e->mode == OB2S_MIXED;
  switch (e->tile_y) {  // tile height = 8 rows per thread
    case 8:
      return mixed ? launch_iteration<float, 1>(e, variant) : launch_iteration<double, 1>(e, variant);
    case 16:
      return mixed ? launch_iteration<float, 2>(e, variant) : launch_iteration<double, 2>(e, variant);
    default:
      return mixed ? launch_iteration<float, 4>(e, variant) : launch_iteration<double, 4>(e, variant);
  }
}

OB2_API int ob2s_create(ob2s_engine **out, int mode, double tol, double inner_tol, int max_inner,
                        int tile_y) {
  if (mode != OB2S_FP64 && mode != OB2S_MIXED) return OB2S_ERR_BADARG;
  if (tile_y == 0) tile_y = 32;
  if (tile_y != 8 && tile_y != 16 && tile_y != 32) return OB2S_ERR_BADARG;
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return rc(err);
  ob2s_engine *e = new ob2s_engine();
  e->mode = mode;
  e->tile_y = tile_y;
  e->tol = tol;
  e->inner_tol = inner_tol;
  e->max_inner = max_inner > 0 ? max_inner : 100000;
  cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, dev);
  if ((err = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking)) != cudaSuccess ||
      (err = cudaMalloc(&e->R_d, sizeof(Req) * MAXA)) != cudaSuccess ||
      (err = cudaMalloc(&e->W_d, sizeof(Work))) != cudaSuccess ||
      (err = cudaMemset(e->R_d, 0, sizeof(Req) * MAXA)) != cudaSuccess ||
      (err = cudaMemset(e->W_d, 0, sizeof(Work))) != cudaSuccess ||
      (err = cudaFuncSetAttribute(adi_x, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(ADI_XL * (ADI_MAX_N + 1) * sizeof(double)))) !=
          cudaSuccess) {
    delete e;
    return rc(err);
  }
  {
    // persistent grids: as many CTAs as can be resident at once
    int nb = 0;
    const bool mixed = mode == OB2S_MIXED;
    auto occ = [&](const void *f) {
      int b = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, TX * CTA_Y, 0);
      return b;
    };
    switch (tile_y) {
      case 8:
        nb = occ(mixed ? (const void *)pois_pass<float, 1> : (const void *)pois_pass<double, 1>);
        break;
      case 16:
        nb = occ(mixed ? (const void *)pois_pass<float, 2> : (const void *)pois_pass<double, 2>);
        break;
      default:
        nb = occ(mixed ? (const void *)pois_pass<float, 4> : (const void *)pois_pass<double, 4>);
    }
    const int nb2 = nb;
    e->pois_ctas_per_sm = std::max(1, std::min(nb, nb2));
  }
  e->R.assign(MAXA, Req());
  memset(e->R.data(), 0, sizeof(Req) * MAXA);
  e->used.assign(MAXA, 0);
  e->active.assign(MAXA, 0);
  e->reported.assign(MAXA, 0);
  e->mem.assign(MAXA, nullptr);
  e->bytes.assign(MAXA, 0);
  e->work_dirty = true;
  e->launches = 0;
  *out = e;
  return 0;
}

OB2_API void ob2s_destroy(ob2s_engine *e) {
  if (!e) return;
  cudaStreamSynchronize(e->st);
  for (auto &g : e->graphs) cudaGraphExecDestroy(g.exec);
  for (int k = 0; k < MAXA; k++)
    if (e->mem[k]) cudaFreeAsync(e->mem[k], e->st);
  cudaStreamSynchronize(e->st);
  cudaFree(e->R_d);
  cudaFree(e->W_d);
  cudaStreamDestroy(e->st);
  delete e;
}

static void host_thomas_coefs(int n, double lambda, std::vector<double> &cp,
                              std::vector<double> &mm, double *a_out) {
  // rows 0 and n-1: identity (Dirichlet); interior: a = c = -lambda/2,
  // b = 1 + lambda (adi/preproc_kernel.h).  c'_i and 1/(b_i - a_i c'_{i-1}).
  const double a = -0.5 * lambda, b = 1.0 + lambda, c = -0.5 * lambda;
  cp.assign(n, 0.0);
  mm.assign(n, 0.0);
  mm[0] = 1.0;
  cp[0] = 0.0;
  for (int i = 1; i < n; i++) {
    const bool edge = i == n - 1;
    const double ai = edge ? 0.0 : a, bi = edge ? 1.0 : b, ci = edge ? 0.0 : c;
    mm[i] = 1.0 / (bi - ai * cp[i - 1]);
    cp[i] = ci * mm[i];
  }
  *a_out = a;
}

OB2_API int ob2s_submit(ob2s_engine *e, int kind, int n, int seed, int steps, int *id) {
  const bool grid2d = kind == OB2S_POISSON2D || kind == OB2S_HEAT2D;
  if (grid2d ? (n < 1 || n > 32768 || (kind == OB2S_HEAT2D && steps < 1))
             : (kind != OB2S_ADI3D || n < 3 || n > ADI_MAX_N || steps < 1))
    return OB2S_ERR_BADARG;
  int slot = -1;
  for (int k = 0; k < MAXA; k++)
    if (!e->used[k]) {
      slot = k;
      break;
    }
  if (slot < 0) return OB2S_ERR_FULL;
  const size_t nb = ob2s_request_bytes(e->mode, kind, n);
  void *m = nullptr;
  cudaError_t err = cudaMallocAsync(&m, nb, e->st);
  if (err != cudaSuccess) return rc(err);
  if ((err = cudaMemsetAsync(m, 0, nb, e->st)) != cudaSuccess) {
    cudaFreeAsync(m, e->st);
    return rc(err);
  }
  Req q;
  memset(&q, 0, sizeof(q));
  q.kind = kind;
  q.n = n;
  char *c = (char *)m;
  auto take = [&c](size_t b) {
    char *p = c;
    c += (b + 255) / 256 * 256;
    return (void *)p;
  };
  if (grid2d) {
    q.pitch = n + 2;
    q.tiles_x = (n + TX - 1) / TX;
    q.tiles = q.tiles_x * ((n + e->tile_y - 1) / e->tile_y);
    const size_t p = (size_t)q.pitch * q.pitch;
    const size_t ei = elem_inner(e->mode);
    // the layout ob2s_request_bytes counts (each array rounded up to 256
    // bytes: within its 4 KB slack); every array starts zeroed
    q.x = (double *)take(p * 8);
    q.b = (double *)take(p * 8);
    for (int c = 0; c < 2; c++) {
      q.r[c] = take(p * ei);
      q.w[c] = take(p * ei);
      q.s[c] = take(p * ei);
    }
    q.p = take(p * ei);
    q.y = e->mode == OB2S_MIXED ? take(p * ei) : nullptr;
    q.part = (double *)take((size_t)8 * NPART * q.tiles);
    if (kind == OB2S_HEAT2D) {  // backward Euler, dt = h^2: (1 + 4) x - (neighbours)
      q.diag = 1.0 + 4.0 * kHeatRho;
      q.off = kHeatRho;
      q.steps = steps;
    } else {
      q.diag = 4.0;
      q.off = 1.0;
    }
    q.tol = e->tol;
    q.inner_tol = e->inner_tol;
    q.max_inner = e->max_inner;
    q.max_outer = 1000;
  } else {
    q.u = (double *)take((size_t)n * n * n * 8);
    q.du = (double *)take((size_t)n * n * n * 8);
    q.cp = (double *)take((size_t)n * 8);
    q.mm = (double *)take((size_t)n * 8);
  }
  if ((size_t)(c - (char *)m) > nb) {  // cannot happen: the slack covers the rounding
    cudaFreeAsync(m, e->st);
    return OB2S_ERR_BADARG;
  }
  if (kind == OB2S_POISSON2D) {
    pois_init<<<dim3((n + 127) / 128, n), 128, 0, e->st>>>(q.b, n, q.pitch, seed);
  } else if (kind == OB2S_HEAT2D) {  // u0 is the first right-hand side and first guess
    heat_init<<<dim3((n + 127) / 128, n), 128, 0, e->st>>>(q.b, q.x, n, q.pitch, seed);
  } else {
    q.lambda = 1.0;
    q.steps = steps;
    std::vector<double> cp, mm;
    host_thomas_coefs(n, q.lambda, cp, mm, &q.a_coef);
    cudaMemcpyAsync(q.cp, cp.data(), (size_t)n * 8, cudaMemcpyHostToDevice, e->st);
    cudaMemcpyAsync(q.mm, mm.data(), (size_t)n * 8, cudaMemcpyHostToDevice, e->st);
    adi_init<<<dim3((n + 127) / 128, n, n), 128, 0, e->st>>>(q.u, n, seed);
    // the coefficient tables are copied from host vectors that go out of
    // scope: wait for them
    cudaStreamSynchronize(e->st);
  }
  err = cudaMemcpyAsync(e->R_d + slot, &q, sizeof(Req), cudaMemcpyHostToDevice, e->st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->st);
  if (err != cudaSuccess) {
    cudaFreeAsync(m, e->st);
    return rc(err);
  }
  err = cudaGetLastError();
  if (err != cudaSuccess) return rc(err);
  e->R[slot] = q;
  e->used[slot] = 1;
  e->active[slot] = 1;
  e->reported[slot] = 0;
  e->mem[slot] = m;
  e->bytes[slot] = nb;
  e->work_dirty = true;
  *id = slot;
  return 0;
}

static int upload_work(ob2s_engine *e) {
  Work w;
  memset(&w, 0, sizeof(w));
  for (int k = 0; k < MAXA; k++) {
    if (!e->active[k]) continue;
    const Req &q = e->R[k];
    if (q.kind != OB2S_ADI3D) {
      w.pois_slot[w.npois] = k;
      w.pois_pref[w.npois + 1] = w.pois_pref[w.npois] + q.tiles;
      w.npois++;
    } else {
      const int n = q.n;
      const int a = w.nadi;
      w.adi_slot[a] = k;
      w.pre_pref[a + 1] = w.pre_pref[a] + (long long)((n + 31) / 32) * ((n + 7) / 8) * n;
      w.x_pref[a + 1] = w.x_pref[a] + (long long)((n + ADI_XL - 1) / ADI_XL) * n;
      w.yz_pref[a + 1] = w.yz_pref[a] + (long long)((n + 31) / 32) * ((n + ADI_YZ - 1) / ADI_YZ);
      w.nadi++;
    }
  }
  cudaError_t err = cudaMemcpyAsync(e->W_d, &w, sizeof(w), cudaMemcpyHostToDevice, e->st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->st);  // w is a stack object
  e->work_dirty = false;
  return rc(err);
}

OB2_API int ob2s_run(ob2s_engine *e, int iters, int *ids, int cap, int *n_done) {
  if (iters < 1) return OB2S_ERR_BADARG;
  *n_done = 0;
  int err;
  if (e->work_dirty && (err = upload_work(e))) return err;
  int variant = 0;
  for (int k = 0; k < MAXA; k++)
    if (e->active[k]) variant |= e->R[k].kind != OB2S_ADI3D ? 1 : 2;
  if (variant) {
    ob2s_engine::Graph *gr = nullptr;
    for (auto &g : e->graphs)
      if (g.iters == iters && g.variant == variant) gr = &g;
    if (!gr) {
      cudaGraph_t graph;
      cudaGraphExec_t ge = nullptr;
      cudaError_t ce = cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal);
      if (ce != cudaSuccess) return rc(ce);
      int kernels = 0;
      for (int i = 0; i < iters; i++) kernels += launch_iteration_any(e, variant);
      ce = cudaStreamEndCapture(e->st, &graph);
      if (ce != cudaSuccess) return rc(ce);
      ce = cudaGraphInstantiate(&ge, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return rc(ce);
      e->graphs.push_back({iters, variant, kernels, ge});
      gr = &e->graphs.back();
    }
    cudaError_t ce = cudaGraphLaunch(gr->exec, e->st);
    if (ce != cudaSuccess) return rc(ce);
    e->launches += gr->kernels;
  }
  cudaError_t ce = cudaMemcpyAsync(e->R.data(), e->R_d, sizeof(Req) * MAXA,
                                   cudaMemcpyDeviceToHost, e->st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->st);
  if (ce != cudaSuccess) return rc(ce);
  for (int k = 0; k < MAXA; k++) {
    if (!e->used[k] || !e->R[k].done) continue;
    if (e->active[k]) {
      e->active[k] = 0;
      e->work_dirty = true;
    }
    if (!e->reported[k]) {
      e->reported[k] = 1;
      if (*n_done < cap) ids[*n_done] = k;
      (*n_done)++;
    }
  }
  return 0;
}

OB2_API int ob2s_active(ob2s_engine *e) {
  int n = 0;
  for (int k = 0; k < MAXA; k++) n += e->active[k];
  return n;
}

OB2_API int ob2s_fetch(ob2s_engine *e, int id, double *host, size_t count) {
  if (id < 0 || id >= MAXA || !e->used[id]) return OB2S_ERR_BADARG;
  const Req &q = e->R[id];
  if (!q.done) return OB2S_ERR_NOTDONE;
  const int n = q.n;
  if (q.kind != OB2S_ADI3D) {
    if (count < (size_t)n * n) return OB2S_ERR_BADARG;
    double *tmp = nullptr;
    cudaError_t ce = cudaMallocAsync(&tmp, (size_t)n * n * 8, e->st);
    if (ce != cudaSuccess) return rc(ce);
    interior_copy<<<dim3((n + 127) / 128, n), 128, 0, e->st>>>(q.x, tmp, n, q.pitch, 1);
    ce = cudaMemcpyAsync(host, tmp, (size_t)n * n * 8, cudaMemcpyDeviceToHost, e->st);
    cudaFreeAsync(tmp, e->st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->st);
    return rc(ce);
  }
  const size_t m = (size_t)n * n * n;
  if (count < m) return OB2S_ERR_BADARG;
  cudaError_t ce = cudaMemcpyAsync(host, q.u, m * 8, cudaMemcpyDeviceToHost, e->st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->st);
  return rc(ce);
}

OB2_API int ob2s_result_of(ob2s_engine *e, int id, ob2s_result *res) {
  if (id < 0 || id >= MAXA || !e->used[id]) return OB2S_ERR_BADARG;
  const Req &q = e->R[id];
  memset(res, 0, sizeof(*res));
  res->kind = q.kind;
  res->n = q.n;
  res->done = q.done;
  res->iterations = q.iters;
  res->outer = q.outer;
  res->rel_residual = q.rel;
  if (!q.done) return 0;
  const size_t m = q.kind != OB2S_ADI3D ? (size_t)q.n * q.n : (size_t)q.n * q.n * q.n;
  std::vector<double> h(m);
  int err = ob2s_fetch(e, id, h.data(), m);
  if (err) return err;
  double s = 0.0;
  for (size_t i = 0; i < m; i++) s += h[i];
  res->checksum = s;
  return 0;
}

OB2_API int ob2s_release(ob2s_engine *e, int id) {
  if (id < 0 || id >= MAXA || !e->used[id]) return OB2S_ERR_BADARG;
  cudaError_t ce = cudaStreamSynchronize(e->st);
  if (ce != cudaSuccess) return rc(ce);
  if (e->active[id]) e->work_dirty = true;
  cudaFreeAsync(e->mem[id], e->st);
  e->mem[id] = nullptr;
  e->used[id] = 0;
  e->active[id] = 0;
  e->bytes[id] = 0;
  // the slot's device state is left as is: no kernel reads a slot that is
  // not in the work list, and the work list is rebuilt before the next run
  return 0;
}

OB2_API long long ob2s_launches(ob2s_engine *e) { return e->launches; }
