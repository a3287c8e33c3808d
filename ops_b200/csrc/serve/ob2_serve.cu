// ob2_serve.cu -- the solve-serving engine (include/ops_b200_serve.h).
//
// Device state: an array of request slots (struct Req, FP64 CG scalars
// included) and a work list (struct Work) naming the active requests with
// prefix sums of their work units.  Every batched kernel is persistent: a
// grid of a few CTAs per SM walks the global unit index over all active
// requests, finds the request by binary search in the prefix table, and works
// on that request's tile.  One engine iteration:
//   pois_pw       p' = r + beta p, w = A p', per-tile (p', w)
//   scalars_a     alpha per Poisson request
//   pois_xr       x += alpha p' (FP64), r -= alpha w, per-tile (r, r); or
//                 the FP64 residual b - A x
//   adi_pre       right-hand side of the ADI step (adi/preproc_kernel.h)
//   adi_x/y/z     constant-coefficient Thomas solves (z adds into u)
//   scalars_b     per request: fixed-order sum of its tile partials, beta,
//                 residual replacement and convergence; ADI step count
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

constexpr int TX = 32;       // CTA x extent (one warp per row of a tile)
constexpr int TXC = 2 * TX;  // columns per tile: two adjacent columns per thread
constexpr int C0 = 2;        // storage column of interior column 0 (even: 2-column
                             // accesses are 8- or 16-byte aligned)
constexpr int MAXA = OB2S_MAX_ACTIVE;
constexpr int ADI_MAX_N = 192;  // x-solve tile: 32 lines x n points in shared memory
constexpr int ADI_XL = 32;      // lines per x-solve unit
// (OB2S_HEAT2D is declared in ops_b200_serve.h)
constexpr int ADI_YZ = 4;       // planes per y/z-solve unit (CTA 32 x 4 lines)
constexpr double kHeatRho = 1.0;  // heat requests: dt / h^2 of the implicit step

struct Req {
  int kind, n, pitch, tiles_x, tiles;
  int phase, done, outer, inner_it, iters;
  int max_inner, max_outer, steps, step;
  int par;  // p buffer parity
  int newstep;  // heat: the next residual pass starts a time step (b = x)
  double tol, inner_tol;
  double alpha, beta, gamma, gamma_in0, rr0, rel;
  double diag, off;  // heat operator: diag x - off (sum of the 4 neighbours)
  double *x, *b, *part;
  void *r, *w, *p0, *p1;
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
// Layout of a 2D request's arrays: rows -1 .. n (the zero halo rows) at
// storage rows 0 .. n+1, row pitch P even and at least n + 3, interior
// column i at storage column i + C0 (column -1, the left halo, at C0 - 1;
// column n, the right halo, at n + C0); every unused element is zero.
// CTA 32 x 8 threads; each thread handles two adjacent columns (one 8- or
// 16-byte access per array and row) and RY consecutive rows, so a tile is
// 64 x (8 RY) points.  Loads of out-of-range rows are clamped to the last
// interior row (always valid memory) and only the stores are guarded, so the
// loads of all RY rows are issued before any store.
//
// Poisson and heat requests: conjugate gradients (the standard
// two-reduction form) with the iterate x in FP64, the vectors r, w, p in TI
// (FP32 in the mixed mode, FP64 otherwise) and every dot product accumulated
// in FP64.  Poisson: A x = 4 x - (neighbours); heat (one backward-Euler step
// per solve, dt / h^2 = rho): A x = (1 + 4 rho) x - rho (neighbours), b the
// previous step's solution.  The recursive residual is replaced by the true
// one, b - A x computed in FP64, whenever it has dropped by inner_tol since
// the last true residual or meets the tolerance (reliable updates: the
// search direction is kept, so the Krylov convergence of FP64 CG is kept
// too; an FP32 iterate or an FP32 correction accumulated between
// replacements needs far more iterations on fine grids: 10575 instead of
// 5781 at 2048^2, measured).
// Phases:
//   0  start (and restart after a breakdown; for heat requests also the start
//      of each time step, which first sets b = x): r = b - A x in FP64
//   2  CG iteration: p' = r + beta p, w = A p', (p', w)   [pois_pw]
//                    alpha = gamma / (p', w)               [scalars_a]
//                    x += alpha p', r -= alpha w, (r, r)   [pois_xr]
//                    beta, gamma; replacement test         [scalars_b]
//   3  replacement: r = b - A x in FP64, convergence test on it; beta from
//      the true (r, r), p kept
// p is double-buffered (p[par] read, p[par ^ 1] written by pois_pw), since
// pois_pw forms p' of the stencil neighbours itself: w = A p' needs p' at
// the neighbours, and recomputing r + beta p there avoids a separate pass.

constexpr int CTA_Y = 8;
constexpr int NPART = 2;  // partial sums per tile: (p', w) and (r, r)

// two adjacent elements of type T
template <typename T> struct V2;
template <> struct V2<float> { typedef float2 type; };
template <> struct V2<double> { typedef double2 type; };
template <typename T>
__device__ __forceinline__ typename V2<T>::type ld2(const T *p) {
  return *(const typename V2<T>::type *)p;
}
template <typename T>
__device__ __forceinline__ void st2(T *p, T a, T b) {
  typename V2<T>::type v;
  v.x = a;
  v.y = b;
  *(typename V2<T>::type *)p = v;
}

// resident CTAs per SM the Poisson kernels are compiled for (register cap):
// 4 for FP32 vectors; 3 for FP64 ones, whose two columns of RY rows need
// more than 64 registers without spilling
#ifndef OB2S_MINB
#define OB2S_MINB 4
#endif
#define POIS_BOUNDS __launch_bounds__(256, sizeof(TI) == 8 ? 3 : OB2S_MINB)

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

// p' = r + beta p and w = A p' over the tile, (p', w) per tile (phase 2)
template <typename TI, int RY>
__global__ void POIS_BOUNDS pois_pw(const Work *__restrict__ W, Req *R) {
  __shared__ double sh[1][32];
  const long long total = W->pois_pref[W->npois];
  for (long long un = blockIdx.x; un < total; un += gridDim.x) {
    const int k = find_req(W->pois_pref, W->npois, un);
    const Req &q = R[W->pois_slot[k]];
    if (q.done || q.phase != 2) continue;  // uniform over the CTA
    const int t = (int)(un - W->pois_pref[k]);
    const int n = q.n, P = q.pitch;
    const int i = (t % q.tiles_x) * TXC + 2 * threadIdx.x;  // columns i, i + 1
    const int j0 = (t / q.tiles_x) * (CTA_Y * RY) + threadIdx.y * RY;
    double v[1] = {0.0};
    if (j0 < n) {  // uniform over the warp (one threadIdx.y per warp)
      const TI *rr = (const TI *)q.r;
      const TI *pin = (const TI *)(q.par ? q.p1 : q.p0);
      TI *pout = (TI *)(q.par ? q.p0 : q.p1);
      TI *ww = (TI *)q.w;
      const TI beta = (TI)q.beta;
      const bool in0 = i < n, in1 = i + 1 < n;
      const int ic = in0 ? i : ((n - 1) & ~1);  // lanes past the edge load valid memory
      const int lane = threadIdx.x;
      // p' = r + beta p on rows j0-1 .. j0+RY of columns i, i+1 (storage rows
      // clamped into the array; the halo rows and columns of r and p hold
      // zeros); a column past the right edge stands for the zero halo
      TI p0[RY + 2], p1[RY + 2];
      int o[RY + 2];  // (n + 2) P < 2^31 for n <= 32768
#pragma unroll
      for (int m = 0; m < RY + 2; m++) {
        o[m] = (min(j0 + m - 1, n) + 1) * P + ic + C0;
        const auto rv = ld2(rr + o[m]);
        const auto pv = ld2(pin + o[m]);
        p0[m] = in0 ? rv.x + beta * pv.x : (TI)0;
        p1[m] = in1 ? rv.y + beta * pv.y : (TI)0;
      }
#pragma unroll
      for (int m = 0; m < RY; m++) {
        // column i - 1 is the left lane's second column, column i + 2 the
        // right lane's first; the warp's edge lanes form theirs from memory
        // (the same arithmetic, same bits)
        TI pw = __shfl_up_sync(0xffffffffu, p1[m + 1], 1);
        TI pe = __shfl_down_sync(0xffffffffu, p0[m + 1], 1);
        if (lane == 0) pw = rr[o[m + 1] - 1] + beta * pin[o[m + 1] - 1];
        if (lane == TX - 1 && in1) pe = rr[o[m + 1] + 2] + beta * pin[o[m + 1] + 2];
        if (!in0 || j0 + m >= n) continue;
        const TI c0 = p0[m + 1], c1 = p1[m + 1];
        TI a0, a1;
        if (q.kind == OB2S_HEAT2D) {
          a0 = (TI)q.diag * c0 - (TI)q.off * (pw + c1 + p0[m] + p0[m + 2]);
          a1 = in1 ? (TI)q.diag * c1 - (TI)q.off * (c0 + pe + p1[m] + p1[m + 2]) : (TI)0;
        } else {
          a0 = (TI)4 * c0 - pw - c1 - p0[m] - p0[m + 2];
          a1 = in1 ? (TI)4 * c1 - c0 - pe - p1[m] - p1[m + 2] : (TI)0;
        }
        // column n (the right halo) gets zeros when i + 1 == n
        st2(pout + o[m + 1], c0, c1);
        st2(ww + o[m + 1], a0, a1);
        v[0] += (double)c0 * (double)a0 + (double)c1 * (double)a1;
      }
    }
    block_sum<1>(v, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) q.part[NPART * t] = v[0];
  }
}

// phase 2: x += alpha p' (FP64), r -= alpha w, (r, r); phases 0, 3:
// r = b - A x in FP64 and its (r, r).  Column n (the right halo) is written
// only with zeros: there p', w and r are zero, so x keeps its zero.
template <typename TI, int RY>
__global__ void POIS_BOUNDS pois_xr(const Work *__restrict__ W, Req *R) {
  __shared__ double sh[2][32];
  const long long total = W->pois_pref[W->npois];
  for (long long un = blockIdx.x; un < total; un += gridDim.x) {
    const int k = find_req(W->pois_pref, W->npois, un);
    const Req &q = R[W->pois_slot[k]];
    if (q.done) continue;  // uniform over the CTA
    const int ph = q.phase;
    const int t = (int)(un - W->pois_pref[k]);
    const int n = q.n, P = q.pitch;
    const int i = (t % q.tiles_x) * TXC + 2 * threadIdx.x;  // columns i, i + 1
    const int j0 = (t / q.tiles_x) * (CTA_Y * RY) + threadIdx.y * RY;
    double v[2] = {0.0, 0.0};
    if (i < n && j0 < n) {
      const bool in1 = i + 1 < n;
      int o[RY];  // (n + 2) P < 2^31 for n <= 32768
#pragma unroll
      for (int m = 0; m < RY; m++) o[m] = (min(j0 + m, n - 1) + 1) * P + i + C0;
      TI *rr = (TI *)q.r;
      double *x = q.x;
      if (ph == 2) {
        const TI *pn = (const TI *)(q.par ? q.p0 : q.p1);  // written by pois_pw
        const TI *ww = (const TI *)q.w;
        const double alpha64 = q.alpha;
        const TI alpha = (TI)q.alpha;
        double x0[RY], x1[RY];
        TI r0[RY], r1[RY];
#pragma unroll
        for (int m = 0; m < RY; m++) {
          const auto pv = ld2(pn + o[m]);
          const auto wv = ld2(ww + o[m]);
          const auto rv = ld2(rr + o[m]);
          const double2 xv = ld2(x + o[m]);
          x0[m] = xv.x + alpha64 * (double)pv.x;
          x1[m] = xv.y + alpha64 * (double)pv.y;
          r0[m] = rv.x - alpha * wv.x;
          r1[m] = rv.y - alpha * wv.y;
        }
#pragma unroll
        for (int m = 0; m < RY; m++) {
          if (j0 + m >= n) continue;
          st2(x + o[m], x0[m], x1[m]);
          st2(rr + o[m], r0[m], r1[m]);
          v[0] += (double)r0[m] * (double)r0[m] + (double)r1[m] * (double)r1[m];
        }
      } else {
        double *b = q.b;
        double s0[RY], s1[RY];
#pragma unroll
        for (int m = 0; m < RY; m++) {
          const int e = o[m];
          const double2 c = ld2(x + e), up = ld2(x + e - P), dn = ld2(x + e + P);
          const double xw = x[e - 1], xe = x[e + 2];
          double2 bv = ld2(b + e);
          if (q.kind == OB2S_HEAT2D) {
            if (q.newstep) {  // a new time step: its right-hand side is the last solution
              bv = c;
              if (j0 + m < n) {
                st2(b + e, bv.x, bv.y);
                v[1] += bv.x * bv.x + bv.y * bv.y;  // ||b||^2: the step's residuals are relative to it
              }
            }
            s0[m] = bv.x - (q.diag * c.x - q.off * (xw + c.y + up.x + dn.x));
            s1[m] = in1 ? bv.y - (q.diag * c.y - q.off * (c.x + xe + up.y + dn.y)) : 0.0;
          } else {
            s0[m] = bv.x - (4.0 * c.x - xw - c.y - up.x - dn.x);
            s1[m] = in1 ? bv.y - (4.0 * c.y - c.x - xe - up.y - dn.y) : 0.0;
          }
        }
#pragma unroll
        for (int m = 0; m < RY; m++) {
          if (j0 + m >= n) continue;
          st2(rr + o[m], (TI)s0[m], (TI)s1[m]);
          v[0] += s0[m] * s0[m] + s1[m] * s1[m];
        }
      }
    }
    block_sum<2>(v, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      q.part[NPART * t + 1] = v[0];
      // column 0 is free in phase 0 (pois_pw did not run): ||b||^2 of a new
      // heat time step
      if (ph == 0 && q.newstep) q.part[NPART * t] = v[1];
    }
  }
}

// per-request fixed-order sum of one partial column
__device__ __forceinline__ double request_sum(const Req &q, int col, double (*sh)[32]) {
  double v[1] = {0.0};
  for (int t = threadIdx.x; t < q.tiles; t += blockDim.x) v[0] += q.part[NPART * t + col];
  block_sum<1>(v, sh);
  return v[0];
}

// alpha = gamma / (p', w) for requests in phase 2
__global__ void __launch_bounds__(256) scalars_a(const Work *__restrict__ W, Req *R) {
  __shared__ double sh[1][32];
  const int b = blockIdx.x;
  if (b >= W->npois) return;
  Req &q = R[W->pois_slot[b]];
  if (q.done || q.phase != 2) return;
  const double pw = request_sum(q, 0, sh);
  if (threadIdx.x != 0) return;
  if (!(pw > 0.0)) {  // breakdown: pois_xr computes the true residual and
    q.phase = 0;       // scalars_b restarts from it with beta = 0
    return;
  }
  q.alpha = q.gamma / pw;
}

// (r, r) step of every Poisson request; CTAs [MAXA, MAXA + nadi) advance
// the ADI requests' step counts
__global__ void __launch_bounds__(256) scalars_b(const Work *__restrict__ W, Req *R) {
  __shared__ double sh[1][32];
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
  const bool newstep = ph == 0 && q.newstep;  // uniform over the CTA
  const double g = request_sum(q, 1, sh);
  const double bb = newstep ? request_sum(q, 0, sh) : 0.0;
  if (threadIdx.x != 0) return;
  if (ph == 0 || ph == 3) {  // g = (b - A x, b - A x) in FP64
    if (newstep) {  // heat: relative to the step's right-hand side
      q.rr0 = bb;
      q.newstep = 0;
    } else if (q.outer == 0) {
      q.rr0 = g;  // Poisson starts from x = 0: (b, b)
    }
    q.outer++;
    q.rel = q.rr0 > 0.0 ? sqrt(g / q.rr0) : 0.0;
    if (q.rel <= q.tol || q.outer > q.max_outer || q.iters >= q.max_inner) {
      if (q.kind == OB2S_HEAT2D && q.rel <= q.tol && q.step + 1 < q.steps) {
        q.step++;  // next backward-Euler step, from this solution
        q.newstep = 1;
        q.outer = 0;
        q.phase = 0;
        return;
      }
      q.done = 1;
      return;
    }
    q.beta = ph == 0 ? 0.0 : g / q.gamma;
    q.gamma = g;
    q.gamma_in0 = g;
    q.phase = 2;
    return;
  }
  q.iters++;
  q.par ^= 1;
  const double drop = sqrt(g / q.gamma_in0);
  const double relr = q.rr0 > 0.0 ? sqrt(g / q.rr0) : 0.0;
  if (drop <= q.inner_tol || relr <= q.tol || q.iters >= q.max_inner || g == 0.0) {
    q.phase = 3;  // gamma stays the previous (r, r) for beta
    return;
  }
  q.beta = g / q.gamma;
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
  b[(long long)(j + 1) * pitch + i + C0] = h * h * (2.0 * hash_uniform(seed, i, j, 0) - 1.0);
}

// heat request: u0 ~ U(-1,1) into b and x
__global__ void heat_init(double *b, double *x, int n, int pitch, int seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= n) return;
  const double v = 2.0 * hash_uniform(seed, i, j, 3) - 1.0;
  b[(long long)(j + 1) * pitch + i + C0] = v;
  x[(long long)(j + 1) * pitch + i + C0] = v;
}

__global__ void adi_init(double *u, int n, int seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, z = blockIdx.z;
  if (i >= n) return;
  u[((long long)z * n + j) * n + i] = 2.0 * hash_uniform(seed, i, j, z + 1) - 1.0;
}

// rows [roff, roff + n) x columns [coff, coff + n) of src into dst (n x n)
__global__ void interior_copy(const double *src, double *dst, int n, int pitch, int roff,
                              int coff) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= n) return;
  dst[(long long)j * n + i] = src[(long long)(j + roff) * pitch + i + coff];
}

// checksum of a request's solution in a fixed order: CTA c of kSumCtas sums
// rows [c R / G, (c + 1) R / G) of the R rows of ncols elements (element
// (i, r) at off + r pitch + i), thread-strided, then block_sum; one CTA sums
// the partials in order
constexpr int kSumCtas = 256;
__global__ void __launch_bounds__(256) sum_rows(const double *src, long long nrows, int ncols,
                                                long long pitch, long long off, double *part) {
  __shared__ double sh[1][32];
  const long long G = gridDim.x, c = blockIdx.x;
  const long long r0 = nrows * c / G, r1 = nrows * (c + 1) / G;
  double v[1] = {0.0};
  for (long long r = r0; r < r1; r++)
    for (int i = threadIdx.x; i < ncols; i += blockDim.x) v[0] += src[off + r * pitch + i];
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) part[c] = v[0];
}
__global__ void __launch_bounds__(256) sum_parts(const double *part, int np, double *out) {
  __shared__ double sh[1][32];
  double v[1] = {0.0};
  for (int k = threadIdx.x; k < np; k += blockDim.x) v[0] += part[k];
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) *out = v[0];
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
  // the requests' memory: a pool of the engine's own that keeps freed
  // memory mapped (a request admitted after another retired reuses its
  // pages instead of mapping new ones)
  cudaMemPool_t pool;
  double *sum_d;  // checksum scratch: kSumCtas partials and the result
};

static int rc(cudaError_t e) { return (int)e; }

static size_t elem_inner(int mode) { return mode == OB2S_MIXED ? 4 : 8; }

OB2_API size_t ob2s_request_bytes(int mode, int kind, int n) {
  if (kind == OB2S_POISSON2D || kind == OB2S_HEAT2D) {
    const size_t p = (size_t)((n + 4) & ~1) * (n + 2);  // pitch x rows
    const size_t tiles = (size_t)((n + TXC - 1) / TXC) * (size_t)((n + 7) / 8);  // smallest tile
    return p * (16 + 4 * elem_inner(mode)) + 8 * NPART * tiles + 4096;
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
    pois_pw<TI, RY><<<g, dim3(TX, CTA_Y), 0, e->st>>>(e->W_d, e->R_d);
    scalars_a<<<MAXA, 256, 0, e->st>>>(e->W_d, e->R_d);
    pois_xr<TI, RY><<<g, dim3(TX, CTA_Y), 0, e->st>>>(e->W_d, e->R_d);
    k += 3;
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
    int nb = 0, nb2 = 0;
    const bool mixed = mode == OB2S_MIXED;
    auto occ = [&](const void *f) {
      int b = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, TX * CTA_Y, 0);
      return b;
    };
    switch (tile_y) {
      case 8:
        nb = occ(mixed ? (const void *)pois_pw<float, 1> : (const void *)pois_pw<double, 1>);
        nb2 = occ(mixed ? (const void *)pois_xr<float, 1> : (const void *)pois_xr<double, 1>);
        break;
      case 16:
        nb = occ(mixed ? (const void *)pois_pw<float, 2> : (const void *)pois_pw<double, 2>);
        nb2 = occ(mixed ? (const void *)pois_xr<float, 2> : (const void *)pois_xr<double, 2>);
        break;
      default:
        nb = occ(mixed ? (const void *)pois_pw<float, 4> : (const void *)pois_pw<double, 4>);
        nb2 = occ(mixed ? (const void *)pois_xr<float, 4> : (const void *)pois_xr<double, 4>);
    }
    e->pois_ctas_per_sm = std::max(1, std::min(nb, nb2));
  }
  {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    unsigned long long keep = ~0ULL;  // never return freed memory to the device
    if ((err = cudaMemPoolCreate(&e->pool, &props)) != cudaSuccess) {
      cudaStreamDestroy(e->st);
      cudaFree(e->R_d);
      cudaFree(e->W_d);
      delete e;
      return rc(err);
    }
    cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if ((err = cudaMalloc(&e->sum_d, sizeof(double) * (kSumCtas + 1))) != cudaSuccess) {
      cudaMemPoolDestroy(e->pool);
      cudaStreamDestroy(e->st);
      cudaFree(e->R_d);
      cudaFree(e->W_d);
      delete e;
      return rc(err);
    }
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

OB2_API int ob2s_reserve(ob2s_engine *e, size_t bytes) {
  if (!e) return OB2S_ERR_BADARG;
  if (bytes == 0) return 0;
  void *m = nullptr;
  cudaError_t err = cudaMallocFromPoolAsync(&m, bytes, e->pool, e->st);
  if (err != cudaSuccess) {
    cudaGetLastError();  // too large for the device: not sticky, leave no trace
    return rc(err);
  }
  err = cudaFreeAsync(m, e->st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->st);
  return rc(err);
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
  cudaFree(e->sum_d);
  cudaMemPoolDestroy(e->pool);
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
  cudaError_t err = cudaMallocFromPoolAsync(&m, nb, e->pool, e->st);
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
    q.pitch = (n + 4) & ~1;  // even, >= n + 3: columns 0 .. n + C0
    q.tiles_x = (n + TXC - 1) / TXC;
    q.tiles = q.tiles_x * ((n + e->tile_y - 1) / e->tile_y);
    const size_t p = (size_t)q.pitch * (n + 2);
    const size_t ei = elem_inner(e->mode);
    // the layout ob2s_request_bytes counts (seven arrays, each rounded up to
    // 256 bytes: within its 4 KB slack)
    q.x = (double *)take(p * 8);
    q.b = (double *)take(p * 8);
    q.r = take(p * ei);
    q.w = take(p * ei);
    q.p0 = take(p * ei);
    q.p1 = take(p * ei);
    q.part = (double *)take((size_t)8 * NPART * q.tiles);
    if (kind == OB2S_HEAT2D) {  // backward Euler: (1 + 4 rho) x - rho (neighbours)
      q.diag = 1.0 + 4.0 * kHeatRho;
      q.off = kHeatRho;
      q.steps = steps;
      q.newstep = 1;  // the first step's right-hand side is u0 (= x)
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
  } else if (kind == OB2S_HEAT2D) {  // u0 is the first right-hand side and guess
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
    cudaError_t ce = cudaMallocFromPoolAsync(&tmp, (size_t)n * n * 8, e->pool, e->st);
    if (ce != cudaSuccess) return rc(ce);
    interior_copy<<<dim3((n + 127) / 128, n), 128, 0, e->st>>>(q.x, tmp, n, q.pitch, 1, C0);
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
  const int n = q.n;
  if (q.kind != OB2S_ADI3D)  // interior rows 1 .. n, columns C0 .. C0 + n - 1
    sum_rows<<<kSumCtas, 256, 0, e->st>>>(q.x, n, n, q.pitch, (long long)q.pitch + C0, e->sum_d);
  else
    sum_rows<<<kSumCtas, 256, 0, e->st>>>(q.u, (long long)n * n, n, n, 0, e->sum_d);
  sum_parts<<<1, 256, 0, e->st>>>(e->sum_d, kSumCtas, e->sum_d + kSumCtas);
  double s = 0.0;
  cudaError_t ce = cudaMemcpyAsync(&s, e->sum_d + kSumCtas, sizeof(double),
                                   cudaMemcpyDeviceToHost, e->st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->st);
  if (ce != cudaSuccess) return rc(ce);
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
