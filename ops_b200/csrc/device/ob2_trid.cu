// ob2_trid.cu -- batched tridiagonal solves behind ops_tridMultiDimBatch(_Inc).
//
// The reference hands these to the external tridsolver library
// (ops/c/src/tridiag/ops_tridiag_cuda.cpp:96-251).  This backend solves them
// with its own register-blocked Thomas/PCR hybrid (the chunked scheme
// published by Laszlo, Giles and Appleyard, "Manycore algorithms for batch
// scalar and block tridiagonal solvers", ACM TOMS 42(4), 2016):
//
//   * a line of n points is cut into P nearly equal chunks (lengths differ by
//     at most one, every chunk 8..16 points when n > 16), one thread per
//     chunk, coefficients held in FP64 registers;
//   * each thread eliminates its chunk so that every row couples only to the
//     chunk's first and last unknowns ("modified Thomas");
//   * the chunk end rows form a tridiagonal system of 2P unknowns per line,
//     solved by parallel cyclic reduction in shared memory;
//   * each thread substitutes its chunk and writes the solution (or adds it
//     to u for the _Inc form, leaving d untouched).
//
// Each coefficient is read once and the solution written once: the DRAM
// traffic is the algorithmic 5 values per point (7 for _Inc).  For unit-stride
// lines the P threads of a line hold adjacent chunks; for strided lines
// neighbouring threads hold neighbouring lines, so every warp load is a
// contiguous run along x.  Elimination is FP64 for double and float storage.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ops_b200_device.h"

namespace {

constexpr int kMaxL = 16;          // max points per chunk (registers)
constexpr int kMaxThreads = 256;   // => max line length 4096

// After chunk_reduce, row i of a chunk of length L reads
//   a_i * x_first + x_i + c_i * x_last = d_i        (0 < i < L-1)
//   a_0 * x_prev  + x_0 + c_0 * x_last = d_0        (row 0)
//   a_{L-1} * x_0 + x_{L-1} + c_{L-1} * x_next = d_{L-1}   (row L-1)
// where x_prev / x_next are the end unknowns of the neighbouring chunks.
__device__ __forceinline__ void chunk_reduce(int L, double *a, double *b, double *c, double *d) {
  if (L <= 2) {
#pragma unroll
    for (int i = 0; i < 2; i++)
      if (i < L) {
        double r = 1.0 / b[i];
        a[i] *= r; c[i] *= r; d[i] *= r;
      }
    return;
  }
  {
    double r = 1.0 / b[0];
    a[0] *= r; c[0] *= r; d[0] *= r;
    r = 1.0 / b[1];
    a[1] *= r; c[1] *= r; d[1] *= r;
  }
  // forward: row i (i >= 2) loses x_{i-1}, gains x_0
#pragma unroll
  for (int i = 2; i < kMaxL; i++)
    if (i < L) {
      double r = 1.0 / (b[i] - a[i] * c[i - 1]);
      d[i] = r * (d[i] - a[i] * d[i - 1]);
      a[i] = -r * a[i] * a[i - 1];
      c[i] = r * c[i];
    }
  // backward: row i (L-3 >= i >= 1) loses x_{i+1}, gains x_{L-1}
#pragma unroll
  for (int i = kMaxL - 3; i >= 1; i--)
    if (i <= L - 3) {
      d[i] = d[i] - c[i] * d[i + 1];
      a[i] = a[i] - c[i] * a[i + 1];
      c[i] = -c[i] * c[i + 1];
    }
  // row 0 loses x_1, gains x_{L-1}
  {
    double r = 1.0 / (1.0 - c[0] * a[1]);
    d[0] = r * (d[0] - c[0] * d[1]);
    a[0] = r * a[0];
    c[0] = -r * c[0] * c[1];
  }
}

template <typename T, bool INC>
__global__ void __launch_bounds__(256) trid_hybrid_kernel(
    int n, int P, int LPB, long long nlines, int unit, long long stride, int o1n, long long o1s,
    long long o2s, const T *__restrict__ A, const T *__restrict__ B, const T *__restrict__ C,
    T *__restrict__ D, T *__restrict__ U) {
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  int l, p;
  if (unit) {
    p = tid % P;
    l = tid / P;
  } else {
    l = tid % LPB;
    p = tid / LPB;
  }
  const long long line = (long long)blockIdx.x * LPB + l;
  const bool active = line < nlines;
  const int m = 2 * P;
  double *ra = sm + (size_t)l * m * 3;
  double *rc = ra + m;
  double *rd = rc + m;

  long long base = 0;
  if (active) {
    long long i1 = line % o1n, i2 = line / o1n;
    base = i1 * o1s + i2 * o2s;
  }
  const int k0 = (int)(((long long)p * n) / P);
  const int k1 = (int)(((long long)(p + 1) * n) / P);
  const int len = active ? (k1 - k0) : 0;

  double a[kMaxL], b[kMaxL], c[kMaxL], d[kMaxL];
#pragma unroll
  for (int i = 0; i < kMaxL; i++) {
    a[i] = 0.0; b[i] = 1.0; c[i] = 0.0; d[i] = 0.0;
    if (i < len) {
      long long e = base + (long long)(k0 + i) * stride;
      a[i] = (double)A[e];
      b[i] = (double)B[e];
      c[i] = (double)C[e];
      d[i] = (double)D[e];
    }
  }
  if (len > 0 && k0 == 0) a[0] = 0.0;          // no left neighbour
  if (len > 0 && k1 == n) c[len - 1] = 0.0;    // no right neighbour

  chunk_reduce(len > 0 ? len : 1, a, b, c, d);

  if (len >= 2) {
    ra[2 * p] = a[0]; rc[2 * p] = c[0]; rd[2 * p] = d[0];
    ra[2 * p + 1] = a[len - 1]; rc[2 * p + 1] = c[len - 1]; rd[2 * p + 1] = d[len - 1];
  } else if (len == 1) {
    // only when P == 1: the single row is decoupled on both sides
    ra[0] = 0.0; rc[0] = 0.0; rd[0] = d[0];
    ra[1] = 0.0; rc[1] = 0.0; rd[1] = d[0];
  } else {
    ra[2 * p] = ra[2 * p + 1] = 0.0;
    rc[2 * p] = rc[2 * p + 1] = 0.0;
    rd[2 * p] = rd[2 * p + 1] = 0.0;
  }
  __syncthreads();

  // parallel cyclic reduction of the 2P end unknowns of each line
  for (int s = 1; s < m; s <<= 1) {
    double na[2], nc[2], nd[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int r = 2 * p + q;
      const double ar = ra[r], cr = rc[r], dr = rd[r];
      double a1 = 0.0, c1 = 0.0, d1 = 0.0, a2 = 0.0, c2 = 0.0, d2 = 0.0;
      const bool hl = r - s >= 0, hr = r + s < m;
      if (hl) { a1 = ra[r - s]; c1 = rc[r - s]; d1 = rd[r - s]; }
      if (hr) { a2 = ra[r + s]; c2 = rc[r + s]; d2 = rd[r + s]; }
      const double k1l = hl ? ar : 0.0, k2r = hr ? cr : 0.0;
      const double inv = 1.0 / (1.0 - k1l * c1 - k2r * a2);
      na[q] = -k1l * a1 * inv;
      nc[q] = -k2r * c2 * inv;
      nd[q] = (dr - k1l * d1 - k2r * d2) * inv;
    }
    __syncthreads();
    ra[2 * p] = na[0]; rc[2 * p] = nc[0]; rd[2 * p] = nd[0];
    ra[2 * p + 1] = na[1]; rc[2 * p + 1] = nc[1]; rd[2 * p + 1] = nd[1];
    __syncthreads();
  }

  if (len <= 0) return;
  const double xf = rd[2 * p];
  const double xl = rd[2 * p + 1];
#pragma unroll
  for (int i = 0; i < kMaxL; i++)
    if (i < len) {
      double x;
      if (i == 0)
        x = xf;
      else if (i == len - 1)
        x = xl;
      else
        x = d[i] - a[i] * xf - c[i] * xl;
      long long e = base + (long long)(k0 + i) * stride;
      if (INC)
        U[e] = (T)((double)U[e] + x);
      else
        D[e] = (T)x;
    }
}

template <typename T>
int launch(int ndim, int solvedim, const int *dims, const long long *strides, const void *a,
           const void *b, const void *c, void *d, void *u) {
  const int n = dims[solvedim];
  int o1 = -1, o2 = -1;
  for (int i = 0; i < 3; i++) {
    if (i == solvedim) continue;
    if (o1 < 0) o1 = i; else o2 = i;
  }
  const int d1 = o1 < ndim ? dims[o1] : 1;
  const int d2 = o2 < ndim ? dims[o2] : 1;
  const long long s1 = o1 < ndim ? strides[o1] : 0;
  const long long s2 = o2 < ndim ? strides[o2] : 0;
  const long long nlines = (long long)d1 * d2;
  if (n <= 0 || nlines <= 0) return 0;
  const int P = (n + kMaxL - 1) / kMaxL;
  if (P > kMaxThreads) return (int)cudaErrorInvalidValue;
  const int unit = strides[solvedim] == 1 ? 1 : 0;
  int LPB = 256 / P;
  if (LPB < 1) LPB = 1;
  const int threads = LPB * P;
  const size_t shmem = (size_t)LPB * 2 * P * 3 * sizeof(double);
  const long long grid = (nlines + LPB - 1) / LPB;
  if (grid > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)ob2_dev_stream();
  if (u)
    trid_hybrid_kernel<T, true><<<(unsigned)grid, threads, shmem, st>>>(
        n, P, LPB, nlines, unit, strides[solvedim], d1, s1, s2, (const T *)a, (const T *)b,
        (const T *)c, (T *)d, (T *)u);
  else
    trid_hybrid_kernel<T, false><<<(unsigned)grid, threads, shmem, st>>>(
        n, P, LPB, nlines, unit, strides[solvedim], d1, s1, s2, (const T *)a, (const T *)b,
        (const T *)c, (T *)d, (T *)nullptr);
  return (int)cudaGetLastError();
}

}  // namespace

OB2_API int ob2_trid_batch(int type_size, int ndim, int solvedim, const int *dims,
                           const long long *strides, const void *a, const void *b,
                           const void *c, void *d, void *u) {
  if (ndim < 1 || ndim > 3 || solvedim < 0 || solvedim >= ndim) return (int)cudaErrorInvalidValue;
  int dd[3] = {1, 1, 1};
  long long ss[3] = {0, 0, 0};
  for (int i = 0; i < ndim; i++) {
    dd[i] = dims[i];
    ss[i] = strides[i];
  }
  if (type_size == 8) return launch<double>(ndim, solvedim, dd, ss, a, b, c, d, u);
  if (type_size == 4) return launch<float>(ndim, solvedim, dd, ss, a, b, c, d, u);
  return (int)cudaErrorInvalidValue;
}
