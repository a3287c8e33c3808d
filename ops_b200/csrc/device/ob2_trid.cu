// ob2_trid.cu -- batched tridiagonal solves behind ops_tridMultiDimBatch(_Inc).
//
// The reference hands these to the external tridsolver library
// (ops/c/src/tridiag/ops_tridiag_cuda.cpp:96-251).  This backend solves them
// with its own register-blocked Thomas/PCR hybrid (the chunked scheme
// published by Laszlo, Giles and Appleyard, "Manycore algorithms for batch
// scalar and block tridiagonal solvers", ACM TOMS 42(4), 2016):
//
//   * a line of n points is cut into P = ceil(n/CL) chunks of CL points (the
//     last one padded with identity rows), one thread per chunk, the chunk's
//     coefficients held in FP64 registers;
//   * each thread eliminates its chunk so that every row couples only to the
//     chunk's first and last unknowns ("modified Thomas");
//   * the chunk end rows form a tridiagonal system of 2P unknowns per line,
//     solved by parallel cyclic reduction (PCR);
//   * each thread substitutes its chunk and writes the solution (or adds it
//     to u for the _Inc form, leaving d untouched).
//
// Lines of up to 256 points: unit-stride lines (x) one warp per line with
// vector loads and stores of each lane's 8-point chunk (trid_xw_kernel);
// strided lines (y, z) 8 neighbouring lines per CTA, consecutive threads on
// the same chunk of neighbouring lines so that every warp access is
// contiguous runs along x, each line's PCR in one warp after one exchange
// through shared memory (trid_lmw_kernel).  The reciprocals of the
// eliminations come from a Newton-Raphson refinement of the hardware
// approximation (rcp64).  Other forms stay selectable (OB2_TRID_*): a
// scalar warp-per-line kernel, a staged one, line-major CTA kernels with
// the PCR in shared memory, a pipelined persistent one, and the Thomas
// algorithm one thread per line (trid_thomas_kernel).  Longer lines use a
// CTA per group of lines with PCR in shared memory.  Each coefficient is read once and the
// solution written once: the DRAM traffic is the algorithmic 5 values per
// point (7 for _Inc).  Elimination is FP64 for double and float storage.
// Every register array is indexed with compile-time indices only (a run-time
// index would move the arrays to local memory).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>

#include "ops_b200_device.h"

namespace {

constexpr int kThreads = 256;  // CTA size

// 1 / x for the eliminations: the Newton-Raphson iteration
// y <- y + y (1 - x y), each step doubling the correct bits, twice from the
// hardware reciprocal approximation (PTX rcp.approx.ftz.f64), with fused
// multiply-adds; zeros, infinities, NaNs and magnitudes whose reciprocal
// could leave the normal range take the IEEE division.  On the GPU the
// result equals 1.0 / x in every bit over 4M random inputs with exponents in
// [-60, 60]; it replaces a division sequence that is several times longer.
__device__ __forceinline__ double rcp64(double x) {
  const double ax = fabs(x);
  if (!(ax > 0x1p-1000 && ax < 0x1p1000)) return 1.0 / x;
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = __fma_rn(-x, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-x, y, 1.0);
  return __fma_rn(y, e, y);
}

// After chunk_reduce (all CL rows; padding rows are b = 1, a = c = d = 0),
// row i of the chunk reads
//   a_i * x_first + x_i + c_i * x_last = d_i        (0 < i < CL-1)
//   a_0 * x_prev  + x_0 + c_0 * x_last = d_0        (row 0)
//   a_{CL-1} * x_0 + x_{CL-1} + c_{CL-1} * x_next = d_{CL-1}   (last row)
// where x_prev / x_next are the end unknowns of the neighbouring chunks.
template <int CL>
__device__ __forceinline__ void chunk_reduce(double *a, const double *b, double *c, double *d) {
  {
    double r = rcp64(b[0]);
    a[0] *= r; c[0] *= r; d[0] *= r;
    r = rcp64(b[1]);
    a[1] *= r; c[1] *= r; d[1] *= r;
  }
  // forward: row i (i >= 2) loses x_{i-1}, gains x_0
#pragma unroll
  for (int i = 2; i < CL; i++) {
    const double r = rcp64(b[i] - a[i] * c[i - 1]);
    d[i] = r * (d[i] - a[i] * d[i - 1]);
    a[i] = -r * a[i] * a[i - 1];
    c[i] = r * c[i];
  }
  // backward: row i (CL-3 >= i >= 1) loses x_{i+1}, gains x_{CL-1}
#pragma unroll
  for (int i = CL - 3; i >= 1; i--) {
    d[i] = d[i] - c[i] * d[i + 1];
    a[i] = a[i] - c[i] * a[i + 1];
    c[i] = -c[i] * c[i + 1];
  }
  // row 0 loses x_1, gains x_{CL-1}
  {
    const double r = rcp64(1.0 - c[0] * a[1]);
    d[0] = r * (d[0] - c[0] * d[1]);
    a[0] = r * a[0];
    c[0] = -r * c[0] * c[1];
  }
}

// PCR over the 64 end unknowns of a line held two per lane (rows 2*lane and
// 2*lane+1) with warp shuffles; returns this lane's two solutions.  Rows are
// a x_{r-s} + x_r + c x_{r+s} = d at each stride s.
__device__ __forceinline__ void warp_pcr(double a0, double c0, double d0, double a1, double c1,
                                         double d1, int lane, double &xf, double &xl) {
  const unsigned full = 0xffffffffu;
  // s = 1: row 2p couples to 2p-1 (lane p-1, last) and 2p+1 (own last);
  // row 2p+1 couples to 2p (own first) and 2p+2 (lane p+1, first)
  {
    const double pa1 = __shfl_up_sync(full, a1, 1), pc1 = __shfl_up_sync(full, c1, 1),
                 pd1 = __shfl_up_sync(full, d1, 1);
    const double na0 = __shfl_down_sync(full, a0, 1), nc0 = __shfl_down_sync(full, c0, 1),
                 nd0 = __shfl_down_sync(full, d0, 1);
    const bool hasl = lane > 0, hasr = lane < 31;
    double k1 = hasl ? a0 : 0.0, k2 = c0;
    double inv = rcp64(1.0 - k1 * (hasl ? pc1 : 0.0) - k2 * a1);
    const double A0 = -k1 * (hasl ? pa1 : 0.0) * inv, C0 = -k2 * c1 * inv,
                 D0 = (d0 - k1 * (hasl ? pd1 : 0.0) - k2 * d1) * inv;
    k1 = a1;
    k2 = hasr ? c1 : 0.0;
    inv = rcp64(1.0 - k1 * c0 - k2 * (hasr ? na0 : 0.0));
    const double A1 = -k1 * a0 * inv, C1 = -k2 * (hasr ? nc0 : 0.0) * inv,
                 D1 = (d1 - k1 * d0 - k2 * (hasr ? nd0 : 0.0)) * inv;
    a0 = A0; c0 = C0; d0 = D0;
    a1 = A1; c1 = C1; d1 = D1;
  }
  // s = 2h rows: both rows of a lane couple to the same slot of lanes p -/+ h
#pragma unroll
  for (int h = 1; h < 32; h <<= 1) {
    const bool hasl = lane >= h, hasr = lane + h < 32;
    const double la0 = __shfl_up_sync(full, a0, h), lc0 = __shfl_up_sync(full, c0, h),
                 ld0 = __shfl_up_sync(full, d0, h);
    const double ra0 = __shfl_down_sync(full, a0, h), rc0 = __shfl_down_sync(full, c0, h),
                 rd0 = __shfl_down_sync(full, d0, h);
    const double la1 = __shfl_up_sync(full, a1, h), lc1 = __shfl_up_sync(full, c1, h),
                 ld1 = __shfl_up_sync(full, d1, h);
    const double ra1 = __shfl_down_sync(full, a1, h), rc1 = __shfl_down_sync(full, c1, h),
                 rd1 = __shfl_down_sync(full, d1, h);
    {
      const double k1 = hasl ? a0 : 0.0, k2 = hasr ? c0 : 0.0;
      const double inv = rcp64(1.0 - k1 * (hasl ? lc0 : 0.0) - k2 * (hasr ? ra0 : 0.0));
      const double nA = -k1 * (hasl ? la0 : 0.0) * inv, nC = -k2 * (hasr ? rc0 : 0.0) * inv;
      d0 = (d0 - k1 * (hasl ? ld0 : 0.0) - k2 * (hasr ? rd0 : 0.0)) * inv;
      a0 = nA; c0 = nC;
    }
    {
      const double k1 = hasl ? a1 : 0.0, k2 = hasr ? c1 : 0.0;
      const double inv = rcp64(1.0 - k1 * (hasl ? lc1 : 0.0) - k2 * (hasr ? ra1 : 0.0));
      const double nA = -k1 * (hasl ? la1 : 0.0) * inv, nC = -k2 * (hasr ? rc1 : 0.0) * inv;
      d1 = (d1 - k1 * (hasl ? ld1 : 0.0) - k2 * (hasr ? rd1 : 0.0)) * inv;
      a1 = nA; c1 = nC;
    }
  }
  xf = d0;
  xl = d1;
}

// Warp-per-line form (n <= 32*CL): lane p holds chunk p; lanes past the last
// chunk carry identity rows.
template <typename T, bool INC, int CL>
__global__ void __launch_bounds__(kThreads) trid_warp_kernel(
    int n, long long nlines, long long stride, int o1n, long long o1s, long long o2s,
    const T *__restrict__ A, const T *__restrict__ B, const T *__restrict__ C,
    T *__restrict__ D, T *__restrict__ U) {
  const int lane = threadIdx.x & 31;
  const long long line = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (line >= nlines) return;  // the whole warp leaves together
  const long long base = (line % o1n) * o1s + (line / o1n) * o2s;
  const int k0 = lane * CL;
  const int len = max(0, min(CL, n - k0));
  double a[CL], b[CL], c[CL], d[CL];
#pragma unroll
  for (int i = 0; i < CL; i++) {
    a[i] = 0.0; b[i] = 1.0; c[i] = 0.0; d[i] = 0.0;
    if (i < len) {
      const long long e = base + (long long)(k0 + i) * stride;
      a[i] = (k0 + i == 0) ? 0.0 : (double)A[e];      // no left neighbour
      b[i] = (double)B[e];
      c[i] = (k0 + i == n - 1) ? 0.0 : (double)C[e];  // no right neighbour
      d[i] = (double)D[e];
    }
  }
  chunk_reduce<CL>(a, b, c, d);
  double xf, xl;
  warp_pcr(a[0], c[0], d[0], a[CL - 1], c[CL - 1], d[CL - 1], lane, xf, xl);
#pragma unroll
  for (int i = 0; i < CL; i++)
    if (i < len) {
      const double x = (i == 0) ? xf : ((i == CL - 1) ? xl : d[i] - a[i] * xf - c[i] * xl);
      const long long e = base + (long long)(k0 + i) * stride;
      if (INC)
        U[e] = (T)((double)U[e] + x);
      else
        D[e] = (T)x;
    }
}

// Eight consecutive elements from p into FP64 registers with the widest
// aligned vector loads (16 bytes when p allows; p's alignment is uniform
// over a warp whose lanes start chunks of 8 elements of one line).
template <typename T>
__device__ __forceinline__ void load8(const T *p, double (&v)[8]) {
  const uintptr_t ad = (uintptr_t)p;
  if (sizeof(T) == 8) {
    const double *q = (const double *)p;
    if ((ad & 15) == 0) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const double2 t = ((const double2 *)q)[i];
        v[2 * i] = t.x; v[2 * i + 1] = t.y;
      }
    } else {
      v[0] = q[0];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const double2 t = ((const double2 *)(q + 1))[i];
        v[2 * i + 1] = t.x; v[2 * i + 2] = t.y;
      }
      v[7] = q[7];
    }
  } else {
    const float *q = (const float *)p;
    if ((ad & 15) == 0) {
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const float4 t = ((const float4 *)q)[i];
        v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
      }
    } else if ((ad & 7) == 0) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const float2 t = ((const float2 *)q)[i];
        v[2 * i] = t.x; v[2 * i + 1] = t.y;
      }
    } else if ((ad & 7) == 4) {  // one element, three 8-byte pairs, one element
      v[0] = q[0];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const float2 t = ((const float2 *)(q + 1))[i];
        v[2 * i + 1] = t.x; v[2 * i + 2] = t.y;
      }
      v[7] = q[7];
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) v[i] = q[i];
    }
  }
}

template <typename T>
__device__ __forceinline__ void store8(T *p, const double (&v)[8]) {
  const uintptr_t ad = (uintptr_t)p;
  if (sizeof(T) == 8) {
    double *q = (double *)p;
    if ((ad & 15) == 0) {
#pragma unroll
      for (int i = 0; i < 4; i++) ((double2 *)q)[i] = make_double2(v[2 * i], v[2 * i + 1]);
    } else {
      q[0] = v[0];
#pragma unroll
      for (int i = 0; i < 3; i++)
        ((double2 *)(q + 1))[i] = make_double2(v[2 * i + 1], v[2 * i + 2]);
      q[7] = v[7];
    }
  } else {
    float *q = (float *)p;
    if ((ad & 15) == 0) {
#pragma unroll
      for (int i = 0; i < 2; i++)
        ((float4 *)q)[i] = make_float4((float)v[4 * i], (float)v[4 * i + 1], (float)v[4 * i + 2],
                                       (float)v[4 * i + 3]);
    } else if ((ad & 7) == 0) {
#pragma unroll
      for (int i = 0; i < 4; i++) ((float2 *)q)[i] = make_float2((float)v[2 * i], (float)v[2 * i + 1]);
    } else if ((ad & 7) == 4) {
      q[0] = (float)v[0];
#pragma unroll
      for (int i = 0; i < 3; i++)
        ((float2 *)(q + 1))[i] = make_float2((float)v[2 * i + 1], (float)v[2 * i + 2]);
      q[7] = (float)v[7];
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) q[i] = (float)v[i];
    }
  }
}

// Unit-stride lines of up to 256 points, one warp per line, 8-point chunks
// per lane: a lane whose chunk lies inside the line loads and stores it
// with 16-byte vector accesses (8-byte ones and single elements where the
// line's alignment leaves no choice), the line's last, partial chunk element
// by element.  32-bit element offsets when every offset of the batch fits
// (IDX32).  Three CTAs per SM.
template <typename T, bool INC, bool IDX32>
__global__ void __launch_bounds__(kThreads, 3) trid_xw_kernel(
    int n, long long nlines, int o1n, long long o1s, long long o2s, const T *__restrict__ A,
    const T *__restrict__ B, const T *__restrict__ C, T *__restrict__ D, T *__restrict__ U) {
  constexpr int CL = 8;
  const int lane = threadIdx.x & 31;
  const long long line = (long long)blockIdx.x * (kThreads >> 5) + (threadIdx.x >> 5);
  if (line >= nlines) return;  // the whole warp leaves together
  const int k0 = lane * CL;
  const long long base =
      IDX32 ? (long long)((int)(line % o1n) * (int)o1s + (int)(line / o1n) * (int)o2s + k0)
            : (line % o1n) * o1s + (line / o1n) * o2s + k0;
  const int len = max(0, min(CL, n - k0));
  double a[CL], b[CL], c[CL], d[CL];
  if (len == CL) {
    load8(A + base, a);
    load8(B + base, b);
    load8(C + base, c);
    load8(D + base, d);
  } else {
#pragma unroll
    for (int i = 0; i < CL; i++) {
      a[i] = 0.0; b[i] = 1.0; c[i] = 0.0; d[i] = 0.0;
      if (i < len) {
        a[i] = (double)A[base + i];
        b[i] = (double)B[base + i];
        c[i] = (double)C[base + i];
        d[i] = (double)D[base + i];
      }
    }
  }
  if (k0 == 0) a[0] = 0.0;  // no left neighbour
#pragma unroll
  for (int i = 0; i < CL; i++)
    if (k0 + i == n - 1) c[i] = 0.0;  // no right neighbour
  chunk_reduce<CL>(a, b, c, d);
  double xf, xl;
  warp_pcr(a[0], c[0], d[0], a[CL - 1], c[CL - 1], d[CL - 1], lane, xf, xl);
  double x[CL];
#pragma unroll
  for (int i = 0; i < CL; i++)
    x[i] = (i == 0) ? xf : ((i == CL - 1) ? xl : d[i] - a[i] * xf - c[i] * xl);
  T *out = (INC ? U : D) + base;
  if (len == CL) {
    if (INC) {
      double u[CL];
      load8(out, u);
#pragma unroll
      for (int i = 0; i < CL; i++) x[i] += u[i];
    }
    store8(out, x);
  } else {
#pragma unroll
    for (int i = 0; i < CL; i++)
      if (i < len) out[i] = INC ? (T)((double)out[i] + x[i]) : (T)x[i];
  }
}

// Staged warp-per-line form: the CTA's W = 8 lines pass through shared memory
// so that loads and stores are contiguous runs.  Unit-stride lines: consecutive
// threads take consecutive points of a line.  Strided lines: consecutive
// threads take the same point of the 8 lines, which are neighbours along the
// fastest other axis, so each row of the tile is one 8-element run.  Each warp
// then solves one line from shared memory with the shuffle PCR; the solution
// leaves through shared memory the same way.
template <typename T, bool INC, int CL>
__global__ void __launch_bounds__(kThreads) trid_staged_kernel(
    int n, long long nlines, long long stride, int unit, int o1n, long long o1s, long long o2s,
    const T *__restrict__ A, const T *__restrict__ B, const T *__restrict__ C,
    T *__restrict__ D, T *__restrict__ U) {
  extern __shared__ double sm[];
  constexpr int W = kThreads / 32;  // lines per CTA
  constexpr int P = 32;             // chunk slots per line (lanes)
  constexpr int pitch = CL + 1;     // padded chunk pitch (spreads the banks)
  constexpr int per_arr = W * P * pitch;
  double *sA = sm, *sB = sA + per_arr, *sC = sB + per_arr, *sD = sC + per_arr;
  const int tid = threadIdx.x;
  const long long line0 = (long long)blockIdx.x * W;
  const int total = W * n;
  for (int idx = tid; idx < total; idx += kThreads) {
    int lq, k;
    if (unit) { lq = idx / n; k = idx - lq * n; }
    else { k = idx / W; lq = idx - k * W; }
    const long long line = line0 + lq;
    if (line >= nlines) continue;
    const long long e = (line % o1n) * o1s + (line / o1n) * o2s + (long long)k * stride;
    const int s = (lq * P + k / CL) * pitch + (k % CL);
    sA[s] = (double)A[e];
    sB[s] = (double)B[e];
    sC[s] = (double)C[e];
    sD[s] = (double)D[e];
  }
  __syncthreads();
  const int w = tid >> 5, lane = tid & 31;
  const long long line = line0 + w;
  const int k0 = lane * CL;
  const int len = line < nlines ? max(0, min(CL, n - k0)) : 0;
  const int cs = (w * P + lane) * pitch;
  double a[CL], b[CL], c[CL], d[CL];
#pragma unroll
  for (int i = 0; i < CL; i++) {
    a[i] = 0.0; b[i] = 1.0; c[i] = 0.0; d[i] = 0.0;
    if (i < len) {
      a[i] = (k0 + i == 0) ? 0.0 : sA[cs + i];
      b[i] = sB[cs + i];
      c[i] = (k0 + i == n - 1) ? 0.0 : sC[cs + i];
      d[i] = sD[cs + i];
    }
  }
  chunk_reduce<CL>(a, b, c, d);
  double xf, xl;
  warp_pcr(a[0], c[0], d[0], a[CL - 1], c[CL - 1], d[CL - 1], lane, xf, xl);
#pragma unroll
  for (int i = 0; i < CL; i++)
    if (i < len) sD[cs + i] = (i == 0) ? xf : ((i == CL - 1) ? xl : d[i] - a[i] * xf - c[i] * xl);
  __syncthreads();
  for (int idx = tid; idx < total; idx += kThreads) {
    int lq, k;
    if (unit) { lq = idx / n; k = idx - lq * n; }
    else { k = idx / W; lq = idx - k * W; }
    const long long ln = line0 + lq;
    if (ln >= nlines) continue;
    const long long e = (ln % o1n) * o1s + (ln / o1n) * o2s + (long long)k * stride;
    const double x = sD[(lq * P + k / CL) * pitch + (k % CL)];
    if (INC)
      U[e] = (T)((double)U[e] + x);
    else
      D[e] = (T)x;
  }
}

// LPB lines per CTA, P chunks per line spread over the CTA, PCR over the 2P
// end unknowns in shared memory.  Chunk-major mapping (LM false: the P
// chunks of a line on consecutive threads) for long lines (n > 32*16);
// line-major mapping (LM true: consecutive threads on the same chunk of
// neighbouring lines) for strided lines, whose neighbours along the fastest
// other axis are contiguous in memory, so that every load and store of a
// warp is two runs of LPB elements and no scratch is needed.  The
// arithmetic of a line does not depend on the mapping.
template <typename T, bool INC, int CL, bool LM>
__global__ void __launch_bounds__(kThreads) trid_cta_kernel(
    int n, int P, int LPB, long long nlines, long long stride, int o1n, long long o1s,
    long long o2s, const T *__restrict__ A, const T *__restrict__ B, const T *__restrict__ C,
    T *__restrict__ D, T *__restrict__ U) {
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  const int p = LM ? tid / LPB : tid % P, l = LM ? tid % LPB : tid / P;
  const long long line = (long long)blockIdx.x * LPB + l;
  const bool active = line < nlines && l < LPB;
  const int m = 2 * P;
  // a line's 3 x 2P values; the odd pitch spreads neighbouring lines over
  // the shared-memory banks
  double *ra = sm + (size_t)(l < LPB ? l : 0) * (m * 3 + 1);
  double *rc = ra + m;
  double *rd = rc + m;
  long long base = 0;
  if (active) base = (line % o1n) * o1s + (line / o1n) * o2s;
  const int k0 = p * CL;
  const int len = active ? max(0, min(CL, n - k0)) : 0;
  double a[CL], b[CL], c[CL], d[CL];
#pragma unroll
  for (int i = 0; i < CL; i++) {
    a[i] = 0.0; b[i] = 1.0; c[i] = 0.0; d[i] = 0.0;
    if (i < len) {
      const long long e = base + (long long)(k0 + i) * stride;
      a[i] = (k0 + i == 0) ? 0.0 : (double)A[e];
      b[i] = (double)B[e];
      c[i] = (k0 + i == n - 1) ? 0.0 : (double)C[e];
      d[i] = (double)D[e];
    }
  }
  chunk_reduce<CL>(a, b, c, d);
  if (l < LPB) {
    ra[2 * p] = a[0]; rc[2 * p] = c[0]; rd[2 * p] = d[0];
    ra[2 * p + 1] = a[CL - 1]; rc[2 * p + 1] = c[CL - 1]; rd[2 * p + 1] = d[CL - 1];
  }
  __syncthreads();
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
      const double inv = rcp64(1.0 - k1l * c1 - k2r * a2);
      na[q] = -k1l * a1 * inv;
      nc[q] = -k2r * c2 * inv;
      nd[q] = (dr - k1l * d1 - k2r * d2) * inv;
    }
    __syncthreads();
    if (l < LPB) {
      ra[2 * p] = na[0]; rc[2 * p] = nc[0]; rd[2 * p] = nd[0];
      ra[2 * p + 1] = na[1]; rc[2 * p + 1] = nc[1]; rd[2 * p + 1] = nd[1];
    }
    __syncthreads();
  }
  if (len <= 0) return;
  const double xf = rd[2 * p], xl = rd[2 * p + 1];
#pragma unroll
  for (int i = 0; i < CL; i++)
    if (i < len) {
      const double x = (i == 0) ? xf : ((i == CL - 1) ? xl : d[i] - a[i] * xf - c[i] * xl);
      const long long e = base + (long long)(k0 + i) * stride;
      if (INC)
        U[e] = (T)((double)U[e] + x);
      else
        D[e] = (T)x;
    }
}

// Strided lines of up to 256 points (y, z): 8 lines x 32 chunks of 8 points
// per CTA in the line-major mapping of trid_cta_kernel (consecutive threads
// on the same chunk of neighbouring lines, whose elements are contiguous:
// every load and store of a warp is runs of 8 elements), but the PCR over
// each line's 64 chunk-end unknowns runs in one warp with shuffles (warp w
// solves line w): the end rows cross shared memory once each way, with two
// CTA barriers instead of two per PCR level.  Three CTAs per SM; 32-bit
// element offsets when every offset of the batch fits (IDX32).
template <typename T, bool INC, bool IDX32>
__global__ void __launch_bounds__(kThreads, 3) trid_lmw_kernel(
    int n, long long nlines, long long stride, int o1n, long long o1s, long long o2s,
    const T *__restrict__ A, const T *__restrict__ B, const T *__restrict__ C,
    T *__restrict__ D, T *__restrict__ U) {
  constexpr int CL = 8, P = 32, LPB = kThreads / P, M = 2 * P, pitch = 3 * M + 1;
  static_assert(LPB == kThreads / 32, "one warp per line for the PCR");
  __shared__ double sm[LPB * pitch];
  const int tid = threadIdx.x;
  const int p = tid / LPB, l = tid % LPB;
  const long long line = (long long)blockIdx.x * LPB + l;
  const bool active = line < nlines;
  const int k0 = p * CL;
  long long base = 0;
  if (active)
    base = IDX32 ? (long long)((int)(line % o1n) * (int)o1s + (int)(line / o1n) * (int)o2s +
                               k0 * (int)stride)
                 : (line % o1n) * o1s + (line / o1n) * o2s + (long long)k0 * stride;
  const int len = active ? max(0, min(CL, n - k0)) : 0;
  double a[CL], b[CL], c[CL], d[CL];
#pragma unroll
  for (int i = 0; i < CL; i++) {
    a[i] = 0.0; b[i] = 1.0; c[i] = 0.0; d[i] = 0.0;
    if (i < len) {
      const long long e = IDX32 ? (long long)((int)base + i * (int)stride) : base + i * stride;
      a[i] = (k0 + i == 0) ? 0.0 : (double)A[e];
      b[i] = (double)B[e];
      c[i] = (k0 + i == n - 1) ? 0.0 : (double)C[e];
      d[i] = (double)D[e];
    }
  }
  chunk_reduce<CL>(a, b, c, d);
  double *ra = sm + l * pitch, *rc = ra + M, *rd = rc + M;
  ra[2 * p] = a[0]; rc[2 * p] = c[0]; rd[2 * p] = d[0];
  ra[2 * p + 1] = a[CL - 1]; rc[2 * p + 1] = c[CL - 1]; rd[2 * p + 1] = d[CL - 1];
  __syncthreads();
  {
    const int w = tid >> 5, lane = tid & 31;
    double *wa = sm + w * pitch, *wc = wa + M, *wd = wc + M;
    double xf, xl;
    warp_pcr(wa[2 * lane], wc[2 * lane], wd[2 * lane], wa[2 * lane + 1], wc[2 * lane + 1],
             wd[2 * lane + 1], lane, xf, xl);
    wd[2 * lane] = xf;  // this lane's own rows: no other lane reads them
    wd[2 * lane + 1] = xl;
  }
  __syncthreads();
  if (len <= 0) return;
  const double xf = rd[2 * p], xl = rd[2 * p + 1];
#pragma unroll
  for (int i = 0; i < CL; i++)
    if (i < len) {
      const double x = (i == 0) ? xf : ((i == CL - 1) ? xl : d[i] - a[i] * xf - c[i] * xl);
      const long long e = IDX32 ? (long long)((int)base + i * (int)stride) : base + i * stride;
      if (INC)
        U[e] = (T)((double)U[e] + x);
      else
        D[e] = (T)x;
    }
}

// ---------------------------------------------------------------------------
// Pipelined persistent form of trid_cta_kernel (8-point chunks, P <= 32
// chunks per line, LPB = 256 / P lines per work item).  Each CTA walks the
// work items (groups of LPB lines) with a stride of the grid; while it
// eliminates, reduces and substitutes one item, the coefficients of its next
// item are already on their way into shared memory through asynchronous
// copies (cp.async, 4- or 8-byte elements: no alignment demand beyond the
// element's own).  Every thread copies exactly the elements it will consume
// itself, so the staging needs no CTA barrier: cp.async.wait_all makes the
// thread's own copies visible to it.  For the _Inc form u comes through a
// second, double-buffered stage so that the next item's u can land while
// this item's u is still being added to.  Two CTAs per SM keep about 128 KB
// of loads in flight per SM, so the HBM stays busy through the FP64
// divisions of the elimination and the barriers of the PCR.
//
// Mapping: LM (strided lines) puts consecutive threads on the same chunk of
// neighbouring lines (contiguous along x: every copy of a warp is LPB-element
// runs); !LM (unit-stride lines) puts the P chunks of a line on consecutive
// threads.  The arithmetic per line is that of trid_cta_kernel.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_el(void *dst, const void *src, int bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

constexpr int kPipeCL = 8;

template <typename T, bool INC, bool LM>
__global__ void __launch_bounds__(kThreads, 2) trid_pipe_kernel(
    int n, int P, int LPB, long long nitems, long long nlines, long long stride, int o1n,
    long long o1s, long long o2s, const T *__restrict__ A, const T *__restrict__ B,
    const T *__restrict__ C, T *__restrict__ D, T *__restrict__ U) {
  constexpr int CL = kPipeCL;
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  const int p = LM ? tid / LPB : tid % P, l = LM ? tid % LPB : tid / P;
  const bool mine = l < LPB && p < P;  // threads past LPB * P stay idle
  const int m = 2 * P;
  double *ra = sm + (size_t)(l < LPB ? l : 0) * (m * 3 + 1);
  double *rc = ra + m;
  double *rd = rc + m;
  // stage: [array * CL + i][thread] (consecutive threads, consecutive words)
  T *stage = (T *)(sm + (size_t)LPB * (m * 3 + 1));
  T *ustage = stage + (size_t)4 * CL * kThreads;  // [buffer][i][thread], _Inc only
  const int k0 = p * CL;

  auto line_base = [&](long long item, long long &base) -> int {
    const long long line = item * LPB + l;
    if (!mine || line >= nlines) return 0;
    base = (line % o1n) * o1s + (line / o1n) * o2s;
    return max(0, min(CL, n - k0));
  };
  auto issue = [&](long long item, int ub) {
    long long base = 0;
    const int len = line_base(item, base);
#pragma unroll
    for (int i = 0; i < CL; i++)
      if (i < len) {
        const long long e = base + (long long)(k0 + i) * stride;
        cp_async_el(stage + (size_t)(0 * CL + i) * kThreads + tid, A + e, sizeof(T));
        cp_async_el(stage + (size_t)(1 * CL + i) * kThreads + tid, B + e, sizeof(T));
        cp_async_el(stage + (size_t)(2 * CL + i) * kThreads + tid, C + e, sizeof(T));
        cp_async_el(stage + (size_t)(3 * CL + i) * kThreads + tid, D + e, sizeof(T));
        if (INC)
          cp_async_el(ustage + (size_t)(ub * CL + i) * kThreads + tid, U + e, sizeof(T));
      }
    cp_async_commit();
  };

  long long item = blockIdx.x;
  int ub = 0;
  if (item < nitems) issue(item, ub);
  for (; item < nitems; item += gridDim.x, ub ^= 1) {
    cp_async_wait_all();
    long long base = 0;
    const int len = line_base(item, base);
    double a[CL], b[CL], c[CL], d[CL];
#pragma unroll
    for (int i = 0; i < CL; i++) {
      a[i] = 0.0; b[i] = 1.0; c[i] = 0.0; d[i] = 0.0;
      if (i < len) {
        a[i] = (k0 + i == 0) ? 0.0 : (double)stage[(size_t)(0 * CL + i) * kThreads + tid];
        b[i] = (double)stage[(size_t)(1 * CL + i) * kThreads + tid];
        c[i] = (k0 + i == n - 1) ? 0.0 : (double)stage[(size_t)(2 * CL + i) * kThreads + tid];
        d[i] = (double)stage[(size_t)(3 * CL + i) * kThreads + tid];
      }
    }
    // the next item's copies go into the slots just read (this thread's own)
    if (item + gridDim.x < nitems) issue(item + gridDim.x, ub ^ 1);
    chunk_reduce<CL>(a, b, c, d);
    if (mine) {
      ra[2 * p] = a[0]; rc[2 * p] = c[0]; rd[2 * p] = d[0];
      ra[2 * p + 1] = a[CL - 1]; rc[2 * p + 1] = c[CL - 1]; rd[2 * p + 1] = d[CL - 1];
    }
    __syncthreads();
    for (int s = 1; s < m; s <<= 1) {
      double na[2], nc[2], nd[2];
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int r = 2 * (mine ? p : 0) + q;
        const double ar = ra[r], cr = rc[r], dr = rd[r];
        double a1 = 0.0, c1 = 0.0, d1 = 0.0, a2 = 0.0, c2 = 0.0, d2 = 0.0;
        const bool hl = r - s >= 0, hr = r + s < m;
        if (hl) { a1 = ra[r - s]; c1 = rc[r - s]; d1 = rd[r - s]; }
        if (hr) { a2 = ra[r + s]; c2 = rc[r + s]; d2 = rd[r + s]; }
        const double k1l = hl ? ar : 0.0, k2r = hr ? cr : 0.0;
        const double inv = rcp64(1.0 - k1l * c1 - k2r * a2);
        na[q] = -k1l * a1 * inv;
        nc[q] = -k2r * c2 * inv;
        nd[q] = (dr - k1l * d1 - k2r * d2) * inv;
      }
      __syncthreads();
      if (mine) {
        ra[2 * p] = na[0]; rc[2 * p] = nc[0]; rd[2 * p] = nd[0];
        ra[2 * p + 1] = na[1]; rc[2 * p + 1] = nc[1]; rd[2 * p + 1] = nd[1];
      }
      __syncthreads();
    }
    if (len > 0) {
      const double xf = rd[2 * p], xl = rd[2 * p + 1];
#pragma unroll
      for (int i = 0; i < CL; i++)
        if (i < len) {
          const double x = (i == 0) ? xf : ((i == CL - 1) ? xl : d[i] - a[i] * xf - c[i] * xl);
          const long long e = base + (long long)(k0 + i) * stride;
          if (INC)
            U[e] = (T)((double)ustage[(size_t)(ub * CL + i) * kThreads + tid] + x);
          else
            D[e] = (T)x;
        }
    }
    __syncthreads();  // the next item's end rows overwrite ra / rc / rd
  }
  cp_async_wait_all();
}

// Strided lines (y, z): one thread per line, neighbouring threads on
// neighbouring lines along the fastest other axis, so every load and store
// of a warp is one contiguous run.  The Thomas algorithm in FP64 with the
// operation order of the sequential restatement (c'_i = c_i m_i,
// d'_i = (d_i - a_i d'_{i-1}) m_i, m_i = 1 / (b_i - a_i c'_{i-1}), then
// x_i = d'_i - c'_i x_{i+1}), every product and difference rounded on its own
// (no contraction), so the solution equals the oracle's bit for bit.  The
// forward sweep keeps c' and d' in a device scratch array laid out
// [point][line] (coalesced too); the backward sweep reads them back, mostly
// from L2.  Traffic: the algorithmic 4 reads + 1 write per point, plus the
// scratch's 2 writes + 2 reads where it leaves L2.
template <typename T, bool INC>
__global__ void __launch_bounds__(128) trid_thomas_kernel(
    int n, long long nlines, long long stride, int o1n, long long o1s, long long o2s,
    const T *__restrict__ A, const T *__restrict__ B, const T *__restrict__ C,
    T *__restrict__ D, T *__restrict__ U, double *__restrict__ cpd) {
  for (long long line = (long long)blockIdx.x * blockDim.x + threadIdx.x; line < nlines;
       line += (long long)gridDim.x * blockDim.x) {
    const long long base = (line % o1n) * o1s + (line / o1n) * o2s;
    double *cp = cpd + line, *dp = cpd + (long long)n * nlines + line;
    double m = __ddiv_rn(1.0, (double)B[base]);
    double cprev = __dmul_rn((double)C[base], m);
    double dprev = __dmul_rn((double)D[base], m);
    cp[0] = cprev;
    dp[0] = dprev;
#pragma unroll 4
    for (int k = 1; k < n; k++) {
      const long long e = base + (long long)k * stride;
      const double a = (double)A[e], b = (double)B[e], c = (double)C[e], d = (double)D[e];
      m = __ddiv_rn(1.0, __dsub_rn(b, __dmul_rn(a, cprev)));
      cprev = __dmul_rn(c, m);
      dprev = __dmul_rn(__dsub_rn(d, __dmul_rn(a, dprev)), m);
      cp[(long long)k * nlines] = cprev;
      dp[(long long)k * nlines] = dprev;
    }
    double x = dprev;
    {
      const long long e = base + (long long)(n - 1) * stride;
      if (INC)
        U[e] = (T)__dadd_rn((double)U[e], x);
      else
        D[e] = (T)x;
    }
#pragma unroll 4
    for (int k = n - 2; k >= 0; k--) {
      x = __dsub_rn(dp[(long long)k * nlines], __dmul_rn(cp[(long long)k * nlines], x));
      const long long e = base + (long long)k * stride;
      if (INC)
        U[e] = (T)__dadd_rn((double)U[e], x);
      else
        D[e] = (T)x;
    }
  }
}

struct Lines {
  int n, unit, o1n;
  long long nlines, stride, o1s, o2s;
};

// scratch for the Thomas kernel's c' and d' (grown on demand, kept)
double *g_cpd = nullptr;
size_t g_cpd_cap = 0;

template <typename T>
int launch_thomas(const Lines &g, const void *a, const void *b, const void *c, void *d,
                  void *u) {
  const size_t need = (size_t)2 * g.n * g.nlines * sizeof(double);
  cudaStream_t st = (cudaStream_t)ob2_dev_stream();
  if (need > g_cpd_cap) {
    if (g_cpd) {
      cudaStreamSynchronize(st);
      cudaFree(g_cpd);
      g_cpd = nullptr;
      g_cpd_cap = 0;
    }
    cudaError_t e = cudaMalloc(&g_cpd, need);
    if (e != cudaSuccess) return (int)e;
    g_cpd_cap = need;
  }
  // a persistent grid: every line in flight at once would keep 16 bytes
  // per point of scratch live, far beyond L2 for large batches
  int sms = 148;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  static int mult = -1;
  if (mult < 0) {
    const char *env = getenv("OB2_TRID_THOMAS_CTAS");
    mult = env ? atoi(env) : 4;
    if (mult < 1) mult = 1;
  }
  long long grid = std::min((g.nlines + 127) / 128, (long long)sms * mult);
  if (u)
    trid_thomas_kernel<T, true><<<(unsigned)grid, 128, 0, st>>>(
        g.n, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, (const T *)a, (const T *)b, (const T *)c,
        (T *)d, (T *)u, g_cpd);
  else
    trid_thomas_kernel<T, false><<<(unsigned)grid, 128, 0, st>>>(
        g.n, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, (const T *)a, (const T *)b, (const T *)c,
        (T *)d, (T *)nullptr, g_cpd);
  return (int)cudaGetLastError();
}

template <typename T, int CL>
int launch_warp(const Lines &g, const void *a, const void *b, const void *c, void *d, void *u) {
  const int warps = kThreads / 32;
  const long long grid = (g.nlines + warps - 1) / warps;
  if (grid > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)ob2_dev_stream();
  if (u)
    trid_warp_kernel<T, true, CL><<<(unsigned)grid, kThreads, 0, st>>>(
        g.n, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, (const T *)a, (const T *)b, (const T *)c,
        (T *)d, (T *)u);
  else
    trid_warp_kernel<T, false, CL><<<(unsigned)grid, kThreads, 0, st>>>(
        g.n, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, (const T *)a, (const T *)b, (const T *)c,
        (T *)d, (T *)nullptr);
  return (int)cudaGetLastError();
}

// 1: every element offset of the batch fits 32-bit arithmetic
bool offsets_fit32(const Lines &g) {
  if (g.o1s < 0 || g.o2s < 0 || g.stride < 0) return false;
  const long long d2 = (g.nlines + g.o1n - 1) / g.o1n;
  const long long mx =
      (long long)(g.o1n - 1) * g.o1s + (d2 - 1) * g.o2s + (long long)(g.n - 1) * g.stride;
  return mx < 0x7fffffffLL;
}

template <typename T>
int launch_xw(const Lines &g, const void *a, const void *b, const void *c, void *d, void *u) {
  const long long grid = (g.nlines + (kThreads / 32) - 1) / (kThreads / 32);
  if (grid > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)ob2_dev_stream();
  const bool i32 = offsets_fit32(g);
  const T *A = (const T *)a, *B = (const T *)b, *C = (const T *)c;
  T *D = (T *)d, *U = (T *)u;
  if (u) {
    if (i32)
      trid_xw_kernel<T, true, true><<<(unsigned)grid, kThreads, 0, st>>>(g.n, g.nlines, g.o1n, g.o1s, g.o2s, A, B, C, D, U);
    else
      trid_xw_kernel<T, true, false><<<(unsigned)grid, kThreads, 0, st>>>(g.n, g.nlines, g.o1n, g.o1s, g.o2s, A, B, C, D, U);
  } else {
    if (i32)
      trid_xw_kernel<T, false, true><<<(unsigned)grid, kThreads, 0, st>>>(g.n, g.nlines, g.o1n, g.o1s, g.o2s, A, B, C, D, nullptr);
    else
      trid_xw_kernel<T, false, false><<<(unsigned)grid, kThreads, 0, st>>>(g.n, g.nlines, g.o1n, g.o1s, g.o2s, A, B, C, D, nullptr);
  }
  return (int)cudaGetLastError();
}

template <typename T>
int launch_lmw(const Lines &g, const void *a, const void *b, const void *c, void *d, void *u) {
  constexpr int LPB = kThreads / 32;
  const long long grid = (g.nlines + LPB - 1) / LPB;
  if (grid > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)ob2_dev_stream();
  const bool i32 = offsets_fit32(g);
  const T *A = (const T *)a, *B = (const T *)b, *C = (const T *)c;
  T *D = (T *)d, *U = (T *)u;
  if (u) {
    if (i32)
      trid_lmw_kernel<T, true, true><<<(unsigned)grid, kThreads, 0, st>>>(g.n, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, A, B, C, D, U);
    else
      trid_lmw_kernel<T, true, false><<<(unsigned)grid, kThreads, 0, st>>>(g.n, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, A, B, C, D, U);
  } else {
    if (i32)
      trid_lmw_kernel<T, false, true><<<(unsigned)grid, kThreads, 0, st>>>(g.n, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, A, B, C, D, nullptr);
    else
      trid_lmw_kernel<T, false, false><<<(unsigned)grid, kThreads, 0, st>>>(g.n, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, A, B, C, D, nullptr);
  }
  return (int)cudaGetLastError();
}

template <typename T, int CL>
int launch_staged(const Lines &g, const void *a, const void *b, const void *c, void *d, void *u) {
  const int W = kThreads / 32;
  const long long grid = (g.nlines + W - 1) / W;
  if (grid > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
  const size_t shmem = (size_t)4 * W * 32 * (CL + 1) * sizeof(double);
  cudaStream_t st = (cudaStream_t)ob2_dev_stream();
  if (u) {
    cudaFuncSetAttribute(trid_staged_kernel<T, true, CL>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
    trid_staged_kernel<T, true, CL><<<(unsigned)grid, kThreads, shmem, st>>>(
        g.n, g.nlines, g.stride, g.unit, g.o1n, g.o1s, g.o2s, (const T *)a, (const T *)b,
        (const T *)c, (T *)d, (T *)u);
  } else {
    cudaFuncSetAttribute(trid_staged_kernel<T, false, CL>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
    trid_staged_kernel<T, false, CL><<<(unsigned)grid, kThreads, shmem, st>>>(
        g.n, g.nlines, g.stride, g.unit, g.o1n, g.o1s, g.o2s, (const T *)a, (const T *)b,
        (const T *)c, (T *)d, (T *)nullptr);
  }
  return (int)cudaGetLastError();
}

template <typename T, int CL, bool LM>
int launch_cta(const Lines &g, const void *a, const void *b, const void *c, void *d, void *u) {
  const int P = (g.n + CL - 1) / CL;
  if (P > kThreads) return (int)cudaErrorInvalidValue;
  const int LPB = kThreads / P;
  const int threads = LPB * P;
  const size_t shmem = (size_t)LPB * (2 * P * 3 + 1) * sizeof(double);
  const long long grid = (g.nlines + LPB - 1) / LPB;
  if (grid > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)ob2_dev_stream();
  if (u)
    trid_cta_kernel<T, true, CL, LM><<<(unsigned)grid, threads, shmem, st>>>(
        g.n, P, LPB, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, (const T *)a, (const T *)b,
        (const T *)c, (T *)d, (T *)u);
  else
    trid_cta_kernel<T, false, CL, LM><<<(unsigned)grid, threads, shmem, st>>>(
        g.n, P, LPB, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, (const T *)a, (const T *)b,
        (const T *)c, (T *)d, (T *)nullptr);
  return (int)cudaGetLastError();
}

template <typename T, bool LM>
int launch_pipe(const Lines &g, const void *a, const void *b, const void *c, void *d, void *u) {
  constexpr int CL = kPipeCL;
  const int P = (g.n + CL - 1) / CL;
  if (P > 32) return (int)cudaErrorInvalidValue;
  const int LPB = kThreads / P;
  const long long nitems = (g.nlines + LPB - 1) / LPB;
  const size_t pcr = (size_t)LPB * (2 * P * 3 + 1) * sizeof(double);
  const size_t stage = (size_t)(4 + (u ? 2 : 0)) * CL * kThreads * sizeof(T);
  const size_t shmem = pcr + stage;
  cudaStream_t st = (cudaStream_t)ob2_dev_stream();
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long grid = std::min(nitems, 2LL * sms);
  if (u) {
    cudaFuncSetAttribute(trid_pipe_kernel<T, true, LM>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
    trid_pipe_kernel<T, true, LM><<<(unsigned)grid, kThreads, shmem, st>>>(
        g.n, P, LPB, nitems, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, (const T *)a,
        (const T *)b, (const T *)c, (T *)d, (T *)u);
  } else {
    cudaFuncSetAttribute(trid_pipe_kernel<T, false, LM>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
    trid_pipe_kernel<T, false, LM><<<(unsigned)grid, kThreads, shmem, st>>>(
        g.n, P, LPB, nitems, g.nlines, g.stride, g.o1n, g.o1s, g.o2s, (const T *)a,
        (const T *)b, (const T *)c, (T *)d, (T *)nullptr);
  }
  return (int)cudaGetLastError();
}

// OB2_TRID_PIPE: 0 (default) none, 1 strided lines of 2 to 256 points of
// 4-byte values through the pipelined persistent kernel, 3 strided lines of
// any value size, 2 unit-stride lines too.  Measured on the 256^3 ADI lines
// (CUDA events): FP32 y / z 225 / 307 us pipelined against 173 / 279 us
// for trid_lmw_kernel; FP64 step 1.511-1.512 ms pipelined against
// 1.410-1.429 ms with the line-major CTA kernel; unit-stride x lines 451 us
// against 318 us for the warp-per-line kernel (the chunk-per-lane copies
// are elements 64 bytes apart).  ncu (ADI 256^3, y solve): 24 % of the warp
// slots active (108-118 registers, 108 KB of shared memory: two CTAs per
// SM), the stalls split between shared-memory and CTA barriers of the PCR
// and the FP64 divisions: latency-bound, not memory-bound.
template <typename T>
bool use_pipe(const Lines &g) {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("OB2_TRID_PIPE");
    v = e ? atoi(e) : 0;
  }
  if (g.n < 2 || g.n > 32 * kPipeCL) return false;
  if (g.unit) return v == 2;
  return v >= 2 || (v == 1 && sizeof(T) == 4);
}

// OB2_TRID_STRIDED: how strided lines are solved.  Measured on the 256^3
// FP64 y / z solves (CUDA events): 4 the line-major kernel with the warp
// PCR (trid_lmw_kernel) 147 / 263 us in a stand-alone harness on the ADI
// driver's layout (258-element rows) where mode 3 took 238 / 382 us, and
// 173 / 279 us for FP32 storage (16 lines per CTA instead of 8, for
// 64-byte runs, one CTA per SM: y / z 194 / 309 us FP64, 259 / 375 us FP32
// in the application, against 150 / 267 and 179 / 286); 3 the line-major CTA
// kernel with 8-point chunks and the PCR in shared memory (8 lines x 32
// chunks per CTA, 64-byte runs, 2 CTAs per SM): 226 / 364 us; 2 the same
// with 16-point chunks (16 lines, 128-byte runs, 150 registers, 1 CTA per
// SM): 213 / 438 us; 1 the staged warp-per-line kernel: 300 / 408 us; 0 the
// Thomas kernel (bit-identical to the sequential restatement): 371 / 382 us.
// With FP32 storage the line-major runs shrink to 32 bytes and the staged
// kernel is faster (290 / 400 us against 305 / 428 us).  Default (-1): 4 for
// lines of up to 256 points, 1 otherwise.
int strided_mode() {
  static int v = -2;
  if (v == -2) {
    const char *e = getenv("OB2_TRID_STRIDED");
    v = e ? atoi(e) : -1;
  }
  return v;
}
bool use_thomas(int unit) { return !unit && strided_mode() == 0; }

// the line-major kernel's chunk length for strided lines (-8: the warp-PCR
// form), 0: not used
template <typename T>
int line_major_chunk(const Lines &g) {
  if (g.unit) return 0;
  const int m = strided_mode();
  if (m == 2 && g.n <= 32 * 16) return 16;
  if (m == 3 && g.n <= 32 * 8) return 8;
  if ((m == 4 || m == -1) && g.n <= 32 * 8) return -8;
  return 0;
}

// OB2_TRID_UNIT: 1 (default) unit-stride lines of up to 256 points through
// trid_xw_kernel (vector accesses, 32-bit offsets, three CTAs per SM; the
// 256^3 x solve in a stand-alone harness: 140 / 161 us FP64 on 16-byte
// aligned / 258-element rows against 233 / 240 us for trid_warp_kernel,
// 93 / 142 us FP32 against 166 / 168 us), 0 the kernels below.
int unit_mode() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("OB2_TRID_UNIT");
    v = e ? atoi(e) : 1;
  }
  return v;
}

// OB2_TRID_STAGED: 0 never, 1 always, 2 strided lines only (default)
bool use_staged(int unit) {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("OB2_TRID_STAGED");
    v = e ? atoi(e) : 2;
  }
  return v == 1 || (v == 2 && !unit);
}

template <typename T>
int launch(int ndim, int solvedim, const int *dims, const long long *strides, const void *a,
           const void *b, const void *c, void *d, void *u) {
  Lines g;
  g.n = dims[solvedim];
  int o1 = -1, o2 = -1;
  for (int i = 0; i < 3; i++) {
    if (i == solvedim) continue;
    if (o1 < 0) o1 = i; else o2 = i;
  }
  const int d1 = o1 < ndim ? dims[o1] : 1;
  const int d2 = o2 < ndim ? dims[o2] : 1;
  g.o1n = d1;
  g.o1s = o1 < ndim ? strides[o1] : 0;
  g.o2s = o2 < ndim ? strides[o2] : 0;
  g.nlines = (long long)d1 * d2;
  g.stride = strides[solvedim];
  g.unit = g.stride == 1 ? 1 : 0;
  if (g.n <= 0 || g.nlines <= 0) return 0;
  if (use_thomas(g.unit)) return launch_thomas<T>(g, a, b, c, d, u);
  if (g.unit && g.n <= 32 * 8 && unit_mode() == 1) return launch_xw<T>(g, a, b, c, d, u);
  if (use_pipe<T>(g)) {
    if (g.unit) return launch_pipe<T, false>(g, a, b, c, d, u);
    return launch_pipe<T, true>(g, a, b, c, d, u);
  }
  switch (line_major_chunk<T>(g)) {
    case -8:
      return launch_lmw<T>(g, a, b, c, d, u);
    case 8:
      return launch_cta<T, 8, true>(g, a, b, c, d, u);
    case 16:
      return launch_cta<T, 16, true>(g, a, b, c, d, u);
    default:
      break;
  }
  if (g.n <= 32 * 16) {
    const bool st = use_staged(g.unit);
    if (g.n <= 32 * 4)
      return st ? launch_staged<T, 4>(g, a, b, c, d, u) : launch_warp<T, 4>(g, a, b, c, d, u);
    if (g.n <= 32 * 8)
      return st ? launch_staged<T, 8>(g, a, b, c, d, u) : launch_warp<T, 8>(g, a, b, c, d, u);
    return st ? launch_staged<T, 16>(g, a, b, c, d, u) : launch_warp<T, 16>(g, a, b, c, d, u);
  }
  return launch_cta<T, 16, false>(g, a, b, c, d, u);
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
