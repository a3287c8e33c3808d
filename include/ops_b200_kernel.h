/*
 * ops_b200_kernel.h -- device-side helpers for translator-generated par_loop
 * kernels (included only by generated .cu files).
 *
 * Reductions replace the reference's shared-memory tree reduction
 * (ops/c/include/ops_cuda_reduction.h:49-165) and its host-side finish over
 * per-block partials (templates/cpp/cuda/loop_host.cpp.j2:720-744):
 *   warp shuffle -> one value per warp in shared memory -> one partial per
 *   CTA in global scratch -> the last CTA to finish (atomic ticket) combines
 *   all partials in a fixed order and folds them into the handle's device
 *   accumulator.  The order is fixed for a given launch shape, so results are
 *   deterministic run to run; nothing is copied back until
 *   ops_reduction_result.
 */
#ifndef OPS_B200_KERNEL_H
#define OPS_B200_KERNEL_H

#include <cuda_runtime.h>
#include <float.h>
#include <limits.h>

#include "ops_lib_core.h"
#include "ops_b200_loop.h"

namespace ob2 {

template <typename T> struct lim;
template <> struct lim<double> {
  static __device__ __forceinline__ double lo() { return -DBL_MAX; }
  static __device__ __forceinline__ double hi() { return DBL_MAX; }
};
template <> struct lim<float> {
  static __device__ __forceinline__ float lo() { return -FLT_MAX; }
  static __device__ __forceinline__ float hi() { return FLT_MAX; }
};
template <> struct lim<int> {
  static __device__ __forceinline__ int lo() { return INT_MIN; }
  static __device__ __forceinline__ int hi() { return INT_MAX; }
};
template <> struct lim<long long> {
  static __device__ __forceinline__ long long lo() { return LLONG_MIN; }
  static __device__ __forceinline__ long long hi() { return LLONG_MAX; }
};

/* identity, combination, lane exchange and volatile read of each reduction
 * (ops_lib_core.cpp:840-965); complex values (ops_lib_core.cpp:935-952)
 * have their own rules below */
template <typename T, int OP> struct red {
  static __device__ __forceinline__ T identity() {
    if (OP == OPS_MIN) return lim<T>::hi();
    if (OP == OPS_MAX) return lim<T>::lo();
    return T(0);
  }
  static __device__ __forceinline__ T combine(T a, T b) {
    if (OP == OPS_MIN) return b < a ? b : a;
    if (OP == OPS_MAX) return b > a ? b : a;
    return a + b;
  }
  static __device__ __forceinline__ T shfl_xor(T v, int o) {
    return __shfl_xor_sync(0xffffffffu, v, o);
  }
  static __device__ __forceinline__ T load(const T *p) { return *(const volatile T *)p; }
};
/* complex: sums (OPS_INC); the reference starts OPS_MIN at (MAX, MAX) and
 * OPS_MAX at (0, 0) and defines no order, so only sums are combined */
template <typename R, int OP> struct red<cuda::std::complex<R>, OP> {
  typedef cuda::std::complex<R> C;
  static __device__ __forceinline__ C identity() {
    return OP == OPS_MIN ? C(lim<R>::hi(), lim<R>::hi()) : C(0, 0);
  }
  static __device__ __forceinline__ C combine(C a, C b) { return a + b; }
  static __device__ __forceinline__ C shfl_xor(C v, int o) {
    return C(__shfl_xor_sync(0xffffffffu, v.real(), o), __shfl_xor_sync(0xffffffffu, v.imag(), o));
  }
  static __device__ __forceinline__ C load(const C *p) {
    const volatile R *q = (const volatile R *)p;
    const R re = q[0], im = q[1];
    return C(re, im);
  }
};

template <typename T, int OP> __device__ __forceinline__ T identity() {
  return red<T, OP>::identity();
}

template <typename T, int OP> __device__ __forceinline__ T combine(T a, T b) {
  return red<T, OP>::combine(a, b);
}

template <typename T, int OP> __device__ __forceinline__ T warp_reduce(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = combine<T, OP>(v, red<T, OP>::shfl_xor(v, o));
  return v;
}

/* whole-CTA reduction; result valid in thread 0.  `sh` needs 32 slots. */
template <typename T, int OP> __device__ __forceinline__ T block_reduce(T v, T *sh) {
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  v = warp_reduce<T, OP>(v);
  const int nw = (nt + 31) >> 5;
  __syncthreads();
  if ((t & 31) == 0) sh[t >> 5] = v;
  __syncthreads();
  if (t < 32) {
    v = t < nw ? sh[t] : identity<T, OP>();
    v = warp_reduce<T, OP>(v);
  }
  return v;
}

/* Step 1 (every reduction argument): this CTA's partial into its slot.
 * part holds nblocks * dim values of one reduction argument. */
template <typename T, int OP>
__device__ __forceinline__ void block_partial(const T *local, int dim, T *part, T *sh) {
  const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  for (int d = 0; d < dim; d++) {
    T v = block_reduce<T, OP>(local[d], sh);
    if (t == 0) part[(size_t)b * dim + d] = v;
  }
}

/* Step 2 (once per kernel): returns true in every thread of the last CTA. */
__device__ __forceinline__ bool last_block(unsigned int *counter, int *flag) {
  const int nb = gridDim.x * gridDim.y * gridDim.z;
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  __threadfence();
  __syncthreads();
  if (t == 0) {
    unsigned int ticket = atomicAdd(counter, 1u);
    *flag = (ticket == (unsigned int)nb - 1u);
  }
  __syncthreads();
  if (*flag) __threadfence();
  return *flag != 0;
}

/* Step 3 (last CTA, every reduction argument): fixed-order combine of all
 * partials, folded into the handle's accumulator. */
template <typename T, int OP>
__device__ __forceinline__ void final_combine(int dim, const T *part, T *acc, int first, T *sh) {
  const int nb = gridDim.x * gridDim.y * gridDim.z;
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  for (int d = 0; d < dim; d++) {
    T v = identity<T, OP>();
    for (int i = t; i < nb; i += nt)
      v = combine<T, OP>(v, red<T, OP>::load(part + (size_t)i * dim + d));
    v = block_reduce<T, OP>(v, sh);
    if (t == 0) acc[d] = first ? v : combine<T, OP>(acc[d], v);
  }
}

/* Step 4 (last CTA, once): re-arm the ticket for the next launch. */
__device__ __forceinline__ void reset_counter(unsigned int *counter) {
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if (t == 0) *counter = 0u;
}

/* CTA tile of the temporal-blocking kernels (ob2_tblock, ops_b200_loop.h) */
#ifndef OB2_TB_TX
#define OB2_TB_TX 64
#endif
#ifndef OB2_TB_TY
#define OB2_TB_TY 16
#endif

/* ---- halo group folded into a loop launch (ob2_hfuse, ops_b200_loop.h) ----
 * Copies the cells of the folded group that lie in this CTA's footprint: the
 * CTA's tile [x0,x1) x [y0,y1) x [z0,z1) in loop coordinates widened by the
 * loop's stencil reach.  A cell is located exactly as the halo transfer
 * kernel locates it (destination storage index start + t or, flipped,
 * start + L - 1 - t along each dimension); overlapping footprints copy the
 * same value from the same source.  The caller synchronises the CTA before
 * the loop reads the copied cells. */
__device__ __forceinline__ void hfuse_copy(const ob2_halo_task &T, const long long *s,
                                           const int *t) {
  long long so = 0, dof = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const int a = T.src_axis[i];
    const int ti = T.src_flip[i] ? T.iter[a] - 1 - t[a] : t[a];
    so += (long long)(T.src_start[i] + ti) * T.src_cum[i];
    dof += s[i] * T.dst_cum[i];
  }
  for (int c = 0; c < T.ncomp; c++) {
    const long long se = T.src_soa ? so + c * T.src_npts_total : so * T.ncomp + c;
    const long long de = T.dst_soa ? dof + c * T.dst_npts_total : dof * T.ncomp + c;
    const char *sp = T.src + se * T.src_type;
    char *dp = T.dst + de * T.dst_type;
    if (T.src_type == T.dst_type) {
      if (T.src_type == 8)
        *(unsigned long long *)dp = *(const unsigned long long *)sp;
      else if (T.src_type == 4)
        *(unsigned int *)dp = *(const unsigned int *)sp;
      else if (T.src_type == 2)
        *(unsigned short *)dp = *(const unsigned short *)sp;
      else
        for (int b = 0; b < T.src_type; b++) dp[b] = sp[b];
    } else {
      const double v = T.src_type == 8   ? *(const double *)sp
                       : T.src_type == 2 ? (double)__half2float(*(const __half *)sp)
                                         : (double)*(const float *)sp;
      if (T.dst_type == 8)
        *(double *)dp = v;
      else if (T.dst_type == 2)
        *(__half *)dp = __double2half(v);
      else
        *(float *)dp = (float)v;
    }
  }
}

__device__ __forceinline__ void hfuse_prologue(const ob2_hfuse &h, int inst, int x0, int x1,
                                               int y0, int y1, int z0, int z1) {
  if (x0 >= x1 || y0 >= y1 || z0 >= z1) return;  // no points: no footprint
  const int flo[3] = {x0 - h.mlo[0], y0 - h.mlo[1], z0 - h.mlo[2]};
  const int fhi[3] = {x1 + h.mhi[0], y1 + h.mhi[1], z1 + h.mhi[2]};
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  for (int e = 0; e < h.n; e++) {
    if (h.inst[e] != inst) continue;
    const ob2_halo_task &T = h.tasks[h.task[e]];
    int lo[3], cnt[3];
    long long total = 1;
#pragma unroll
    for (int i = 0; i < 3; i++) {  // the task's cells along dim i, in loop coordinates
      const int a = h.org[e][i] + T.dst_start[i];
      const int b = a + T.iter[T.dst_axis[i]];
      lo[i] = max(a, flo[i]);
      cnt[i] = max(0, min(b, fhi[i]) - lo[i]);
      total *= cnt[i];
    }
    for (long long k = tid; k < total; k += nt) {
      long long s[3];
      int t[3];
      long long rem = k;
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int off = (int)(rem % cnt[i]);
        rem /= cnt[i];
        s[i] = (long long)(lo[i] + off - h.org[e][i]);  // destination storage index
        const int ti = (int)(s[i] - T.dst_start[i]);
        const int a = T.dst_axis[i];
        t[a] = T.dst_flip[i] ? T.iter[a] - 1 - ti : ti;
      }
      hfuse_copy(T, s, t);
    }
  }
}

/* ---- division in user kernels -------------------------------------------
 * The translator rewrites every binary `/` of a user kernel it can parse
 * safely into div(lhs, rhs) (ops_b200/translator/divrewrite.py).  A double
 * quotient is computed by ddiv, every other quotient by the operator itself.
 *
 * Why: CUDA's double division takes a long guarded path when the numerator
 * is zero (measured on the B200, 7 divisions per point over 16M points:
 * 109 us with nonzero numerators, 332 us with zero ones), and hydrodynamics
 * kernels divide zero gradients and fluxes on every cell at rest.  ddiv
 * costs the same for both (129-135 us).
 *
 * ddiv(a, b) returns the correctly rounded quotient, the same bits as the
 * IEEE division, by Newton-Raphson iteration on the reciprocal and
 * Markstein's correction of the quotient (P. Markstein, "Computation of
 * elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
 * Dev. 34(1), 1990; the theorems as stated in J.-M. Muller et al., Handbook
 * of Floating-Point Arithmetic, ch. 4-5):
 *   y0 = the hardware reciprocal approximation of b (rcp.approx.ftz.f64);
 *   y <- y + y (1 - b y), three times with fused multiply-adds: two steps
 *        bring y within one ulp of 1/b, and the third then rounds it
 *        correctly (Markstein's reciprocal theorem; it excludes divisors
 *        whose significand is all ones, which take the IEEE division here);
 *   q0 = RN(a y) is within one ulp of a/b; r = a - b q0 is exact with an
 *        FMA; q = RN(q0 + r y) is RN(a/b) (Markstein's division theorem).
 * The theorems need every intermediate in the normal range: |a| and |b| in
 * [2^-500, 2^500) guarantee that (the quotient, the residual and the
 * reciprocal stay far from underflow and overflow).  Zero numerators return
 * RN(a y), the correctly signed zero.  Every other operand (subnormal, huge,
 * zero divisor, infinity, NaN) takes the IEEE division.  Checked against
 * CUDA's `/` bit for bit on 10^10 generated pairs (tests/test_gpu_ddiv.py).
 * A zero-numerator shortcut in front of the IEEE division was measured as
 * well and was slower inside the CloverLeaf kernels (5.27 against 4.79 ms
 * per 3840^2 step). */
__device__ __forceinline__ double ddiv(double a, double b) {
  const unsigned ha = (unsigned)__double2hiint(a), hb = (unsigned)__double2hiint(b);
  const unsigned ea = (ha >> 20) & 0x7ffu, eb = (hb >> 20) & 0x7ffu;
  const bool b_ok = (eb - 523u < 1000u) &&
                    !((hb & 0xfffffu) == 0xfffffu && __double2loint(b) == -1);
  const bool a_ok = (ea - 523u < 1000u) || a == 0.0;
  if (!(a_ok && b_ok)) return a / b;
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  const double q0 = __dmul_rn(a, y);
  const double r = __fma_rn(-b, q0, a);
  return a == 0.0 ? q0 : __fma_rn(r, y, q0);
}

template <typename A, typename B>
using quot_t = decltype(std::declval<A>() / std::declval<B>());

/* quotients that are not double: the operator itself (constexpr, so a
 * rewritten integer division still works in a constant expression) */
template <typename A, typename B,
          typename std::enable_if<!std::is_same<quot_t<A, B>, double>::value,
                                        int>::type = 0>
__host__ __device__ constexpr quot_t<A, B> div(A a, B b) {
  return a / b;
}

/* double quotients (after the usual arithmetic conversions) */
template <typename A, typename B,
          typename std::enable_if<std::is_same<quot_t<A, B>, double>::value,
                                        int>::type = 0>
__device__ __forceinline__ double div(A a, B b) {
  return ddiv((double)a, (double)b);
}

}  // namespace ob2

#endif /* OPS_B200_KERNEL_H */
