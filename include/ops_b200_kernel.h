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

/* identity of each reduction (ops_lib_core.cpp:840-854) */
template <typename T, int OP> __device__ __forceinline__ T identity() {
  if (OP == OPS_MIN) return lim<T>::hi();
  if (OP == OPS_MAX) return lim<T>::lo();
  return T(0);
}

template <typename T, int OP> __device__ __forceinline__ T combine(T a, T b) {
  if (OP == OPS_MIN) return b < a ? b : a;
  if (OP == OPS_MAX) return b > a ? b : a;
  return a + b;
}

template <typename T, int OP> __device__ __forceinline__ T warp_reduce(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = combine<T, OP>(v, __shfl_xor_sync(0xffffffffu, v, o));
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
      v = combine<T, OP>(v, ((const volatile T *)part)[(size_t)i * dim + d]);
    v = block_reduce<T, OP>(v, sh);
    if (t == 0) acc[d] = first ? v : combine<T, OP>(acc[d], v);
  }
}

/* Step 4 (last CTA, once): re-arm the ticket for the next launch. */
__device__ __forceinline__ void reset_counter(unsigned int *counter) {
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if (t == 0) *counter = 0u;
}

}  // namespace ob2

#endif /* OPS_B200_KERNEL_H */
