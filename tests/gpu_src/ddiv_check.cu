// Test harness (GPU tests only): compares ob2::ddiv, the division that the
// translator puts into user kernels (include/ops_b200_kernel.h), with the
// IEEE division of CUDA's `/` operator on generated operand pairs, bit for
// bit.  Each thread draws its pairs from a counter-based hash of (seed, index).
#include <cstdint>
#include <cstring>

#include "ops_b200_kernel.h"

namespace {

__device__ __forceinline__ uint64_t mix(uint64_t x) {  // splitmix64 finaliser
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ double with_exp(uint64_t bits, unsigned e) {
  return __longlong_as_double((long long)((bits & 0x800fffffffffffffull) | ((uint64_t)e << 52)));
}

// mode 0: both operands in the fast domain, random signs and significands
// mode 1: quotients next to a rounding midpoint (a = RN(b * (q + ulp(q)/2)))
// mode 2: zero numerators of both signs and small integers, over ordinary
//         divisors and zeros, infinities, NaNs and subnormals
// mode 3: divisors with significands near all ones and powers of two
// mode 4: any bit pattern (subnormals, infinities, NaNs: the IEEE path)
__device__ void pair(int mode, uint64_t r0, uint64_t r1, uint64_t r2, double &a, double &b) {
  const unsigned ea = 523u + (unsigned)(r2 % 1000u), eb = 523u + (unsigned)((r2 >> 20) % 1000u);
  switch (mode) {
    case 0:
      a = with_exp(r0, ea);
      b = with_exp(r1, eb);
      break;
    case 1: {
      const unsigned eq = 923u + (unsigned)(r2 % 200u);
      b = with_exp(r1, 1023u + (unsigned)((r2 >> 20) % 64u) - 32u);
      const double q = fabs(with_exp(r0, eq));
      const double half_ulp = ldexp(1.0, (int)eq - 1023 - 53);
      a = __fma_rn(b, q, b * half_ulp);  // about b (q + ulp/2), rounded once
      break;
    }
    case 2: {
      a = (r0 & 1) ? -0.0 : 0.0;
      if (r0 & 2) a = (double)((int64_t)(r0 >> 40) - (1 << 23));
      b = (r1 & 4) ? with_exp(r1, eb) : (double)((int64_t)(r1 >> 44) | 1) * ((r1 & 8) ? -1 : 1);
      const double sg = (r1 & 16) ? -1.0 : 1.0;
      switch ((r1 >> 5) % 16) {  // divisors with special IEEE rules, one pair in four
        case 0: b = sg * 0.0; break;
        case 1: b = sg * __longlong_as_double(0x7ff0000000000000ll); break;
        case 2: b = __longlong_as_double(0x7ff8000000000000ll); break;
        case 3: b = sg * __longlong_as_double((long long)((r1 >> 12) & 0xfffffffffffffull) | 1); break;
        default: break;
      }
      break;
    }
    case 3: {
      a = with_exp(r0, ea);
      uint64_t m = 0xfffffffffffffull - (r1 >> 58);
      if (r1 & 1) m = r1 & 0xfull;
      b = __longlong_as_double((long long)(((r1 >> 1) & 0x8000000000000000ull) |
                                           ((uint64_t)eb << 52) | m));
      break;
    }
    default:
      a = __longlong_as_double((long long)r0);
      b = __longlong_as_double((long long)r1);
  }
}

__global__ void check_kernel(uint64_t n, uint64_t seed, int mode, unsigned long long *bad,
                             double *first) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t h = mix(seed ^ mix(i));
    double a, b;
    pair(mode, h, mix(h), mix(h ^ 0x5bd1e995ull), a, b);
    const double want = a / b, got = ob2::ddiv(a, b);
    const bool same = __double_as_longlong(want) == __double_as_longlong(got) ||
                      (want != want && got != got);
    if (!same) {
      if (atomicAdd(bad, 1ull) == 0ull) {
        first[0] = a;
        first[1] = b;
        first[2] = got;
      }
    }
  }
}

}  // namespace

// n pairs of the given mode; returns a CUDA error code, *mismatches the count
// of pairs whose quotients differ, first[0..2] = a, b, ddiv(a, b) of one of them
extern "C" int ddiv_check(unsigned long long n, unsigned long long seed, int mode,
                          unsigned long long *mismatches, double *first) {
  unsigned long long *d_bad = nullptr;
  double *d_first = nullptr;
  cudaError_t e = cudaMalloc(&d_bad, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&d_first, 3 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(d_bad, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(d_first, 0, 3 * sizeof(double));
  if (e == cudaSuccess) {
    check_kernel<<<148 * 8, 256>>>(n, seed, mode, d_bad, d_first);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(mismatches, d_bad, sizeof(unsigned long long),
                                       cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(first, d_first, 3 * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d_bad);
  cudaFree(d_first);
  return (int)e;
}
