// ob2_device.cu -- CUDA side of the thin C ABI (include/ops_b200_device.h):
// device selection, the work stream, memory, events, halo transfer, box
// copies and fills.  Kernels here are HBM-bound byte/element moves: no tensor
// cores; coalesced along x, grids sized from the SM count.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>

#include "ops_b200_device.h"

namespace {

// CUDA's lazy module loading (the default since CUDA 12.2) loads a kernel at
// its first launch; in a process that alternates kernels of several
// libraries (an application's generated kernels, then this library's), a
// launch of this library's x-direction tridiagonal kernel blocked about
// 220 us on the host at every ADI step with the device left idle meanwhile
// (256^3 FP64 ADI step: 1.13 ms lazy, 0.89 ms eager, measured).  So when
// the library is loaded, before any CUDA call of the process, it asks for
// eager loading unless the process chose a mode itself (an explicit
// CUDA_MODULE_LOADING=LAZY is kept).  A process that initialised CUDA
// before loading the library keeps the mode it started with.
__attribute__((constructor)) void ob2_module_loading() {
  if (!getenv("CUDA_MODULE_LOADING")) setenv("CUDA_MODULE_LOADING", "EAGER", 0);
}

cudaStream_t g_stream = nullptr;   // current work stream
cudaStream_t g_default = nullptr;  // the runtime's own non-blocking stream
int g_sms = 148;
int g_device = -1;                 // the device ob2_dev_init selected

inline int rc(cudaError_t e) { return (int)e; }

}  // namespace

OB2_API int ob2_dev_init(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return rc(e);
  if (n == 0) return (int)cudaErrorNoDevice;
  if (device < 0 || device >= n) device = 0;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return rc(e);
  g_device = device;
  cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, device);
  if (!g_default) {
    e = cudaStreamCreateWithFlags(&g_default, cudaStreamNonBlocking);
    if (e != cudaSuccess) return rc(e);
  }
  g_stream = g_default;
  return 0;
}

OB2_API int ob2_dev_count(int *n) { return rc(cudaGetDeviceCount(n)); }
OB2_API int ob2_dev_sm_count(int *n) {
  *n = g_sms;
  return 0;
}
OB2_API void *ob2_dev_stream(void) { return (void *)g_stream; }
OB2_API int ob2_dev_set_stream(void *s) {
  g_stream = s ? (cudaStream_t)s : g_default;
  return 0;
}
OB2_API int ob2_dev_malloc(void **p, size_t n) { return rc(cudaMalloc(p, n ? n : 16)); }
OB2_API int ob2_dev_free(void *p) { return p ? rc(cudaFree(p)) : 0; }
OB2_API int ob2_dev_memset(void *p, int v, size_t n) {
  return rc(cudaMemsetAsync(p, v, n, g_stream));
}
OB2_API int ob2_dev_h2d(void *dst, const void *src, size_t n) {
  cudaError_t e = cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, g_stream);
  if (e != cudaSuccess) return rc(e);
  return rc(cudaStreamSynchronize(g_stream));
}
OB2_API int ob2_dev_d2h(void *dst, const void *src, size_t n) {
  cudaError_t e = cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, g_stream);
  if (e != cudaSuccess) return rc(e);
  return rc(cudaStreamSynchronize(g_stream));
}
OB2_API int ob2_dev_d2d(void *dst, const void *src, size_t n) {
  return rc(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, g_stream));
}
OB2_API int ob2_dev_h2d_async(void *dst, const void *src, size_t n) {
  return rc(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, g_stream));
}
OB2_API int ob2_dev_d2h_async(void *dst, const void *src, size_t n) {
  return rc(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, g_stream));
}
OB2_API int ob2_dev_sync(void) { return rc(cudaStreamSynchronize(g_stream)); }
OB2_API int ob2_host_alloc_pinned(void **p, size_t n) {
  return rc(cudaHostAlloc(p, n ? n : 16, cudaHostAllocPortable));
}
OB2_API int ob2_host_free_pinned(void *p) { return p ? rc(cudaFreeHost(p)) : 0; }
OB2_API const char *ob2_error_string(int code) {
  if (code == OB2_ERR_NOALLOC_LIMIT)
    return "halo task table larger than the allocation-free maximum (OB2_HALO_STATIC_MAX)";
  return cudaGetErrorString((cudaError_t)code);
}
OB2_API int ob2_last_launch_error(void) { return rc(cudaGetLastError()); }
OB2_API int ob2_mem_info(size_t *f, size_t *t) { return rc(cudaMemGetInfo(f, t)); }

OB2_API int ob2_event_create(void **ev) {
  return rc(cudaEventCreate((cudaEvent_t *)ev));
}
OB2_API int ob2_event_record(void *ev) { return rc(cudaEventRecord((cudaEvent_t)ev, g_stream)); }
OB2_API int ob2_event_elapsed_ms(void *a, void *b, float *ms) {
  cudaError_t e = cudaEventSynchronize((cudaEvent_t)b);
  if (e != cudaSuccess) return rc(e);
  return rc(cudaEventElapsedTime(ms, (cudaEvent_t)a, (cudaEvent_t)b));
}
OB2_API int ob2_event_destroy(void *ev) { return rc(cudaEventDestroy((cudaEvent_t)ev)); }

// ---------------------------------------------------------------------------
// Halo transfer: one CTA row (blockIdx.y) per halo task, threads stride over
// the task's points.  Index math mirrors the oracle restatement of
// ops_host_singlenode.cpp:172-446: iteration point t -> per-dimension storage
// index start + (flip ? L-1-t_axis : t_axis).
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ long long storage_offset(const int *axis, const int *flip,
                                                    const int *start, const long long *cum,
                                                    const int *t, const int *iter) {
  long long off = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    int a = axis[i];
    int ti = flip[i] ? iter[a] - 1 - t[a] : t[a];
    off += (long long)(start[i] + ti) * cum[i];
  }
  return off;
}

__device__ __forceinline__ double load_as_double(const char *p, int ts) {
  if (ts == 8) return *(const double *)p;
  if (ts == 2) return (double)__half2float(*(const __half *)p);
  return (double)*(const float *)p;
}

__global__ void halo_kernel(const ob2_halo_task *__restrict__ tasks) {
  const ob2_halo_task &T = tasks[blockIdx.y];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < T.npts;
       i += (long long)gridDim.x * blockDim.x) {
    int t[3];
    long long r = i;
    t[0] = (int)(r % T.iter[0]);
    r /= T.iter[0];
    t[1] = (int)(r % T.iter[1]);
    t[2] = (int)(r / T.iter[1]);
    long long so = storage_offset(T.src_axis, T.src_flip, T.src_start, T.src_cum, t, T.iter);
    long long dof = storage_offset(T.dst_axis, T.dst_flip, T.dst_start, T.dst_cum, t, T.iter);
    for (int c = 0; c < T.ncomp; c++) {
      long long se = T.src_soa ? so + c * T.src_npts_total : so * T.ncomp + c;
      long long de = T.dst_soa ? dof + c * T.dst_npts_total : dof * T.ncomp + c;
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
        double v = load_as_double(sp, T.src_type);
        if (T.dst_type == 8)
          *(double *)dp = v;
        else if (T.dst_type == 2)
          *(__half *)dp = __double2half(v);
        else
          *(float *)dp = (float)v;
      }
    }
  }
}

}  // namespace

OB2_API int ob2_halo_run(const ob2_halo_task *tasks_dev, int ntasks, long long max_pts) {
  if (ntasks <= 0 || max_pts <= 0) return 0;
  long long blocks = (max_pts + 255) / 256;
  if (blocks > 4LL * g_sms) blocks = 4LL * g_sms;
  dim3 grid((unsigned)blocks, (unsigned)ntasks);
  halo_kernel<<<grid, 256, 0, g_stream>>>(tasks_dev);
  return rc(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Allocation-free halo transfer: the task table lives in a fixed array
// compiled into this library instead of caller-allocated device memory.
// ---------------------------------------------------------------------------
namespace {

__device__ __align__(256) ob2_halo_task g_halo_static[OB2_HALO_STATIC_MAX];

constexpr int kMaxDevices = 64;
// device address of g_halo_static, looked up once per device (host code may
// not pass the symbol itself to a kernel: its host-side name is a stand-in);
// atomic so that first calls from several host threads do not race
std::atomic<ob2_halo_task *> g_halo_static_addr[kMaxDevices];

}  // namespace

OB2_API int ob2_halo_run_noalloc(const ob2_halo_task *tasks_host, int ntasks) {
  if (ntasks < 0 || (ntasks > 0 && !tasks_host)) return (int)cudaErrorInvalidValue;
  if (ntasks > OB2_HALO_STATIC_MAX) return OB2_ERR_NOALLOC_LIMIT;
  if (ntasks == 0) return 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return rc(e);
  if (dev < 0 || dev >= kMaxDevices) return (int)cudaErrorInvalidDevice;
  // the launch goes to the work stream, which belongs to the device that
  // ob2_dev_init selected: the array looked up must be that device's
  if (g_device >= 0 && dev != g_device) return (int)cudaErrorInvalidDevice;
  ob2_halo_task *table = g_halo_static_addr[dev].load(std::memory_order_acquire);
  if (!table) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_halo_static);
    if (e != cudaSuccess) return rc(e);
    table = (ob2_halo_task *)p;
    g_halo_static_addr[dev].store(table, std::memory_order_release);
  }
  long long max_pts = 0;
  for (int i = 0; i < ntasks; i++)
    if (tasks_host[i].npts > max_pts) max_pts = tasks_host[i].npts;
  // stream-ordered: an earlier launch on this stream still reading the table
  // finishes before it is overwritten
  e = cudaMemcpyAsync(table, tasks_host, sizeof(ob2_halo_task) * ntasks,
                      cudaMemcpyHostToDevice, g_stream);
  if (e != cudaSuccess) return rc(e);
  return ob2_halo_run(table, ntasks, max_pts);
}

// ---------------------------------------------------------------------------
// Box copy between a dat (storage coordinates start3/count3) and a dense AoS
// buffer, for fetch/set data and slabs (ops_util.cpp:353-500 semantics).
// ---------------------------------------------------------------------------
namespace {

__global__ void box_copy_kernel(char *dat, int ts, int nc, int soa, long long sx, long long sy,
                                long long ntot, int s0, int s1, int s2, int c0, int c1, int c2,
                                char *buf, int dir) {
  long long n = (long long)c0 * c1 * c2;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int x = (int)(i % c0);
    long long r = i / c0;
    int y = (int)(r % c1);
    int z = (int)(r / c1);
    long long pt = (long long)(s0 + x) + (long long)(s1 + y) * sx + (long long)(s2 + z) * sy;
    for (int c = 0; c < nc; c++) {
      long long de = soa ? pt + c * ntot : pt * nc + c;
      char *dp = dat + de * ts;
      char *bp = buf + (i * nc + c) * ts;
      char *from = dir == 0 ? dp : bp;
      char *to = dir == 0 ? bp : dp;
      if (ts == 8)
        *(unsigned long long *)to = *(const unsigned long long *)from;
      else if (ts == 4)
        *(unsigned int *)to = *(const unsigned int *)from;
      else
        for (int b = 0; b < ts; b++) to[b] = from[b];
    }
  }
}

}  // namespace

OB2_API int ob2_box_copy(char *dat, int ts, int nc, int soa, const int *size3, const int *start3,
                         const int *count3, char *buf, int dir) {
  long long n = (long long)count3[0] * count3[1] * count3[2];
  if (n <= 0) return 0;
  long long blocks = (n + 255) / 256;
  if (blocks > 8LL * g_sms) blocks = 8LL * g_sms;
  long long sx = size3[0], sy = (long long)size3[0] * size3[1];
  long long ntot = sy * size3[2];
  box_copy_kernel<<<(unsigned)blocks, 256, 0, g_stream>>>(dat, ts, nc, soa, sx, sy, ntot,
                                                          start3[0], start3[1], start3[2],
                                                          count3[0], count3[1], count3[2],
                                                          buf, dir);
  return rc(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Fills
// ---------------------------------------------------------------------------
namespace {

__global__ void fill_kernel(char *p, unsigned long long v, int ts, size_t count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x) {
    if (ts == 8)
      ((unsigned long long *)p)[i] = v;
    else if (ts == 4)
      ((unsigned int *)p)[i] = (unsigned int)v;
    else if (ts == 2)
      ((unsigned short *)p)[i] = (unsigned short)v;
    else
      p[i] = (char)v;
  }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

__global__ void random_kernel(char *p, int ts, size_t count, unsigned long long seed,
                              unsigned long long counter, int normal) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long k = counter + i;
    unsigned long long r1 = mix64(seed * 0x100000001b3ULL ^ (2 * k));
    double u1 = (double)(r1 >> 11) * (1.0 / 9007199254740992.0);
    double v = u1;
    if (normal) {
      unsigned long long r2 = mix64(seed * 0x100000001b3ULL ^ (2 * k + 1));
      double u2 = (double)(r2 >> 11) * (1.0 / 9007199254740992.0);
      v = sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307179586 * u2);
    }
    if (ts == 8)
      ((double *)p)[i] = v;
    else
      ((float *)p)[i] = (float)v;
  }
}

}  // namespace

namespace {
template <typename T>
__global__ void nan_find_kernel(const T *__restrict__ p, int ncomp, int soa, size_t count,
                                unsigned long long *first) {
  const size_t npts = count / (size_t)ncomp;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < count;
       e += (size_t)gridDim.x * blockDim.x) {
    const T v = p[e];
    if (v != v) {
      const unsigned long long key =
          soa ? (unsigned long long)(e % npts) * ncomp + e / npts : (unsigned long long)e;
      atomicMin(first, key);
    }
  }
}
}  // namespace

OB2_API int ob2_nan_find(const void *p, int ts, int ncomp, int soa, size_t count,
                         long long *first) {
  *first = -1;
  if (count == 0 || ncomp < 1) return 0;
  if (ts != 8 && ts != 4) return (int)cudaErrorInvalidValue;
  unsigned long long *d = nullptr, h = ~0ULL;
  cudaError_t e = cudaMallocAsync(&d, sizeof(h), g_stream);
  if (e != cudaSuccess) return rc(e);
  e = cudaMemcpyAsync(d, &h, sizeof(h), cudaMemcpyHostToDevice, g_stream);
  const unsigned blocks = (unsigned)std::min<size_t>((count + 255) / 256, (size_t)g_sms * 8);
  if (e == cudaSuccess) {
    if (ts == 8)
      nan_find_kernel<double><<<blocks, 256, 0, g_stream>>>((const double *)p, ncomp, soa, count, d);
    else
      nan_find_kernel<float><<<blocks, 256, 0, g_stream>>>((const float *)p, ncomp, soa, count, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, g_stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_stream);
  cudaFreeAsync(d, g_stream);
  if (e != cudaSuccess) return rc(e);
  *first = h == ~0ULL ? -1 : (long long)h;
  return 0;
}

OB2_API int ob2_fill_value(void *p, const void *val, int ts, size_t count) {
  if (count == 0) return 0;
  if (ts == 16) {  // a complex value whose two halves are equal: 2 count 8-byte values
    if (memcmp(val, (const char *)val + 8, 8) != 0) return (int)cudaErrorInvalidValue;
    ts = 8;
    count *= 2;
  }
  if (ts > 8 || ts < 1) return (int)cudaErrorInvalidValue;
  unsigned long long v = 0;
  memcpy(&v, val, ts <= 8 ? ts : 8);
  size_t blocks = (count + 255) / 256;
  if (blocks > (size_t)8 * g_sms) blocks = (size_t)8 * g_sms;
  fill_kernel<<<(unsigned)blocks, 256, 0, g_stream>>>((char *)p, v, ts, count);
  return rc(cudaGetLastError());
}

OB2_API int ob2_fill_random(void *p, int ts, size_t count, unsigned long long seed,
                            unsigned long long counter, int normal) {
  if (count == 0) return 0;
  size_t blocks = (count + 255) / 256;
  if (blocks > (size_t)8 * g_sms) blocks = (size_t)8 * g_sms;
  random_kernel<<<(unsigned)blocks, 256, 0, g_stream>>>((char *)p, ts, count, seed, counter,
                                                          normal);
  return rc(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Graph capture of the work stream (loop chains)
// ---------------------------------------------------------------------------
OB2_API int ob2_graph_begin_capture(void) {
  return rc(cudaStreamBeginCapture(g_stream, cudaStreamCaptureModeThreadLocal));
}
OB2_API int ob2_graph_end_capture(void **exec) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(g_stream, &g);
  if (e != cudaSuccess) return rc(e);
  if (*exec) {
    cudaGraphExecUpdateResultInfo info;
    e = cudaGraphExecUpdate((cudaGraphExec_t)*exec, g, &info);
    if (e == cudaSuccess) {
      cudaGraphDestroy(g);
      return 0;
    }
    (void)cudaGetLastError();  // a refused update is not an error
    cudaGraphExecDestroy((cudaGraphExec_t)*exec);
    *exec = nullptr;
  }
  cudaGraphExec_t ge = nullptr;
  e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return rc(e);
  *exec = (void *)ge;
  return 0;
}
OB2_API int ob2_graph_launch(void *exec) {
  return rc(cudaGraphLaunch((cudaGraphExec_t)exec, g_stream));
}
OB2_API int ob2_graph_destroy(void *exec) {
  return exec ? rc(cudaGraphExecDestroy((cudaGraphExec_t)exec)) : 0;
}
