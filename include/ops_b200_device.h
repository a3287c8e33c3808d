/*
 * ops_b200_device.h -- the thin C ABI between the OPS host runtime and CUDA.
 *
 * Plain pointers, sizes and integer status codes (0 = success, otherwise a
 * cudaError_t value); no CUDA or torch types cross it.  The host runtime
 * (ops_b200/csrc/host) turns non-zero codes into OPSException, matching the
 * reference's cutilSafeCall behaviour (ops/c/src/cuda/ops_cuda_common.cu:50-58).
 *
 * Each entry names the reference routine it replaces.
 */
#ifndef OPS_B200_DEVICE_H
#define OPS_B200_DEVICE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#define OB2_API extern "C" __attribute__((visibility("default")))
#else
#define OB2_API extern __attribute__((visibility("default")))
#endif

/* ---- device / stream / memory (ops_cuda_common.cu:68-182) ---- */
OB2_API int ob2_dev_init(int device);           /* cutilDeviceInit */
OB2_API int ob2_dev_count(int *n);
OB2_API int ob2_dev_sm_count(int *n);           /* SMs of the current device */
OB2_API void *ob2_dev_stream(void);             /* the runtime's work stream */
OB2_API int ob2_dev_set_stream(void *stream);   /* 0 restores the default work stream */
OB2_API int ob2_dev_malloc(void **p, size_t n); /* ops_device_malloc */
OB2_API int ob2_dev_free(void *p);              /* ops_device_free */
OB2_API int ob2_dev_memset(void *p, int v, size_t n);
OB2_API int ob2_dev_h2d(void *dst, const void *src, size_t n); /* ops_device_memcpy_h2d */
OB2_API int ob2_dev_d2h(void *dst, const void *src, size_t n); /* ops_device_memcpy_d2h */
OB2_API int ob2_dev_d2d(void *dst, const void *src, size_t n);
OB2_API int ob2_dev_h2d_async(void *dst, const void *src, size_t n);
OB2_API int ob2_dev_d2h_async(void *dst, const void *src, size_t n);
OB2_API int ob2_dev_sync(void);                 /* ops_device_sync */
OB2_API int ob2_host_alloc_pinned(void **p, size_t n);
OB2_API int ob2_host_free_pinned(void *p);
OB2_API const char *ob2_error_string(int code);
OB2_API int ob2_last_launch_error(void);
OB2_API int ob2_mem_info(size_t *free_b, size_t *total_b);

/* ---- events (timing of device work on the work stream) ---- */
OB2_API int ob2_event_create(void **ev);
OB2_API int ob2_event_record(void *ev);
OB2_API int ob2_event_elapsed_ms(void *start, void *end, float *ms);
OB2_API int ob2_event_destroy(void *ev);

/* ---- multi-block halo transfer (ops_device_singlenode_common.cpp:262-346,
 *      ops_cuda_rt_support.cu:55-253).  One task per halo: copies the box
 *      iter_size from `src` into `dst` with per-axis permutation/flip; all
 *      tasks of a group run in one launch. ---- */
typedef struct ob2_halo_task {
  char *src;             /* device base of the source dat */
  char *dst;             /* device base of the target dat */
  int src_type;          /* bytes per component: 2, 4 or 8 */
  int dst_type;
  int ncomp;             /* components per point copied */
  int src_soa, dst_soa;
  int iter[3];           /* box extent along iteration axes */
  long long npts;        /* iter[0]*iter[1]*iter[2] */
  /* for dat dimension i: iteration axis, flip flag, storage start, element
   * stride of one step along dimension i (points, not bytes) */
  int src_axis[3], src_flip[3], src_start[3];
  long long src_cum[3];
  int dst_axis[3], dst_flip[3], dst_start[3];
  long long dst_cum[3];
  long long src_npts_total, dst_npts_total; /* for SoA component strides */
  int float_kind;        /* 1 when src/dst are float/double (conversion allowed) */
} ob2_halo_task;

/* tasks: device array of ntasks entries; max_pts: largest npts */
OB2_API int ob2_halo_run(const ob2_halo_task *tasks_dev, int ntasks, long long max_pts);

/* Halo transfer that allocates nothing (no counterpart in the reference).
 *
 * For callers that must not call cudaMalloc: code that runs while another
 * component owns the device memory budget (a serving process whose pool is
 * carved up in advance, a framework's caching allocator), or host code that
 * may not create allocations between setup and teardown.  ob2_halo_run needs
 * its task table in device memory that the caller allocated; this variant
 * takes the table in host memory and stages it, with an ordinary stream-
 * ordered copy, into a fixed array of OB2_HALO_STATIC_MAX tasks that is
 * compiled into the library (a file-scope __device__ array: every GPU that
 * loads the library holds its OB2_HALO_STATIC_MAX x sizeof(ob2_halo_task),
 * about 210 KB, until the process exits).  The halo
 * kernel itself is the same as ob2_halo_run's.
 *
 * - Returns OB2_ERR_NOALLOC_LIMIT (see ob2_error_string) when ntasks exceeds
 *   OB2_HALO_STATIC_MAX, and cudaErrorInvalidValue when ntasks is negative
 *   (or tasks_host is NULL with ntasks > 0), without copying or launching
 *   anything.
 * - Must be called with the device that ob2_dev_init selected current (the
 *   work stream belongs to it); otherwise returns cudaErrorInvalidDevice.
 * - The first call on a device looks up the array's device address on that
 *   device (cudaGetSymbolAddress); make that first call before any stream
 *   capture begins.
 * - The table is copied with cudaMemcpyAsync on the work stream.  From pinned
 *   host memory that copy runs later, when the stream reaches it: keep the
 *   caller's table unchanged until then (for example until ob2_dev_sync
 *   returns).  From pageable memory the table is read before the call
 *   returns.
 * - All calls share the one array, which keeps the last call's table: two
 *   calls whose work overlaps on the GPU (different streams, or different
 *   host threads) race on it.  Calls on one stream are ordered and safe.
 * - Calls no cudaMalloc / cudaFree and no allocating library routine. */
#define OB2_HALO_STATIC_MAX 1024
#define OB2_ERR_NOALLOC_LIMIT 100001
OB2_API int ob2_halo_run_noalloc(const ob2_halo_task *tasks_host, int ntasks);

/* ---- dense box copy between a dat and a packed AoS buffer
 *      (ops_cuda_rt_support.cu:256-451, fetch/set slab).  dir 0: dat->buf,
 *      dir 1: buf->dat.  buf may be device or host-pinned memory. ---- */
OB2_API int ob2_box_copy(char *dat, int type_size, int ncomp, int soa, const int *size3,
                         const int *start3, const int *count3, char *buf, int dir);

/* ---- fills ---- */
/* count values of type_size bytes (1-8, or 16 when both 8-byte halves of
 * the value are equal, as for complex identities) */
OB2_API int ob2_fill_value(void *p, const void *val, int type_size, size_t count);
/* smallest key of a NaN element (key = point * ncomp + component; elements
 * are SoA when soa != 0, AoS otherwise) into *first, or -1 when none;
 * type_size 8 (double) or 4 (float) */
OB2_API int ob2_nan_find(const void *p, int type_size, int ncomp, int soa, size_t count,
                         long long *first);
/* counter-based uniform / normal stream (splitmix64 of seed and index);
 * type_size 8 (double) or 4 (float) */
OB2_API int ob2_fill_random(void *p, int type_size, size_t count, unsigned long long seed,
                            unsigned long long counter, int normal);

/* ---- batched tridiagonal solves (ops_tridiag_cuda.cpp:96-251; solver is
 *      this backend's own).  Arrays point at the first solved point; strides
 *      in elements.  u == NULL: solution overwrites d; else u += solution.
 *      type_size 8 (double) or 4 (float storage, FP64 elimination). ---- */
OB2_API int ob2_trid_batch(int type_size, int ndim, int solvedim, const int *dims,
                           const long long *strides, const void *a, const void *b,
                           const void *c, void *d, void *u);

/* ---- loop-chain graphs: stream capture of queued work ---- */
OB2_API int ob2_graph_begin_capture(void);
/* Ends the capture.  *graph_exec == NULL: instantiates a new executable graph.
 * Otherwise first tries to update *graph_exec in place with the captured
 * launches (same topology, new kernel parameters: no instantiation); when the
 * update is refused, replaces *graph_exec with a new instantiation. */
OB2_API int ob2_graph_end_capture(void **graph_exec);
OB2_API int ob2_graph_launch(void *graph_exec);
OB2_API int ob2_graph_destroy(void *graph_exec);

#endif /* OPS_B200_DEVICE_H */
