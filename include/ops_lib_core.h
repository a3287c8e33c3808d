/*
 * ops_lib_core.h -- app-facing OPS API of the B200 backend.
 *
 * This header keeps the OPS C/C++ API (same names, argument meaning, error
 * behaviour) so that OPS applications compile against it unchanged.  Every
 * non-template entry point has C linkage and is exported by libops_b200.so;
 * the templates are thin inline wrappers over those C entry points.
 *
 * Reference interface replaced (paths inside the OPS tree):
 *   types              ops/c/include/ops_lib_core.h:183-552
 *   C API              ops/c/include/ops_lib_core.h:579-1296
 *   *_char ABI         ops/c/include/ops_internal1.h:89-95
 *   ACC<T> accessor    ops/c/include/ops_lib_core.h:1357-2038
 *   OPSException       ops/c/include/ops_exceptions.h:46-53
 *
 * Struct layouts of ops_dat_core / ops_block_core / ops_stencil_core /
 * ops_arg / ops_halo_core / ops_reduction_core keep the reference field names
 * because applications read those fields directly (dat->size, block->instance,
 * ...).  The numeric values of OPS_READ..OPS_MAX, OPS_ARG_* and the exception
 * codes are kept so that Fortran / ctypes callers that pass integers keep
 * working.
 */
#ifndef OPS_B200_LIB_CORE_H
#define OPS_B200_LIB_CORE_H

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef __cplusplus
#include <exception>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <type_traits>
#endif

#if !defined(__CUDACC__)
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

/* The 16-bit `half` element type of half-precision dats (the choice of
 * ops_lib_core.h:96-118 of the reference): CUDA's __half in code nvcc
 * compiles (kernels and their stubs), the compiler's IEEE binary16
 * _Float16 in host code, so that both sides share the 2-byte layout. */
#if defined(__CUDACC__)
#ifndef __HALF_DEFINED__
#include <cuda_fp16.h>
#endif
typedef __half half;
#elif defined(__STDCPP_FLOAT16_T__) || defined(FLT16_MIN) || defined(__FLT16_MIN__)
typedef _Float16 half;
#else
typedef uint16_t half;
#endif

/* Complex element types (ops_lib_core.h:95-96 of the reference): std::complex
 * in host code, libcu++'s cuda::std::complex in code nvcc compiles (the
 * generated kernels), both two consecutive values, real then imaginary. */
#ifdef __cplusplus
#if defined(__CUDACC__)
#include <cuda/std/complex>
typedef cuda::std::complex<double> complexd;
typedef cuda::std::complex<float> complexf;
#else
#include <complex>
typedef std::complex<double> complexd;
typedef std::complex<float> complexf;
#endif
#define ZERO_complexd complexd(0, 0)
#define INFINITY_complexd complexd(DBL_MAX, DBL_MAX)
#define ZERO_complexf complexf(0, 0)
#define INFINITY_complexf complexf(FLT_MAX, FLT_MAX)
#endif

#ifdef __cplusplus
#define OPS_EXTERN_C extern "C"
#else
#define OPS_EXTERN_C extern
#endif
#define OPS_API OPS_EXTERN_C __attribute__((visibility("default")))

/* ---------------------------------------------------------------------------
 * Constants (ops_lib_core.h:35-50 of the reference)
 * ------------------------------------------------------------------------- */
#define OPS_MAX_DIM 5
#ifndef OPS_ALIGNMENT
#define OPS_ALIGNMENT 64
#endif

#define OPS_READ 0
#define OPS_WRITE 1
#define OPS_RW 2
#define OPS_INC 3
#define OPS_MIN 4
#define OPS_MAX 5

#define OPS_ARG_GBL 0
#define OPS_ARG_DAT 1
#define OPS_ARG_IDX 2

#define OPS_HOST 1
#define OPS_DEVICE 2

/* exception codes (ops_exceptions.h:46-53) */
#define OPS_NOT_IMPLEMENTED 1
#define OPS_RUNTIME_CONFIGURATION_ERROR 2
#define OPS_INTERNAL_ERROR 3
#define OPS_RUNTIME_ERROR 4
#define OPS_HDF5_ERROR 5
#define OPS_INVALID_ARGUMENT 6

typedef int ops_access;
typedef int ops_arg_type;
typedef int ops_memspace;

#ifndef __cplusplus
typedef struct OPS_instance OPS_instance;
#endif
typedef unsigned int uint;
typedef long long ll;
typedef unsigned long long ull;
typedef unsigned long ul;

/* ---------------------------------------------------------------------------
 * Core objects
 * ------------------------------------------------------------------------- */
#ifdef __cplusplus
class OPS_instance;
#endif

typedef struct ops_block_core {
  int index;
  int dims;
  char const *name;
  OPS_instance *instance;
#ifdef __cplusplus
  /* C++ object API (ops_lib_core.h:190-232 of the reference, OPS_CPP_API):
   * block->decl_dat(...) = ops_decl_dat(block, ...) */
  template <class T>
  struct ops_dat_core *decl_dat(int data_size, int *block_size, int *base, int *d_m, int *d_p,
                                T *data, char const *type, char const *name);
  template <class T>
  struct ops_dat_core *decl_dat(int data_size, int *block_size, int *base, int *d_m, int *d_p,
                                int *stride, T *data, char const *type, char const *name);
#endif
} ops_block_core;
typedef ops_block_core *ops_block;

typedef struct ops_dat_core {
  int index;
  ops_block block;
  int dim;                 /* components per grid point */
  int type_size;           /* bytes per component */
  int elem_size;           /* bytes per grid point = dim * type_size */
  int size[OPS_MAX_DIM];   /* allocated extent per dimension, halos included */
  int base[OPS_MAX_DIM];
  int d_m[OPS_MAX_DIM];    /* negative-side halo depth (<= 0) */
  int d_p[OPS_MAX_DIM];    /* positive-side halo depth (>= 0) */
  int x_pad;
  char *data;              /* host copy (may be NULL until first host access) */
  char *data_d;            /* device copy: authoritative between loops */
  char const *name;
  char const *type;
  int dirty_hd;            /* 0 clean, 1 host newer, 2 device newer */
  int locked_hd;           /* raw pointer handed out, not released yet */
  int user_managed;
  int is_hdf5;
  char const *hdf5_file;
  int e_dat;               /* edge (low-dimensional) dat */
  size_t mem;
  size_t base_offset;      /* bytes from data start to index (0,0,..) */
  int stride[OPS_MAX_DIM];
} ops_dat_core;
typedef ops_dat_core *ops_dat;

typedef struct ops_stencil_core {
  int index;
  int dims;
  int points;
  char const *name;
  int *stencil;       /* points * dims offsets */
  int *stride;        /* per-dimension loop stride (0 = dimension not walked) */
  int *mgrid_stride;
  int type;           /* 0 regular, 1 prolong, 2 restrict */
} ops_stencil_core;
typedef ops_stencil_core *ops_stencil;

typedef struct ops_arg {
  ops_dat dat;
  ops_stencil stencil;
  int dim;
  int elem_size;
  char *data;
  char *data_d;
  ops_access acc;
  ops_arg_type argtype;
  int opt;
} ops_arg;

typedef struct ops_halo_core {
  ops_dat from;
  ops_dat to;
  int iter_size[OPS_MAX_DIM];
  int from_base[OPS_MAX_DIM];
  int to_base[OPS_MAX_DIM];
  int from_dir[OPS_MAX_DIM];
  int to_dir[OPS_MAX_DIM];
  int index;
} ops_halo_core;
typedef ops_halo_core *ops_halo;

typedef struct ops_halo_group_core {
  int nhalos;
  ops_halo *halos;
  int index;
  OPS_instance *instance;
#ifdef __cplusplus
  void halo_transfer();  /* = ops_halo_transfer(group) */
#endif
} ops_halo_group_core;
typedef ops_halo_group_core *ops_halo_group;

typedef struct ops_reduction_core {
  char *data;          /* host value (valid after ops_reduction_result) */
  int size;            /* bytes */
  int initialized;
  int index;
  ops_access acc;
  char *type;
  char *name;
  OPS_instance *instance;
#ifdef __cplusplus
  template <class T> void get_result(T *ptr);  /* = ops_reduction_result(handle, ptr) */
#endif
} ops_reduction_core;
typedef ops_reduction_core *ops_reduction;

/* ---------------------------------------------------------------------------
 * Instance object.  One per process; API calls come from one host thread
 * (same contract as ops_instance.cpp:9-40 of the reference).
 * ------------------------------------------------------------------------- */
#ifdef __cplusplus
class __attribute__((visibility("default"))) OPS_instance {
 public:
  static OPS_instance *getOPSInstance();
  int OPS_soa;
  int OPS_diags;
  int OPS_hybrid_gpu;
  void *backend;     /* backend runtime state */
  std::ostream *os_; /* the stream ostream() returns (NULL: std::cout) */
  OPS_instance() {}
  /* C++ object API (ops_instance.cpp of the reference, OPS_CPP_API): the
   * object an application creates becomes the library's instance (its
   * OPS_soa and output stream are the ones used) and runs ops_init;
   * deleting it runs ops_exit.  One instance per process. */
  OPS_instance(const int argc, const char *const argv[], const int diags = 1,
               std::ostream &os = std::cout);
  ~OPS_instance();
  int is_root() { return 1; }
  std::ostream &ostream() { return os_ ? *os_ : std::cout; }
  void reset_power_counters() {}
  /* member forms of the declaration API (definitions at the end) */
  struct ops_block_core *decl_block(int dims, char const *name);
  struct ops_stencil_core *decl_stencil(int dims, int points, int *sten, char const *name);
  struct ops_stencil_core *decl_strided_stencil(int dims, int points, int *sten, int *stride,
                                                char const *name);
  struct ops_stencil_core *decl_restrict_stencil(int dims, int points, int *sten, int *stride,
                                                 char const *name);
  struct ops_stencil_core *decl_prolong_stencil(int dims, int points, int *sten, int *stride,
                                                char const *name);
  struct ops_halo_core *decl_halo(struct ops_dat_core *from, struct ops_dat_core *to,
                                  int *iter_size, int *from_base, int *to_base, int *from_dir,
                                  int *to_dir);
  struct ops_halo_group_core *decl_halo_group(int nhalos, struct ops_halo_core **halos);
  struct ops_reduction_core *decl_reduction_handle(int size, char const *type, char const *name);
  template <class T> void decl_const(char const *name, int dim, char const *type, T *data);
  template <class T> void update_const(char const *name, int dim, char const *type, T *data);
  void partition(char const *routine);
  void diagnostic_output();
  void timing_output(std::ostream &stream);
};

/* ---------------------------------------------------------------------------
 * Exceptions: same class name, code member and stream-append behaviour as
 * the reference (ops_exceptions.h:57-130).
 * ------------------------------------------------------------------------- */
struct OPSException : public std::exception {
  int code;
  std::stringstream msg;
  mutable std::string text;
  explicit OPSException(int c) : code(c) {}
  OPSException(int c, const char *m) : code(c) { msg << m; }
  OPSException(const OPSException &o) : std::exception(), code(o.code) { msg << o.msg.str(); }
  template <class T> OPSException &operator<<(const T &v) { msg << v; return *this; }
  const char *what() const throw() { text = msg.str(); return text.c_str(); }
  virtual ~OPSException() throw() {}
};
#endif

/* ---------------------------------------------------------------------------
 * C API (exported with C linkage from libops_b200.so)
 * ------------------------------------------------------------------------- */
/* ops_lib_core.h:602 */
OPS_API void ops_init(const int argc, const char *const argv[], const int diags_level);
/* ops_lib_core.h:608 */
OPS_API void ops_exit(void);
OPS_API void ops_set_soa(const int soa_val);
/* ops_lib_core.h:618 */
OPS_API ops_block ops_decl_block(int dims, const char *name);
/* ops_internal1.h:92 */
OPS_API ops_dat ops_decl_dat_char(ops_block block, int dim, int *size, int *base, int *d_m,
                                  int *d_p, int *stride, char *data, int type_size,
                                  char const *type, char const *name);
OPS_API void ops_free_dat(ops_dat dat);
OPS_API ops_dat ops_dat_copy(ops_dat orig_dat);
OPS_API void ops_dat_deep_copy(ops_dat target, ops_dat orig_dat);
/* ops_lib_core.h:733-793 */
OPS_API ops_arg ops_arg_dat(ops_dat dat, int dim, ops_stencil stencil, char const *type,
                            ops_access acc);
OPS_API ops_arg ops_arg_dat_opt(ops_dat dat, int dim, ops_stencil stencil, char const *type,
                                ops_access acc, int flag);
OPS_API ops_arg ops_arg_idx(void);
OPS_API ops_arg ops_arg_reduce(ops_reduction handle, int dim, const char *type, ops_access acc);
OPS_API ops_arg ops_arg_gbl_char(char *data, int dim, int size, ops_access acc);
/* ops_lib_core.h:812-888 */
OPS_API ops_reduction ops_decl_reduction_handle(int size, const char *type, const char *name);
OPS_API ops_stencil ops_decl_stencil(int dims, int points, int *stencil, char const *name);
OPS_API ops_stencil ops_decl_strided_stencil(int dims, int points, int *sten, int *stride,
                                             char const *name);
OPS_API ops_stencil ops_decl_restrict_stencil(int dims, int points, int *sten, int *stride,
                                              char const *name);
OPS_API ops_stencil ops_decl_prolong_stencil(int dims, int points, int *sten, int *stride,
                                             char const *name);
OPS_API ops_halo ops_decl_halo(ops_dat from, ops_dat to, int *iter_size, int *from_base,
                               int *to_base, int *from_dir, int *to_dir);
OPS_API ops_halo_group ops_decl_halo_group(int nhalos, ops_halo *halos);
/* ops_lib_core.h:911 */
OPS_API void ops_halo_transfer(ops_halo_group group);
/* ops_internal1.h:95 */
OPS_API void ops_reduction_result_char(ops_reduction handle, int type_size, char *ptr);
/* ops_internal1.h:94 */
OPS_API void ops_decl_const_char(OPS_instance *instance, int dim, char const *type,
                                 int type_size, char *data, char const *name);
/* ops_internal2.h:287 */
#ifdef __cplusplus
OPS_API void ops_execute(OPS_instance *instance = NULL);
#else
OPS_API void ops_execute(OPS_instance *instance);
#endif
OPS_API void ops_printf(const char *format, ...);
OPS_API void ops_fprintf(FILE *stream, const char *format, ...);
OPS_API void ops_diagnostic_output(void);
OPS_API void ops_timing_output_stdout(void);
/* Writes the timing table into buf (NUL-terminated, truncated to n bytes);
 * returns the full length. */
OPS_API size_t ops_timing_output_str(char *buf, size_t n);
OPS_API void ops_timers_core(double *cpu, double *et);
OPS_API void ops_timers(double *cpu, double *et);
OPS_API void ops_print_dat_to_txtfile(ops_dat dat, const char *file_name);
OPS_API void ops_get_data(ops_dat dat);
OPS_API void ops_put_data(ops_dat dat);
OPS_API int ops_is_root(void);
/* process rank and count (ops_dummy_singlenode.cpp:200-202: 0 and 1) */
OPS_API int ops_get_proc(void);
OPS_API int ops_num_procs(void);
/* Stops the program (exit status 2) with the index of the first NaN in a
 * float or double dat (ops_internal2.h:219, ops_dummy_singlenode.cpp:871-878;
 * the search runs on the device). */
OPS_API void ops_NaNcheck(ops_dat dat);
OPS_API void ops_partition(const char *routine);
/* External access (ops_lib_core.h:1092-1296) */
OPS_API int ops_dat_get_local_npartitions(ops_dat dat);
OPS_API int ops_dat_get_global_npartitions(ops_dat dat);
OPS_API void ops_dat_get_extents(ops_dat dat, int part, int *disp, int *size);
OPS_API size_t ops_dat_get_slab_extents(ops_dat dat, int part, int *disp, int *size, int *slab);
OPS_API void ops_dat_get_raw_metadata(ops_dat dat, int part, int *disp, int *size, int *stride,
                                      int *d_m, int *d_p);
OPS_API char *ops_dat_get_raw_pointer(ops_dat dat, int part, ops_stencil stencil,
                                      ops_memspace *memspace);
OPS_API void ops_dat_release_raw_data(ops_dat dat, int part, ops_access acc);
OPS_API void ops_dat_release_raw_data_memspace(ops_dat dat, int part, ops_access acc,
                                               ops_memspace *memspace);
OPS_API void ops_dat_fetch_data(ops_dat dat, int part, char *data);
OPS_API void ops_dat_fetch_data_memspace(ops_dat dat, int part, char *data, ops_memspace memspace);
OPS_API void ops_dat_fetch_data_slab_memspace(ops_dat dat, int part, char *data, int *range,
                                              ops_memspace memspace);
OPS_API void ops_dat_set_data(ops_dat dat, int part, char *data);
OPS_API void ops_dat_set_data_memspace(ops_dat dat, int part, char *data, ops_memspace memspace);
OPS_API void ops_dat_set_data_slab_memspace(ops_dat dat, int part, char *data, int *range,
                                            ops_memspace memspace);
/* random fills (ops_lib_core.h:1302-1308) */
OPS_API void ops_randomgen_init(unsigned int seed, int options);
OPS_API void ops_fill_random_uniform(ops_dat dat);
OPS_API void ops_fill_random_normal(ops_dat dat);
OPS_API void ops_randomgen_exit(void);
/* checkpointing is not provided (needs HDF5); returns false like the
 * reference's no-HDF5 build (ops_checkpointing.h:64-100). */
enum {
  OPS_CHECKPOINT_INITPHASE = 1,
  OPS_CHECKPOINT_MANUAL_DATLIST = 2,
  OPS_CHECKPOINT_FASTFW = 4,
  OPS_CHECKPOINT_MANUAL = 8
};
#ifdef __cplusplus
OPS_API bool ops_checkpointing_init(const char *filename, double interval, int options);
/* the rest of the checkpointing API as in the reference's build without
 * checkpointing (ops_checkpointing.cpp, #else branch): no data is saved,
 * "fast forward" never happens, every loop runs */
OPS_API bool ops_checkpointing_before(ops_arg *args, int nargs, int *range, int loop_id);
OPS_API bool ops_checkpointing_name_before(ops_arg *args, int nargs, int *range,
                                           const char *s);
OPS_API void ops_checkpointing_manual_datlist(int ndats, ops_dat *datlist);
OPS_API bool ops_checkpointing_fastfw(int nbytes, char *payload);
OPS_API bool ops_checkpointing_manual_datlist_fastfw(int ndats, ops_dat *datlist, int nbytes,
                                                     char *payload);
OPS_API bool ops_checkpointing_manual_datlist_fastfw_trigger(int ndats, ops_dat *datlist,
                                                             int nbytes, char *payload);
#endif
/* HDF5 output (ops_hdf5.h:130-166): this backend has no HDF5; the calls
 * report that on stderr and write nothing. */
OPS_API void ops_fetch_dat_hdf5_file(ops_dat dat, char const *file_name);
OPS_API void ops_fetch_block_hdf5_file(ops_block block, char const *file_name);
OPS_API void ops_fetch_stencil_hdf5_file(ops_stencil stencil, char const *file_name);
OPS_API void ops_fetch_halo_hdf5_file(ops_halo halo, char const *file_name);
/* checked allocators used by apps (ops_util.h:41-45): abort on failure */
OPS_API void *xmalloc(size_t size);
OPS_API void *xrealloc(void *ptr, size_t size);
OPS_API void *xcalloc(size_t number, size_t size);
OPS_API void ops_print_dat_to_txtfile_core(ops_dat dat, const char *file_name);
OPS_API void ops_checkpointing_initphase_done(void);
/* energy counters (ops_lib_core.h:1334-1336): no NVML in this backend */
OPS_API void ops_reset_gpu_power_counters(void);
OPS_API double ops_get_gpu_energy_consumed(void);

/* ---------------------------------------------------------------------------
 * C++ conveniences: templates over the C entry points
 * ------------------------------------------------------------------------- */
#ifdef __cplusplus
inline void ops_timing_output(std::ostream &stream) {
  size_t n = ops_timing_output_str(NULL, 0);
  std::string s(n + 1, '\0');
  ops_timing_output_str(&s[0], n + 1);
  s.resize(n);
  stream << s;
}
OPS_API void ops_partition_opts_c(const char *routine);
inline void ops_partition_opts(const char *routine, std::map<std::string, void *> &) {
  ops_partition_opts_c(routine);
}

inline int type_error(const double *, const char *t) { return strcmp(t, "double"); }
inline int type_error(const float *, const char *t) { return strcmp(t, "float"); }
inline int type_error(const int *, const char *t) { return strcmp(t, "int"); }
inline int type_error(const uint *, const char *t) {
  return !(strcmp(t, "uint") == 0 || strcmp(t, "unsigned int") == 0);
}
inline int type_error(const long *, const char *t) { return strcmp(t, "long"); }
inline int type_error(const short *, const char *t) { return strcmp(t, "short"); }
inline int type_error(const char *, const char *t) { return strcmp(t, "char"); }
inline int type_error(const ll *, const char *t) {
  return !(strcmp(t, "ll") == 0 || strcmp(t, "long long") == 0);
}
inline int type_error(const ull *, const char *t) {
  return !(strcmp(t, "ull") == 0 || strcmp(t, "unsigned long long") == 0);
}
inline int type_error(const bool *, const char *t) { return strcmp(t, "bool"); }
inline int type_error(const half *, const char *t) { return strcmp(t, "half"); }
inline int type_error(const complexd *, const char *t) { return strcmp(t, "complexd"); }
inline int type_error(const complexf *, const char *t) { return strcmp(t, "complexf"); }

/* ops_lib_core.h:648-694 */
template <class T>
ops_dat ops_decl_dat(ops_block block, int dim, int *size, int *base, int *d_m, int *d_p,
                     int *stride, T *data, char const *type, char const *name) {
  if (type_error(data, type)) {
    OPSException ex(OPS_HDF5_ERROR);
    ex << "Error: incorrect type specified for dataset " << name;
    throw ex;
  }
  return ops_decl_dat_char(block, dim, size, base, d_m, d_p, stride, (char *)data,
                           (int)sizeof(T), type, name);
}
template <class T>
ops_dat ops_decl_dat(ops_block block, int dim, int *size, int *base, int *d_m, int *d_p,
                     T *data, char const *type, char const *name) {
  if (type_error(data, type)) {
    OPSException ex(OPS_HDF5_ERROR);
    ex << "Error: incorrect type specified for dataset " << name;
    throw ex;
  }
  int stride[OPS_MAX_DIM] = {1, 1, 1, 1, 1};
  return ops_decl_dat_char(block, dim, size, base, d_m, d_p, stride, (char *)data,
                           (int)sizeof(T), type, name);
}

/* ops_lib_core.h:793-797 */
template <class T> ops_arg ops_arg_gbl(T *data, int dim, char const *, ops_access acc) {
  return ops_arg_gbl_char((char *)data, dim, (int)sizeof(T), acc);
}
template <class T> ops_arg ops_arg_gbl(const T *data, int dim, char const *, ops_access acc) {
  return ops_arg_gbl_char((char *)data, dim, (int)sizeof(T), acc);
}

/* ops_lib_core.h:922-932 */
template <class T> void ops_reduction_result(ops_reduction handle, T *ptr) {
  if (type_error(ptr, handle->type)) {
    OPSException ex(OPS_HDF5_ERROR);
    ex << "Error: incorrect type specified for constant " << handle->name
       << " in ops_reduction_result";
    throw ex;
  }
  if (!handle->initialized) {
    OPSException ex(OPS_INVALID_ARGUMENT);
    ex << "Error: ops_reduction_result called for " << handle->name
       << " but the handle was not previously used in a reduction since the last "
          "ops_reduction_result call.";
    throw ex;
  }
  ops_reduction_result_char(handle, (int)sizeof(T), (char *)ptr);
}

/* ops_lib_core.h:944-978; ops_internal2.h:452-456.  User struct types need a
 * type_error overload of their own, as in the reference. */
template <class T> void ops_decl_const2(char const *name, int dim, char const *type, T *data) {
  ops_decl_const_char(OPS_instance::getOPSInstance(), dim, type, (int)sizeof(T), (char *)data,
                      name);
}
template <class T> void ops_decl_const(char const *name, int dim, char const *type, T *data) {
  if (type_error(data, type)) {
    OPSException ex(OPS_HDF5_ERROR);
    ex << "Error: incorrect type specified for constant " << name << " in ops_decl_const";
    throw ex;
  }
  ops_decl_const2(name, dim, type, data);
}
template <class T> void ops_update_const(char const *name, int dim, char const *type, T *data) {
  if (type_error(data, type)) {
    OPSException ex(OPS_HDF5_ERROR);
    ex << "Error: incorrect type specified for constant " << name << " in ops_update_const";
    throw ex;
  }
  ops_decl_const2(name, dim, type, data);
}
#endif /* __cplusplus */

/* ---------------------------------------------------------------------------
 * Helper macros used by user kernels (ops_lib_core.h:556-570)
 * ------------------------------------------------------------------------- */
#ifndef MIN
#define MIN(a, b) ((a < b) ? (a) : (b))
#endif
#ifndef MIN3
#define MIN3(a, b, c) MIN(a, MIN(b, c))
#endif
#ifndef MAX
#define MAX(a, b) ((a > b) ? (a) : (b))
#endif
#ifndef MAX3
#define MAX3(a, b, c) MAX(a, MAX(b, c))
#endif
#ifndef SIGN
#define SIGN(a, b) ((b < 0.0) ? (a * (-1)) : (a))
#endif

/* ---------------------------------------------------------------------------
 * ACC<T>: the per-point accessor handed to user kernels.
 *
 * Same call forms as the reference accessor (ops_lib_core.h:1357-2038):
 * offsets relative to the current point, and a leading component index for
 * multi-component dats.  The representation is this backend's own: a pointer
 * to the current point plus element strides per axis, so the same object
 * serves AoS and SoA layouts and strided (multigrid / low-dim) dats.
 * ------------------------------------------------------------------------- */
#ifdef __cplusplus
#ifdef __CUDA_ARCH__
/* atomic min / max by compare-and-swap (floating point has no native one) */
template <typename T> __device__ __forceinline__ void ob2_atomic_minmax(T *a, T v, bool is_min) {
  static_assert(sizeof(T) == 8 || sizeof(T) == 4, "8- or 4-byte types only");
  typedef typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned int>::type U;
  U *ua = (U *)a;
  U old = *ua, assumed;
  do {
    assumed = old;
    T cur;
    memcpy(&cur, &assumed, sizeof(T));
    if (is_min ? !(v < cur) : !(v > cur)) return;
    U nv;
    memcpy(&nv, &v, sizeof(T));
    old = atomicCAS(ua, assumed, nv);
  } while (old != assumed);
}
#endif
template <typename T> class ACC {
 public:
  T *p;      /* component 0 of the current point */
  int sx;    /* elements between neighbouring x points */
  int sy;    /* elements between neighbouring y points */
  int sz;    /* elements between neighbouring z points */
  int sd;    /* elements between components */
  int su;    /* elements between neighbouring points along the 4th axis */
  int sv;    /* elements between neighbouring points along the 5th axis */

  __host__ __device__ __forceinline__ ACC() : p(0), sx(1), sy(0), sz(0), sd(1), su(0), sv(0) {}
  __host__ __device__ __forceinline__ ACC(T *ptr, int sx_, int sy_, int sz_, int sd_)
      : p(ptr), sx(sx_), sy(sy_), sz(sz_), sd(sd_), su(0), sv(0) {}
  __host__ __device__ __forceinline__ ACC(T *ptr, int sx_, int sy_, int sz_, int su_, int sv_,
                                          int sd_)
      : p(ptr), sx(sx_), sy(sy_), sz(sz_), sd(sd_), su(su_), sv(sv_) {}
  __host__ __device__ __forceinline__ void next(long elems) { p += elems; }

  /* accumulation into shared points (low-dim dats): atomic on the device */
  __host__ __device__ __forceinline__ static void acc_inc(T *a, T v) {
#ifdef __CUDA_ARCH__
    atomicAdd(a, v);
#else
    *a += v;
#endif
  }
  __host__ __device__ __forceinline__ static void acc_min(T *a, T v) {
#ifdef __CUDA_ARCH__
    ob2_atomic_minmax(a, v, true);
#else
    if (v < *a) *a = v;
#endif
  }
  __host__ __device__ __forceinline__ static void acc_max(T *a, T v) {
#ifdef __CUDA_ARCH__
    ob2_atomic_minmax(a, v, false);
#else
    if (v > *a) *a = v;
#endif
  }

#if defined(OPS_5D)
  __host__ __device__ __forceinline__ void combine_inc(int x, int y, int z, int u, int w, T v) const {
    acc_inc(&p[x * sx + y * sy + z * sz + u * su + w * sv], v);
  }
  __host__ __device__ __forceinline__ void combine_min(int x, int y, int z, int u, int w, T v) const {
    acc_min(&p[x * sx + y * sy + z * sz + u * su + w * sv], v);
  }
  __host__ __device__ __forceinline__ void combine_max(int x, int y, int z, int u, int w, T v) const {
    acc_max(&p[x * sx + y * sy + z * sz + u * su + w * sv], v);
  }
#elif defined(OPS_4D)
  __host__ __device__ __forceinline__ void combine_inc(int x, int y, int z, int u, T v) const {
    acc_inc(&p[x * sx + y * sy + z * sz + u * su], v);
  }
  __host__ __device__ __forceinline__ void combine_min(int x, int y, int z, int u, T v) const {
    acc_min(&p[x * sx + y * sy + z * sz + u * su], v);
  }
  __host__ __device__ __forceinline__ void combine_max(int x, int y, int z, int u, T v) const {
    acc_max(&p[x * sx + y * sy + z * sz + u * su], v);
  }
#elif defined(OPS_1D)
  __host__ __device__ __forceinline__ void combine_inc(int x, T v) const { acc_inc(&p[x * sx], v); }
  __host__ __device__ __forceinline__ void combine_min(int x, T v) const { acc_min(&p[x * sx], v); }
  __host__ __device__ __forceinline__ void combine_max(int x, T v) const { acc_max(&p[x * sx], v); }
#elif defined(OPS_3D)
  __host__ __device__ __forceinline__ void combine_inc(int x, int y, int z, T v) const {
    acc_inc(&p[x * sx + y * sy + z * sz], v);
  }
  __host__ __device__ __forceinline__ void combine_min(int x, int y, int z, T v) const {
    acc_min(&p[x * sx + y * sy + z * sz], v);
  }
  __host__ __device__ __forceinline__ void combine_max(int x, int y, int z, T v) const {
    acc_max(&p[x * sx + y * sy + z * sz], v);
  }
#else
  __host__ __device__ __forceinline__ void combine_inc(int x, int y, T v) const {
    acc_inc(&p[x * sx + y * sy], v);
  }
  __host__ __device__ __forceinline__ void combine_min(int x, int y, T v) const {
    acc_min(&p[x * sx + y * sy], v);
  }
  __host__ __device__ __forceinline__ void combine_max(int x, int y, T v) const {
    acc_max(&p[x * sx + y * sy], v);
  }
#endif

#if defined(OPS_5D)
  __host__ __device__ __forceinline__ T &operator()(int x, int y, int z, int u, int w) const {
    return p[x * sx + y * sy + z * sz + u * su + w * sv];
  }
  __host__ __device__ __forceinline__ T &operator()(int d, int x, int y, int z, int u,
                                                    int w) const {
    return p[d * sd + x * sx + y * sy + z * sz + u * su + w * sv];
  }
#elif defined(OPS_4D)
  __host__ __device__ __forceinline__ T &operator()(int x, int y, int z, int u) const {
    return p[x * sx + y * sy + z * sz + u * su];
  }
  __host__ __device__ __forceinline__ T &operator()(int d, int x, int y, int z, int u) const {
    return p[d * sd + x * sx + y * sy + z * sz + u * su];
  }
#elif defined(OPS_1D)
  __host__ __device__ __forceinline__ T &operator()(int x) const { return p[x * sx]; }
  __host__ __device__ __forceinline__ T &operator()(int d, int x) const {
    return p[d * sd + x * sx];
  }
#elif defined(OPS_3D)
  __host__ __device__ __forceinline__ T &operator()(int x, int y, int z) const {
    return p[x * sx + y * sy + z * sz];
  }
  __host__ __device__ __forceinline__ T &operator()(int d, int x, int y, int z) const {
    return p[d * sd + x * sx + y * sy + z * sz];
  }
#else /* OPS_2D is the default */
  __host__ __device__ __forceinline__ T &operator()(int x, int y) const {
    return p[x * sx + y * sy];
  }
  __host__ __device__ __forceinline__ T &operator()(int d, int x, int y) const {
    return p[d * sd + x * sx + y * sy];
  }
#endif
};

/* ---------------------------------------------------------------------------
 * C++ object API: member forms of the C entry points (no counterpart in the
 * C API; the reference's OPS_CPP_API methods, ops_lib_core.h:190-560).
 * ------------------------------------------------------------------------- */
/* Makes `inst` the library's instance and runs ops_init (the constructor of
 * OPS_instance); ob2_release_instance runs ops_exit if `inst` is that
 * instance (its destructor).  No counterpart in the reference's C API. */
OPS_API void ob2_adopt_instance(OPS_instance *inst, int argc, const char *const *argv,
                                int diags);
OPS_API void ob2_release_instance(OPS_instance *inst);

inline OPS_instance::OPS_instance(const int argc, const char *const argv[], const int diags,
                                  std::ostream &os)
    : OPS_soa(0), OPS_diags(diags), OPS_hybrid_gpu(1), backend(NULL), os_(&os) {
  ob2_adopt_instance(this, argc, argv, diags);
}
inline OPS_instance::~OPS_instance() { ob2_release_instance(this); }
inline ops_block OPS_instance::decl_block(int dims, char const *name) {
  return ops_decl_block(dims, name);
}
inline ops_stencil OPS_instance::decl_stencil(int dims, int points, int *sten,
                                              char const *name) {
  return ops_decl_stencil(dims, points, sten, name);
}
inline ops_stencil OPS_instance::decl_strided_stencil(int dims, int points, int *sten,
                                                      int *stride, char const *name) {
  return ops_decl_strided_stencil(dims, points, sten, stride, name);
}
inline ops_stencil OPS_instance::decl_restrict_stencil(int dims, int points, int *sten,
                                                       int *stride, char const *name) {
  return ops_decl_restrict_stencil(dims, points, sten, stride, name);
}
inline ops_stencil OPS_instance::decl_prolong_stencil(int dims, int points, int *sten,
                                                      int *stride, char const *name) {
  return ops_decl_prolong_stencil(dims, points, sten, stride, name);
}
inline ops_halo OPS_instance::decl_halo(ops_dat from, ops_dat to, int *iter_size,
                                        int *from_base, int *to_base, int *from_dir,
                                        int *to_dir) {
  return ops_decl_halo(from, to, iter_size, from_base, to_base, from_dir, to_dir);
}
inline ops_halo_group OPS_instance::decl_halo_group(int nhalos, ops_halo *halos) {
  return ops_decl_halo_group(nhalos, halos);
}
inline ops_reduction OPS_instance::decl_reduction_handle(int size, char const *type,
                                                         char const *name) {
  return ops_decl_reduction_handle(size, type, name);
}
template <class T>
void OPS_instance::decl_const(char const *name, int dim, char const *type, T *data) {
  ops_decl_const(name, dim, type, data);
}
template <class T>
void OPS_instance::update_const(char const *name, int dim, char const *type, T *data) {
  ops_update_const(name, dim, type, data);
}
inline void OPS_instance::partition(char const *routine) { ops_partition(routine); }
inline void OPS_instance::diagnostic_output() { ops_diagnostic_output(); }
inline void OPS_instance::timing_output(std::ostream &stream) { ops_timing_output(stream); }
template <class T>
ops_dat ops_block_core::decl_dat(int data_size, int *block_size, int *base, int *d_m,
                                 int *d_p, T *data, char const *type, char const *name) {
  return ops_decl_dat(this, data_size, block_size, base, d_m, d_p, data, type, name);
}
template <class T>
ops_dat ops_block_core::decl_dat(int data_size, int *block_size, int *base, int *d_m,
                                 int *d_p, int *stride, T *data, char const *type,
                                 char const *name) {
  return ops_decl_dat(this, data_size, block_size, base, d_m, d_p, stride, data, type, name);
}
inline void ops_halo_group_core::halo_transfer() { ops_halo_transfer(this); }
template <class T> void ops_reduction_core::get_result(T *ptr) {
  ops_reduction_result(this, ptr);
}
#endif /* __cplusplus */

#endif /* OPS_B200_LIB_CORE_H */
