/*
 * ORACLE -- test infrastructure only (never linked into the product).
 *
 * Host-memory restatement of the OPS single-node sequential runtime, enough to
 * run OPS apps through oracle/include/ops_seq_v2.h.  Each function names the
 * reference code it restates (paths inside the OPS tree).
 *
 * Layout: every dat is one dense host array, x fastest, halos included,
 * size[i] = block_size[i] - d_m[i] + d_p[i] (size 1 stays 1 and marks an edge
 * dat).  Unlike the reference sequential backend there is no x padding to a
 * SIMD multiple (ops_host_singlenode.cpp:66-73); that padding is invisible
 * through ops_dat_fetch_data and the dump hook, which is how results are
 * compared.
 */
#include <string.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <limits>
#include <string>
#include <vector>

#include "ops_b200_dist.h"
#include "ops_lib_core.h"
#include "ops_tridiag.h"

namespace {

struct KernelStat {
  std::string name;
  long count = 0;
  double time = 0.0;
  double transfer = 0.0;
};

struct DistDat {  // the rows a rank holds (see ops_b200_dist.h)
  bool split = false;
  char *alloc = nullptr;
  size_t row_bytes = 0;
  int axis = -1, s_lo = 0, s_hi = 0, o_lo = 0, o_hi = 0, H = 0;
  bool dirty = false;
};

struct OracleState {
  ob2_dist_comm comm = {0, 1, 0, nullptr, nullptr, nullptr};
  bool dist = false;
  std::vector<std::array<int, 5>> bpart;  // per block: G, lo, hi, first, last
  std::vector<DistDat> dd;
  OPS_instance inst;
  std::vector<ops_block> blocks;
  std::vector<ops_dat> dats;
  std::vector<ops_stencil> stencils;
  std::vector<ops_halo> halos;
  std::vector<ops_halo_group> groups;
  std::vector<ops_reduction> reds;
  std::vector<int> edat_prev_acc;
  std::vector<KernelStat> stats;
  double loop_t0 = 0.0;
  unsigned long long rng_seed = 0;
  unsigned long long rng_counter = 0;
};

OracleState *S = nullptr;

OracleState &st() {
  if (!S) {
    S = new OracleState();
    memset(&S->inst, 0, sizeof(S->inst));
  }
  return *S;
}

char *copy_str(const char *s) {
  if (!s) return nullptr;
  size_t n = strlen(s);
  char *r = (char *)malloc(n + 1);
  memcpy(r, s, n + 1);
  return r;
}

double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

size_t dat_points(ops_dat d) {
  size_t n = 1;
  for (int i = 0; i < d->block->dims; i++) n *= (size_t)d->size[i];
  return n;
}

/* element pointer of storage coordinates (s0..s4) and component c */
char *elem_ptr(ops_dat d, const int *s, int c) {
  size_t lin = 0, cum = 1;
  for (int i = 0; i < OPS_MAX_DIM; i++) {
    lin += cum * (size_t)s[i];
    cum *= (size_t)d->size[i];
  }
  if (st().inst.OPS_soa) return d->data + (lin + cum * (size_t)c) * d->type_size;
  return d->data + lin * d->elem_size + (size_t)c * d->type_size;
}

template <typename T> void fill_identity(ops_dat d, int acc) {
  T v = 0;
  if (acc == OPS_MAX) v = std::numeric_limits<T>::lowest();
  if (acc == OPS_MIN) v = std::numeric_limits<T>::max();
  std::fill((T *)d->data, (T *)d->data + d->mem / sizeof(T), v);
}

} // namespace

OPS_instance *OPS_instance::getOPSInstance() { return &st().inst; }

/* ---- init / exit (ops_lib_core.cpp:267-275; flags :100-249) ---- */
static bool dist_layout(ops_dat d, DistDat &x);
static void dist_unsupported(ops_dat d, const char *what);

OPS_API void ops_init(const int argc, const char *const argv[], const int diags) {
  OracleState &s = st();
  s.inst.OPS_diags = diags;
  for (int i = 0; i < argc; i++) {
    if (!argv || !argv[i]) continue;
    const char *p = strstr(argv[i], "-OPS_DIAGS=");
    if (p) s.inst.OPS_diags = atoi(p + 11);
  }
}

OPS_API int oracle_soa(void) { return st().inst.OPS_soa; }
OPS_API void ops_set_soa(const int soa) { st().inst.OPS_soa = soa; }

OPS_API void ops_dump_dats(const char *path);

OPS_API void ops_exit(void) {
  const char *dump = getenv("OPS_DUMP_FILE");
  if (dump && *dump) ops_dump_dats(dump);
}

OPS_API ops_block ops_decl_block(int dims, const char *name) {
  if (dims < 1 || dims > OPS_MAX_DIM)
    throw OPSException(OPS_INVALID_ARGUMENT, "Error: ops_decl_block -- dims must be 1..5");
  ops_block b = (ops_block)calloc(1, sizeof(ops_block_core));
  b->dims = dims;
  b->name = copy_str(name);
  b->instance = &st().inst;
  b->index = (int)st().blocks.size();
  st().blocks.push_back(b);
  return b;
}

/* ops_lib_core.cpp:445-540 (metadata) + ops_host_singlenode.cpp:42-106 */
OPS_API ops_dat ops_decl_dat_char(ops_block block, int dim, int *size, int *base, int *d_m,
                                  int *d_p, int *stride, char *data, int type_size,
                                  char const *type, char const *name) {
  if (dim <= 0) {
    OPSException ex(OPS_INVALID_ARGUMENT);
    ex << "Error: ops_decl_dat -- negative/zero number of items per grid point in dataset: "
       << name;
    throw ex;
  }
  ops_dat d = (ops_dat)calloc(1, sizeof(ops_dat_core));
  d->block = block;
  d->dim = dim;
  d->type_size = type_size;
  d->elem_size = dim * type_size;
  for (int n = 0; n < OPS_MAX_DIM; n++) {
    d->size[n] = 1;
    d->stride[n] = 1;
  }
  for (int n = 0; n < block->dims; n++) {
    if (d_m[n] > 0 || d_p[n] < 0) {
      OPSException ex(OPS_INVALID_ARGUMENT);
      ex << "Error: ops_decl_dat -- invalid halo depth during declaration of: " << name;
      throw ex;
    }
    if (size[n] != 1) {
      d->size[n] = size[n] - d_m[n] + d_p[n];
      d->base[n] = base[n];
    } else {
      d->size[n] = 1;
      d->e_dat = 1;
      d->base[n] = 0;
    }
    d->d_m[n] = d_m[n];
    d->d_p[n] = d_p[n];
    d->stride[n] = stride ? stride[n] : 1;
  }
  d->type = copy_str(type);
  d->name = copy_str(name);
  d->mem = (size_t)d->elem_size * dat_points(d);
  DistDat x;
  if (dist_layout(d, x)) {  // this rank's rows; d->data addresses them by global index
    x.alloc = (char *)calloc((size_t)(x.s_hi - x.s_lo) * x.row_bytes + 1, 1);
    if (data)
      memcpy(x.alloc, data + (size_t)x.s_lo * x.row_bytes, (size_t)(x.s_hi - x.s_lo) * x.row_bytes);
    d->data = x.alloc - (size_t)x.s_lo * x.row_bytes;
    d->user_managed = 0;
  } else if (data) {
    d->data = data;
    d->user_managed = 1;
  } else {
    d->data = (char *)calloc(d->mem ? d->mem : 1, 1);
    d->user_managed = 0;
  }
  size_t cum = 1;
  long long off = 0;
  for (int i = 0; i < block->dims; i++) {
    off += (long long)(st().inst.OPS_soa ? d->type_size : d->elem_size) * (long long)cum *
           (-d->base[i] - d->d_m[i]);
    cum *= d->size[i];
  }
  d->base_offset = (size_t)off;
  d->dirty_hd = 0;
  d->index = (int)st().dats.size();
  st().dats.push_back(d);
  st().edat_prev_acc.push_back(-1);
  st().dd.push_back(x);
  return d;
}

OPS_API void ops_free_dat(ops_dat d) {
  if (!d) return;
  for (auto &p : st().dats)
    if (p == d) p = nullptr;
  const DistDat &x = st().dd[d->index];
  if (x.split)
    free(x.alloc);
  else if (!d->user_managed)
    free(d->data);
  free(d);
}

OPS_API void ops_dat_deep_copy(ops_dat target, ops_dat src) {
  if (target->mem != src->mem || target->data == nullptr) {
    if (target->data && !target->user_managed) free(target->data);
    target->data = (char *)malloc(src->mem ? src->mem : 1);
    target->user_managed = 0;
  }
  char *keep = target->data;
  int idx = target->index;
  int um = target->user_managed;
  ops_block blk = target->block;
  memcpy(target, src, sizeof(ops_dat_core));
  target->data = keep;
  target->index = idx;
  target->user_managed = um;
  target->block = blk ? blk : src->block;
  // the copy is renamed to the source name + "_copy", cut to strlen(name) + 4
  // characters as in ops_lib_core.cpp:2280-2281 (so "u" becomes "u_cop")
  {
    size_t nl = strlen(src->name) + 5;
    char *nm = (char *)malloc(nl + 1);
    snprintf(nm, nl, "%s_copy", src->name);
    target->name = nm;
  }
  target->type = copy_str(src->type);
  memcpy(target->data, src->data, src->mem);
}

OPS_API ops_dat ops_dat_copy(ops_dat src) {
  ops_dat d = (ops_dat)calloc(1, sizeof(ops_dat_core));
  d->block = src->block;
  d->index = (int)st().dats.size();
  st().dats.push_back(d);
  st().edat_prev_acc.push_back(-1);
  st().dd.push_back(DistDat());
  ops_dat_deep_copy(d, src);
  return d;
}

/* ---- args (ops_lib_core.cpp:1047-1105, 856-965) ---- */
OPS_API ops_arg ops_arg_dat(ops_dat dat, int dim, ops_stencil stencil, char const *,
                            ops_access acc) {
  ops_arg a;
  memset(&a, 0, sizeof(a));
  if (acc == OPS_WRITE && stencil && stencil->points != 1)
    throw OPSException(OPS_INVALID_ARGUMENT,
                       "Error: OPS does not support OPS_WRITE arguments with a non (0,0,0) "
                       "stencil due to potential race conditions");
  a.argtype = OPS_ARG_DAT;
  a.dat = dat;
  a.stencil = stencil;
  a.dim = dim;
  a.acc = acc;
  a.opt = 1;
  if (dat) {
    a.data = dat->data;
    a.elem_size = dat->elem_size;
  }
  return a;
}

OPS_API ops_arg ops_arg_dat_opt(ops_dat dat, int dim, ops_stencil stencil, char const *type,
                                ops_access acc, int flag) {
  ops_arg a = ops_arg_dat(dat, dim, stencil, type, acc);
  a.opt = flag;
  return a;
}

OPS_API ops_arg ops_arg_idx(void) {
  ops_arg a;
  memset(&a, 0, sizeof(a));
  a.argtype = OPS_ARG_IDX;
  return a;
}

OPS_API ops_arg ops_arg_gbl_char(char *data, int dim, int size, ops_access acc) {
  ops_arg a;
  memset(&a, 0, sizeof(a));
  a.argtype = OPS_ARG_GBL;
  a.data = data;
  a.dim = dim;
  a.elem_size = size;
  a.acc = acc;
  return a;
}

template <typename T> static void red_init(ops_reduction h, int acc, bool intlike) {
  T *v = (T *)h->data;
  size_t n = (size_t)h->size / sizeof(T);
  for (size_t i = 0; i < n; i++) {
    if (acc == OPS_MIN) v[i] = std::numeric_limits<T>::max();
    if (acc == OPS_MAX)
      v[i] = intlike ? std::numeric_limits<T>::min() : -std::numeric_limits<T>::max();
  }
}

OPS_API ops_arg ops_arg_reduce(ops_reduction h, int dim, const char *type, ops_access acc) {
  ops_arg a;
  memset(&a, 0, sizeof(a));
  a.argtype = OPS_ARG_GBL;
  a.dim = dim;
  a.data = (char *)h;
  a.acc = acc;
  if (!h->initialized) {
    h->initialized = 1;
    h->acc = acc;
    if (acc == OPS_INC) memset(h->data, 0, h->size);
    if (!strcmp(type, "double"))
      red_init<double>(h, acc, false);
    else if (!strcmp(type, "float"))
      red_init<float>(h, acc, false);
    else if (!strcmp(type, "int"))
      red_init<int>(h, acc, true);
    else if (!strcmp(type, "long long") || !strcmp(type, "ll"))
      red_init<long long>(h, acc, true);
    else if (!strcmp(type, "complexd") || !strcmp(type, "complexf")) {
      // ops_lib_core.cpp:935-952: OPS_MIN starts at (MAX, MAX), others at 0
      const bool dbl = type[7] == 'd';
      const int ts = dbl ? 16 : 8;
      memset(h->data, 0, h->size);
      if (acc == OPS_MIN)
        for (int off = 0; off + ts <= h->size; off += ts) {
          if (dbl)
            *(complexd *)(h->data + off) = INFINITY_complexd;
          else
            *(complexf *)(h->data + off) = INFINITY_complexf;
        }
    } else
      throw OPSException(OPS_NOT_IMPLEMENTED, "Error, reduction type not recognised");
  } else if (h->acc != acc) {
    OPSException ex(OPS_INVALID_ARGUMENT);
    ex << "Error: ops_reduction handle " << h->name
       << " was already used with a different access type";
    throw ex;
  }
  return a;
}

OPS_API ops_reduction ops_decl_reduction_handle(int size, const char *type, const char *name) {
  ops_reduction r = (ops_reduction)calloc(1, sizeof(ops_reduction_core));
  r->size = size;
  r->data = (char *)calloc(size, 1);
  r->type = copy_str(type);
  r->name = copy_str(name);
  r->instance = &st().inst;
  r->index = (int)st().reds.size();
  st().reds.push_back(r);
  return r;
}

OPS_API void ops_reduction_result_char(ops_reduction h, int, char *ptr) {
  if (st().dist) {  // combined over the ranks (the reference's MPI_Allreduce)
    int t = !strcmp(h->type, "double") ? 0 : !strcmp(h->type, "float") ? 1
            : !strcmp(h->type, "int") ? 2 : (!strcmp(h->type, "long long") || !strcmp(h->type, "ll")) ? 3 : -1;
    if (t < 0) throw OPSException(OPS_NOT_IMPLEMENTED, "Error: reduction type over ranks");
    const int ts = t == 0 || t == 3 ? 8 : 4;
    if (st().comm.allreduce(st().comm.ctx, h->data, h->size / ts, t, h->acc))
      throw OPSException(OPS_RUNTIME_ERROR, "Error: reduction over the ranks failed");
  }
  memcpy(ptr, h->data, h->size);
  h->initialized = 0;
}

/* ---- stencils (ops_lib_core.cpp:640-836) ---- */
static ops_stencil make_stencil(int dims, int points, int *sten, int *stride, const char *name,
                                int type) {
  ops_stencil s = (ops_stencil)calloc(1, sizeof(ops_stencil_core));
  s->dims = dims;
  s->points = points;
  s->name = copy_str(name);
  s->stencil = (int *)malloc(sizeof(int) * dims * points);
  memcpy(s->stencil, sten, sizeof(int) * dims * points);
  s->stride = (int *)malloc(sizeof(int) * OPS_MAX_DIM);
  s->mgrid_stride = (int *)malloc(sizeof(int) * OPS_MAX_DIM);
  for (int i = 0; i < OPS_MAX_DIM; i++) {
    s->stride[i] = (stride && i < dims) ? stride[i] : 1;
    s->mgrid_stride[i] = 1;
  }
  s->type = type;
  s->index = (int)st().stencils.size();
  st().stencils.push_back(s);
  return s;
}
OPS_API ops_stencil ops_decl_stencil(int dims, int points, int *sten, char const *name) {
  return make_stencil(dims, points, sten, nullptr, name, 0);
}
OPS_API ops_stencil ops_decl_strided_stencil(int dims, int points, int *sten, int *stride,
                                             char const *name) {
  return make_stencil(dims, points, sten, stride, name, 0);
}
OPS_API ops_stencil ops_decl_restrict_stencil(int, int, int *, int *, char const *) {
  throw OPSException(OPS_NOT_IMPLEMENTED, "Error: restrict stencils are not supported");
}
OPS_API ops_stencil ops_decl_prolong_stencil(int, int, int *, int *, char const *) {
  throw OPSException(OPS_NOT_IMPLEMENTED, "Error: prolong stencils are not supported");
}

/* ---- halos (ops_lib_core.cpp:967-1045) ---- */
OPS_API ops_halo ops_decl_halo(ops_dat from, ops_dat to, int *iter_size, int *from_base,
                               int *to_base, int *from_dir, int *to_dir) {
  ops_halo h = (ops_halo)calloc(1, sizeof(ops_halo_core));
  h->from = from;
  h->to = to;
  for (int i = 0; i < OPS_MAX_DIM; i++) {
    bool used = i < from->block->dims;
    h->iter_size[i] = used ? iter_size[i] : 1;
    h->from_base[i] = used ? from_base[i] : 0;
    h->to_base[i] = used ? to_base[i] : 0;
    h->from_dir[i] = used ? from_dir[i] : i + 1;
    h->to_dir[i] = used ? to_dir[i] : i + 1;
  }
  h->index = (int)st().halos.size();
  st().halos.push_back(h);
  return h;
}

OPS_API ops_halo_group ops_decl_halo_group(int nhalos, ops_halo *halos) {
  ops_halo_group g = (ops_halo_group)calloc(1, sizeof(ops_halo_group_core));
  g->nhalos = nhalos;
  g->halos = (ops_halo *)malloc(sizeof(ops_halo) * (nhalos > 0 ? nhalos : 1));
  for (int i = 0; i < nhalos; i++) g->halos[i] = halos[i];
  g->instance = &st().inst;
  g->index = (int)st().groups.size();
  st().groups.push_back(g);
  return g;
}

/*
 * ops_host_singlenode.cpp:172-446.  Per halo: iterate the box iter_size; the
 * source (target) dat's dimension i walks iteration axis |dir[i]|-1, forward
 * from base[i] for dir>0 and backward (flipped) for dir<0.  Values are copied
 * bit for bit, converted between float and double when the dat types differ.
 */
OPS_API void ops_halo_transfer(ops_halo_group g) {
  if (st().dist) dist_unsupported(nullptr, "ops_halo_transfer between blocks");
  for (int hh = 0; hh < g->nhalos; hh++) {
    ops_halo h = g->halos[hh];
    int n = 1;
    for (int i = 0; i < OPS_MAX_DIM; i++) n *= h->iter_size[i];
    int t[OPS_MAX_DIM];
    for (int lin = 0; lin < n; lin++) {
      int r = lin;
      for (int a = 0; a < OPS_MAX_DIM; a++) {
        t[a] = r % h->iter_size[a];
        r /= h->iter_size[a];
      }
      int fs[OPS_MAX_DIM], ts[OPS_MAX_DIM];
      for (int i = 0; i < OPS_MAX_DIM; i++) {
        int fa = abs(h->from_dir[i]) - 1, ta = abs(h->to_dir[i]) - 1;
        int fo = h->from_dir[i] > 0 ? t[fa] : h->iter_size[fa] - 1 - t[fa];
        int to = h->to_dir[i] > 0 ? t[ta] : h->iter_size[ta] - 1 - t[ta];
        fs[i] = h->from_base[i] - h->from->d_m[i] - h->from->base[i] + fo;
        ts[i] = h->to_base[i] - h->to->d_m[i] - h->to->base[i] + to;
      }
      for (int c = 0; c < h->from->dim; c++) {
        char *src = elem_ptr(h->from, fs, c);
        char *dst = elem_ptr(h->to, ts, c);
        // mixed types: each value converted to the destination type
        // (ops_host_singlenode.cpp:279-300 / 398-420 go through the smaller
        // of the two types, the same value as the direct conversion)
        if (h->from->type_size == h->to->type_size) {
          memcpy(dst, src, h->from->type_size);
        } else {
          double v;
          const int fs2 = h->from->type_size, ts2 = h->to->type_size;
          if (fs2 == 8) v = *(double *)src;
          else if (fs2 == 4) v = (double)*(float *)src;
          else if (fs2 == 2) v = (double)*(half *)src;
          else throw OPSException(OPS_NOT_IMPLEMENTED, "Error: unsupported mixed halo types");
          if (ts2 == 8) *(double *)dst = v;
          else if (ts2 == 4) *(float *)dst = (float)v;
          else if (ts2 == 2) *(half *)dst = (half)v;
          else throw OPSException(OPS_NOT_IMPLEMENTED, "Error: unsupported mixed halo types");
        }
      }
    }
  }
}

/* ---- constants: host kernels read the app's globals directly
 *      (sequential backend, ops_host_common.cpp) ---- */
OPS_API void ops_decl_const_char(OPS_instance *, int, char const *, int, char *, char const *) {}

OPS_API void ops_execute(OPS_instance *) {}

/* ---- slab decomposition over ranks (ops_b200_dist.h): the same layout,
 *      exchanges and clipping as the runtime, on host memory ---- */
OPS_API int ob2_dist_init(const ob2_dist_comm *c) {
  if (!c || c->size < 1 || c->rank < 0 || c->rank >= c->size ||
      (c->size > 1 && (!c->sendrecv || !c->allreduce)) || !st().dats.empty())
    return OPS_INVALID_ARGUMENT;
  st().comm = *c;
  st().dist = c->size > 1;
  return 0;
}
OPS_API int ob2_dist_rank(void) { return st().comm.rank; }
OPS_API int ob2_dist_size(void) { return st().comm.size; }

static void dist_unsupported(ops_dat d, const char *what) {
  OPSException ex(OPS_NOT_IMPLEMENTED);
  ex << "Error: " << what << " (dat " << (d ? d->name : "-")
     << ") is not supported with the slab decomposition over ranks";
  throw ex;
}

static std::array<int, 5> &block_part(ops_block b, int G) {
  OracleState &o = st();
  if ((int)o.bpart.size() <= b->index) o.bpart.resize(b->index + 1, {-1, 0, 0, 0, 0});
  std::array<int, 5> &bp = o.bpart[b->index];
  if (bp[0] < 0 && G > 0) {
    bp[0] = G;
    ob2dist::slab(G, o.comm.size, o.comm.rank, &bp[1], &bp[2]);
    bp[3] = o.comm.rank == 0;
    bp[4] = o.comm.rank == o.comm.size - 1;
    if (bp[2] - bp[1] < 1) throw OPSException(OPS_INVALID_ARGUMENT, "Error: too few rows for the ranks");
  }
  return bp;
}

static bool dist_layout(ops_dat d, DistDat &x) {
  if (!st().dist) return false;
  const int ax = d->block->dims - 1;
  if (ax < 0 || ax > 2 || d->size[ax] == 1) return false;
  if (st().inst.OPS_soa && d->dim > 1) dist_unsupported(d, "a multi-component dat in SoA layout");
  const int n = d->size[ax] + d->d_m[ax] - d->d_p[ax];
  std::array<int, 5> &bp = block_part(d->block, n);
  x.split = true;
  x.axis = ax;
  x.H = std::max(1, std::max(-d->d_m[ax], d->d_p[ax]));
  const int sh = -d->base[ax] - d->d_m[ax];
  x.o_lo = bp[3] ? 0 : bp[1] + sh;
  x.o_hi = bp[4] ? d->size[ax] : std::min(d->size[ax], bp[2] + sh);
  x.s_lo = bp[3] ? 0 : std::max(0, x.o_lo - x.H);
  x.s_hi = bp[4] ? d->size[ax] : std::min(d->size[ax], x.o_hi + x.H);
  if (x.o_hi - x.o_lo < x.H && !(bp[3] && bp[4]))
    dist_unsupported(d, "a slab thinner than the dat's halo depth");
  size_t rb = (size_t)d->elem_size;
  for (int i = 0; i < ax; i++) rb *= (size_t)d->size[i];
  x.row_bytes = rb;
  return true;
}

static void dist_exchange(ops_dat d) {
  OracleState &o = st();
  DistDat &x = o.dd[d->index];
  const int up = o.comm.rank + 1 < o.comm.size ? o.comm.rank + 1 : -1;
  const int dn = o.comm.rank > 0 ? o.comm.rank - 1 : -1;
  const size_t nb = (size_t)x.H * x.row_bytes;
  char *base = d->data;
  int e = o.comm.sendrecv(o.comm.ctx, base + (size_t)(x.o_hi - x.H) * x.row_bytes, up >= 0 ? nb : 0,
                          up, base + (size_t)(x.o_lo - x.H) * x.row_bytes, dn >= 0 ? nb : 0, dn);
  if (!e)
    e = o.comm.sendrecv(o.comm.ctx, base + (size_t)x.o_lo * x.row_bytes, dn >= 0 ? nb : 0, dn,
                        base + (size_t)x.o_hi * x.row_bytes, up >= 0 ? nb : 0, up);
  if (e) throw OPSException(OPS_RUNTIME_ERROR, "Error: slab halo exchange failed");
  x.dirty = false;
}

/* exchanges before the loop and clips its slowest-axis range to this rank */
OPS_API void oracle_dist_loop(const char *name, ops_block block, int dim, int *lo, int *hi,
                              ops_arg *args, int nargs) {
  OracleState &o = st();
  if (!o.dist) return;
  const int ax = dim - 1;
  if (ax < 0 || ax > 2) return;
  for (int i = 0; i < nargs; i++) {
    ops_arg &a = args[i];
    if (a.argtype != OPS_ARG_DAT || !a.dat || a.acc == OPS_WRITE) continue;
    DistDat &x = o.dd[a.dat->index];
    if (!x.split) continue;
    int reach = 0;
    if (a.stencil)
      for (int p = 0; p < a.stencil->points; p++)
        if (ax < a.stencil->dims)
          reach = std::max(reach, std::abs(a.stencil->stencil[p * a.stencil->dims + ax]));
    if (reach > x.H) dist_unsupported(a.dat, "a stencil deeper than the halo along the split axis");
    if (reach > 0 && x.dirty) dist_exchange(a.dat);
  }
  for (int i = 0; i < nargs; i++) {
    ops_arg &a = args[i];
    if (a.argtype == OPS_ARG_DAT && a.dat && a.acc != OPS_READ && o.dd[a.dat->index].split)
      o.dd[a.dat->index].dirty = true;
  }
  const std::array<int, 5> &bp = block_part(block, 0);
  if (bp[0] >= 0) ob2dist::clip(bp[1], bp[2], bp[3], bp[4], &lo[ax], &hi[ax]);
  (void)name;
}

/* ---- par_loop hooks: low-dim accumulation init (ops_dummy_singlenode.cpp:235-391) ---- */
OPS_API void oracle_loop_prologue(const char *, ops_block, int, const int *, ops_arg *args,
                                  int nargs) {
  st().loop_t0 = wall();
  for (int i = 0; i < nargs; i++) {
    ops_arg &a = args[i];
    if (a.argtype != OPS_ARG_DAT || !a.opt || !a.dat) continue;
    ops_dat d = a.dat;
    if (!d->e_dat) continue;
    if ((a.acc == OPS_INC || a.acc == OPS_MIN || a.acc == OPS_MAX) &&
        st().edat_prev_acc[d->index] != a.acc) {
      st().edat_prev_acc[d->index] = a.acc;
      if (!strcmp(d->type, "double"))
        fill_identity<double>(d, a.acc);
      else if (!strcmp(d->type, "float"))
        fill_identity<float>(d, a.acc);
      else if (!strcmp(d->type, "int"))
        fill_identity<int>(d, a.acc);
    }
  }
}

OPS_API void oracle_loop_epilogue(const char *name, ops_block block, int, const int *range,
                                  ops_arg *args, int nargs) {
  double dt = wall() - st().loop_t0;
  KernelStat *k = nullptr;
  for (auto &s : st().stats)
    if (s.name == name) k = &s;
  if (!k) {
    st().stats.push_back(KernelStat());
    k = &st().stats.back();
    k->name = name;
  }
  k->count++;
  k->time += dt;
  size_t pts = 1;
  for (int i = 0; i < block->dims; i++) pts *= (size_t)std::max(0, range[2 * i + 1] - range[2 * i]);
  for (int i = 0; i < nargs; i++) {
    ops_arg &a = args[i];
    if (a.argtype != OPS_ARG_DAT || !a.opt || !a.dat) continue;
    if (a.dat->e_dat && a.acc != OPS_READ) st().edat_prev_acc[a.dat->index] = a.acc;
    if (a.acc == OPS_READ && a.dat->e_dat) st().edat_prev_acc[a.dat->index] = OPS_READ;
    k->transfer += (double)pts * a.dat->elem_size * ((a.acc == OPS_RW || a.acc == OPS_INC) ? 2 : 1);
  }
}

/* ---- output / timing ---- */
OPS_API void ops_printf(const char *fmt, ...) {
  if (st().comm.rank != 0) return;  // rank 0 prints
  va_list ap;
  va_start(ap, fmt);
  vprintf(fmt, ap);
  va_end(ap);
}
OPS_API void ops_fprintf(FILE *f, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vfprintf(f, fmt, ap);
  va_end(ap);
}
OPS_API void ops_diagnostic_output(void) {}
OPS_API size_t ops_timing_output_str(char *buf, size_t n) {
  std::string s = "  Timings (oracle)\n";
  char line[256];
  for (auto &k : st().stats) {
    snprintf(line, sizeof line, "%-40s %8ld %12.6f %12.4f\n", k.name.c_str(), k.count, k.time,
             k.time > 0 ? k.transfer / k.time / 1e9 : 0.0);
    s += line;
  }
  if (buf && n) {
    size_t m = std::min(n - 1, s.size());
    memcpy(buf, s.data(), m);
    buf[m] = 0;
  }
  return s.size();
}
OPS_API void ops_timing_output_stdout(void) {
  size_t n = ops_timing_output_str(nullptr, 0);
  std::string s(n + 1, 0);
  ops_timing_output_str(&s[0], n + 1);
  fputs(s.c_str(), stdout);
}
OPS_API void ops_timers_core(double *cpu, double *et) {
  *cpu = (double)clock() / CLOCKS_PER_SEC;
  *et = wall();
}
OPS_API void ops_timers(double *cpu, double *et) { ops_timers_core(cpu, et); }
OPS_API int ops_is_root(void) { return st().comm.rank == 0; }
OPS_API int ops_get_proc(void) { return st().comm.rank; }
OPS_API int ops_num_procs(void) { return st().comm.size; }
/* ops_dummy_singlenode.cpp:871-878 / ops_lib_core.cpp:1845-1936: the first
 * NaN in (point, component) order stops the program with status 2 */
OPS_API void ops_NaNcheck(ops_dat d) {
  ops_printf("ops_NaNcheck_core called for %s \n", d->name);
  const bool dbl = !strcmp(d->type, "double"), flt = !strcmp(d->type, "float");
  if (!dbl && !flt) return;
  size_t npts = 1;
  for (int i = 0; i < OPS_MAX_DIM; i++) npts *= (size_t)std::max(1, d->size[i]);
  for (size_t pt = 0; pt < npts; pt++)
    for (int c = 0; c < d->dim; c++) {
      const size_t e = st().inst.OPS_soa ? pt + (size_t)c * npts : pt * d->dim + c;
      const double v = dbl ? ((const double *)d->data)[e] : ((const float *)d->data)[e];
      if (v != v) {
        int idx[OPS_MAX_DIM];
        size_t q = pt;
        for (int i = 0; i < OPS_MAX_DIM; i++) {
          const int sz = std::max(1, d->size[i]);
          idx[i] = (int)(q % sz) + d->d_m[i];
          q /= sz;
        }
        printf("Error: NaN detected at element dim:%d,index:(%d", c, idx[0]);
        for (int i = 1; i < d->block->dims; i++) printf(",%d", idx[i]);
        printf(")\n");
        fflush(stdout);
        exit(2);
      }
    }
}
OPS_API void ops_partition(const char *) {}
OPS_API void ops_partition_opts_c(const char *) {}
OPS_API void ops_get_data(ops_dat) {}
OPS_API void ops_put_data(ops_dat) {}
OPS_API bool ops_checkpointing_init(const char *, double, int) { return false; }
OPS_API void ops_checkpointing_initphase_done(void) {}
OPS_API bool ops_checkpointing_before(ops_arg *, int, int *, int) { return true; }
OPS_API bool ops_checkpointing_name_before(ops_arg *, int, int *, const char *) { return true; }
OPS_API void ops_checkpointing_manual_datlist(int, ops_dat *) {}
OPS_API bool ops_checkpointing_fastfw(int, char *) { return false; }
OPS_API bool ops_checkpointing_manual_datlist_fastfw(int, ops_dat *, int, char *) {
  return false;
}
OPS_API bool ops_checkpointing_manual_datlist_fastfw_trigger(int, ops_dat *, int, char *) {
  return false;
}
OPS_API void ops_reset_gpu_power_counters(void) {}
OPS_API double ops_get_gpu_energy_consumed(void) { return 0.0; }

OPS_API void ops_print_dat_to_txtfile(ops_dat d, const char *file) {
  FILE *f = fopen(file, "a");
  if (!f) return;
  fprintf(f, "ops_dat %s, dim %d, sizes %d %d %d\n", d->name, d->dim, d->size[0], d->size[1],
          d->size[2]);
  size_t n = dat_points(d) * d->dim;
  for (size_t i = 0; i < n; i++) {
    if (!strcmp(d->type, "double"))
      fprintf(f, " %3.10lf", ((double *)d->data)[i]);
    else if (!strcmp(d->type, "float"))
      fprintf(f, " %3.10f", ((float *)d->data)[i]);
    else if (!strcmp(d->type, "int"))
      fprintf(f, " %d", ((int *)d->data)[i]);
    else if (!strcmp(d->type, "complexd"))  // ops_lib_core.cpp:1422-1429
      fprintf(f, " %3.10lf+%3.10lfi", ((double *)d->data)[2 * i], ((double *)d->data)[2 * i + 1]);
    else if (!strcmp(d->type, "complexf"))
      fprintf(f, " %e+%ei", ((float *)d->data)[2 * i], ((float *)d->data)[2 * i + 1]);
    if ((i + 1) % (size_t)(d->size[0] * d->dim) == 0) fprintf(f, "\n");
  }
  fclose(f);
}

OPS_API void ops_fetch_dat_hdf5_file(ops_dat, char const *) {}
OPS_API void ops_fetch_block_hdf5_file(ops_block, char const *) {}
OPS_API void ops_fetch_stencil_hdf5_file(ops_stencil, char const *) {}
OPS_API void ops_fetch_halo_hdf5_file(ops_halo, char const *) {}
OPS_API void ops_print_dat_to_txtfile_core(ops_dat d, const char *file) {
  ops_print_dat_to_txtfile(d, file);
}
OPS_API void *xmalloc(size_t n) {
  void *p = malloc(n);
  if (!p && n) abort();
  return p;
}
OPS_API void *xrealloc(void *p, size_t n) {
  void *q = realloc(p, n);
  if (!q && n) abort();
  return q;
}
OPS_API void *xcalloc(size_t k, size_t n) {
  void *p = calloc(k, n);
  if (!p && k != 0 && n != 0) abort();
  return p;
}

/* ---- external access (ops_dummy_singlenode.cpp:630-850, ops_util.cpp:353-500) ---- */
OPS_API int ops_dat_get_local_npartitions(ops_dat) { return 1; }
OPS_API int ops_dat_get_global_npartitions(ops_dat) { return 1; }
OPS_API void ops_dat_get_extents(ops_dat d, int, int *disp, int *size) {
  for (int i = 0; i < d->block->dims; i++) {
    if (disp) disp[i] = 0;
    if (size) size[i] = d->size[i] + d->d_m[i] - d->d_p[i];
  }
  const DistDat &x = st().dd[d->index];
  if (st().dist && x.split) {  // this rank's interior rows
    const int ax = x.axis, sh = -d->d_m[ax];
    const int n = d->size[ax] + d->d_m[ax] - d->d_p[ax];
    const int a = std::max(0, x.o_lo - sh), b = std::min(n, x.o_hi - sh);
    if (disp) disp[ax] = a;
    if (size) size[ax] = std::max(0, b - a);
  }
}
OPS_API size_t ops_dat_get_slab_extents(ops_dat d, int part, int *disp, int *size, int *slab) {
  int ext[OPS_MAX_DIM];
  ops_dat_get_extents(d, part, nullptr, ext);
  size_t bytes = d->elem_size;
  for (int i = 0; i < d->block->dims; i++) {
    if (slab[2 * i] < 0 || slab[2 * i + 1] > ext[i])
      throw OPSException(OPS_RUNTIME_ERROR, "Error: ops_dat_get_slab_extents() out of range");
    disp[i] = slab[2 * i];
    size[i] = slab[2 * i + 1] - slab[2 * i];
    bytes *= size[i];
  }
  return bytes;
}
OPS_API void ops_dat_get_raw_metadata(ops_dat d, int part, int *disp, int *size, int *stride,
                                      int *d_m, int *d_p) {
  ops_dat_get_extents(d, part, disp, size);
  for (int i = 0; i < d->block->dims; i++) {
    if (stride) stride[i] = d->size[i];
    if (d_m) d_m[i] = d->d_m[i];
    if (d_p) d_p[i] = d->d_p[i];
  }
}
OPS_API char *ops_dat_get_raw_pointer(ops_dat d, int, ops_stencil, ops_memspace *ms) {
  if (st().dist && st().dd[d->index].split) dist_unsupported(d, "a raw pointer");
  if (ms) *ms = OPS_HOST;
  d->locked_hd = 1;
  return d->data + d->base_offset;
}
OPS_API void ops_dat_release_raw_data(ops_dat d, int, ops_access) { d->locked_hd = 0; }
OPS_API void ops_dat_release_raw_data_memspace(ops_dat d, int, ops_access, ops_memspace *) {
  d->locked_hd = 0;
}

/* copy between a dense AoS slab buffer and the dat (fetch: dir=0, set: dir=1) */
static void slab_copy(ops_dat d, char *buf, const int *range, int dir) {
  int lo[OPS_MAX_DIM] = {0}, cnt[OPS_MAX_DIM] = {1, 1, 1, 1, 1};
  for (int i = 0; i < d->block->dims; i++) {
    lo[i] = range[2 * i];
    cnt[i] = range[2 * i + 1] - range[2 * i];
  }
  size_t b = 0;
  int s[OPS_MAX_DIM] = {0};
  for (int z = 0; z < cnt[2]; z++)
    for (int y = 0; y < cnt[1]; y++)
      for (int x = 0; x < cnt[0]; x++) {
        s[0] = lo[0] + x - d->d_m[0];
        s[1] = lo[1] + y - d->d_m[1];
        s[2] = lo[2] + z - d->d_m[2];
        for (int c = 0; c < d->dim; c++, b++) {
          char *e = elem_ptr(d, s, c);
          if (dir == 0)
            memcpy(buf + b * d->type_size, e, d->type_size);
          else
            memcpy(e, buf + b * d->type_size, d->type_size);
        }
      }
}
static void full_range(ops_dat d, int *r) {
  int ext[OPS_MAX_DIM];
  ops_dat_get_extents(d, 0, nullptr, ext);
  for (int i = 0; i < OPS_MAX_DIM; i++) {
    r[2 * i] = 0;
    r[2 * i + 1] = i < d->block->dims ? ext[i] : 1;
  }
}
OPS_API void ops_dat_fetch_data_memspace(ops_dat d, int, char *data, ops_memspace) {
  int r[2 * OPS_MAX_DIM];
  full_range(d, r);
  slab_copy(d, data, r, 0);
}
OPS_API void ops_dat_fetch_data(ops_dat d, int part, char *data) {
  ops_dat_fetch_data_memspace(d, part, data, OPS_HOST);
}
OPS_API void ops_dat_fetch_data_slab_memspace(ops_dat d, int, char *data, int *range,
                                              ops_memspace) {
  slab_copy(d, data, range, 0);
}
OPS_API void ops_dat_set_data_memspace(ops_dat d, int, char *data, ops_memspace) {
  int r[2 * OPS_MAX_DIM];
  full_range(d, r);
  slab_copy(d, data, r, 1);
}
OPS_API void ops_dat_set_data(ops_dat d, int part, char *data) {
  ops_dat_set_data_memspace(d, part, data, OPS_HOST);
}
OPS_API void ops_dat_set_data_slab_memspace(ops_dat d, int, char *data, int *range,
                                            ops_memspace) {
  slab_copy(d, data, range, 1);
}

/* ---- random fills: counter-based generator shared bit-for-bit with the
 *      device implementation (splitmix64 of seed and a running counter). ---- */
static inline unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
OPS_API void ops_randomgen_init(unsigned int seed, int) {
  st().rng_seed = seed;
  st().rng_counter = 0;
}
OPS_API void ops_randomgen_exit(void) {}
static void fill_rand(ops_dat d, int normal) {
  size_t n = dat_points(d) * d->dim;
  for (size_t i = 0; i < n; i++) {
    unsigned long long k = st().rng_counter + i;
    unsigned long long r1 = mix64(st().rng_seed * 0x100000001b3ULL ^ (2 * k));
    double u1 = (double)(r1 >> 11) * (1.0 / 9007199254740992.0);
    double v = u1;
    if (normal) {
      unsigned long long r2 = mix64(st().rng_seed * 0x100000001b3ULL ^ (2 * k + 1));
      double u2 = (double)(r2 >> 11) * (1.0 / 9007199254740992.0);
      v = sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307179586 * u2);
    }
    if (!strcmp(d->type, "double"))
      ((double *)d->data)[i] = v;
    else if (!strcmp(d->type, "float"))
      ((float *)d->data)[i] = (float)v;
  }
  st().rng_counter += n;
}
OPS_API void ops_fill_random_uniform(ops_dat d) { fill_rand(d, 0); }
OPS_API void ops_fill_random_normal(ops_dat d) { fill_rand(d, 1); }

/* ---- dump hook shared with the product: every live dat, halos included ---- */
OPS_API void ops_dump_dats(const char *path) {
  std::string fp(path);
  if (st().dist) fp += ".r" + std::to_string(st().comm.rank);  // one file per rank
  FILE *f = fopen(fp.c_str(), "wb");
  if (!f) return;
  for (ops_dat d : st().dats) {
    if (!d) continue;
    const DistDat &x = st().dd[d->index];
    if (st().dist && !x.split && st().comm.rank != 0) continue;  // rank 0 writes whole dats
    int sz[OPS_MAX_DIM];
    for (int i = 0; i < OPS_MAX_DIM; i++) sz[i] = d->size[i];
    const char *src = d->data;
    size_t nbytes = d->mem;
    if (st().dist && x.split) {  // this rank's owned rows
      sz[x.axis] = x.o_hi - x.o_lo;
      src = d->data + (size_t)x.o_lo * x.row_bytes;
      nbytes = (size_t)(x.o_hi - x.o_lo) * x.row_bytes;
    }
    int nl = (int)strlen(d->name);
    fwrite("DAT0", 1, 4, f);
    fwrite(&nl, 4, 1, f);
    fwrite(d->name, 1, nl, f);
    int tl = (int)strlen(d->type);
    fwrite(&tl, 4, 1, f);
    fwrite(d->type, 1, tl, f);
    int meta[4] = {d->dim, d->type_size, d->block->dims, st().inst.OPS_soa};
    fwrite(meta, 4, 4, f);
    fwrite(sz, 4, OPS_MAX_DIM, f);
    fwrite(d->d_m, 4, OPS_MAX_DIM, f);
    fwrite(d->d_p, 4, OPS_MAX_DIM, f);
    unsigned long long nb = nbytes;
    fwrite(&nb, 8, 1, f);
    fwrite(src, 1, nbytes, f);
  }
  fclose(f);
}
