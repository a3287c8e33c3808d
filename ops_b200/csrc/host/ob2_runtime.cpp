// ob2_runtime.cpp -- the OPS host runtime of the B200 backend.
//
// Implements the C entry points of include/ops_lib_core.h (and the
// generated-stub ABI of include/ops_b200_loop.h) on top of the thin CUDA ABI
// of include/ops_b200_device.h.  Replaces, for a single GPU:
//   ops/c/src/core/ops_lib_core.cpp      object declaration, args, reductions,
//                                        dirty bits, timing/transfer model
//   ops/c/src/core/ops_device_singlenode_common.cpp   device dats, halo transfer
//   ops/c/src/core/ops_dummy_singlenode.cpp           raw pointers, fetch/set,
//                                        low-dim (edge) dat accumulation init
//   ops/c/src/cuda/ops_cuda_common.cu    device init, memory, random fills
//
// Design: every dat lives in HBM (device copy authoritative); the host copy is
// materialised only when the app asks for host data.  Par_loops, halo
// transfers and tridiagonal solves are queued on one CUDA stream and never
// wait for the device; only reduction results, fetches and host raw pointers
// synchronise.  Errors surface as OPSException with the reference's codes.
#include <dlfcn.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <limits>
#include <string>
#include <unordered_map>
#include <vector>

#include "ops_b200_device.h"
#include "ops_b200_dist.h"
#include "ops_b200_loop.h"
#include "ops_lib_core.h"
#include "ops_tridiag.h"

namespace {

struct KStat {
  std::string name;
  long count = 0;
  double host_s = 0.0;    // host wall time (enqueue, or device time under diags>1)
  double dev_ms = 0.0;    // device time from events (diags > 1)
  double transfer = 0.0;  // bytes, OPS transfer model
  // block-shape autotuning (loops without reductions): 0 not started,
  // 1 every candidate launched once, 2 decided
  int tune_state = 0;
  int tune_next = 0;
  int tune_dim = 2;
  int best[3] = {0, 0, 0};
  std::vector<void *> tune_ev;        // start/end event per candidate
  std::vector<long long> tune_pts;    // points of the candidate's launch
  // temporal-blocking depth autotuning (OPS_B200_TB_DEPTH=auto): 0 trying the
  // candidates, 1 every candidate timed, 2 decided (tb_best sweeps per launch)
  int tb_state = 0;
  int tb_next = 0;
  int tb_best = 0;
  std::vector<void *> tb_ev;          // start/end event per timed chain
  std::vector<long long> tb_sw;       // sweeps of the timed chain
};

// block shapes the autotuner tries (x, y, z); one thread per point, so the
// shape changes neither any point's arithmetic nor, for loops without
// reductions, any result
static const int kTune2[][3] = {{32, 4, 1}, {32, 8, 1}, {64, 4, 1}, {128, 2, 1}, {32, 16, 1},
                                {256, 1, 1}};
static const int kTune3[][3] = {{32, 4, 1}, {32, 8, 1}, {64, 4, 1}, {32, 4, 2}, {32, 2, 4}};
void tune_decide(KStat &k, int dim);

struct DatX {
  int edat_prev_acc = -1;  // last access kind of an edge dat
  // slab decomposition (ops_b200_dist.h): the dat holds storage rows
  // [s_lo, s_hi) of its slowest axis in `alloc`; data_d is offset so that
  // global storage indices address them
  bool split = false;
  char *alloc = nullptr;
  size_t alloc_bytes = 0, row_bytes = 0;
  int axis = -1, s_lo = 0, s_hi = 0, H = 0;
  int o_lo = 0, o_hi = 0;  // owned storage rows
  bool dirty = false;      // written since its last exchange
  char *spare = nullptr;   // temporal blocking: second buffer of the dat's storage
};

struct RedX {
  void *acc_d = nullptr;   // device accumulator
  int pending_first = 0;   // next loop initialises the accumulator
  void *host_pinned = nullptr;
};

struct GroupX {
  void *tasks_d = nullptr;
  int ntasks = 0;
  long long max_pts = 0;
  std::vector<char *> key;  // dat device pointers the table was built for
  // per task, for folding the group into a consuming loop launch: source
  // and destination dat, the destination's loop coordinate of storage index
  // 0 and its box in loop coordinates
  std::vector<int> src_dat, dst_dat;
  std::vector<std::array<int, 3>> org, dlo, dhi;
};

struct Runtime {
  // slab decomposition over ranks (ops_b200_dist.h); size 1: none
  ob2_dist_comm comm = {0, 1, 0, nullptr, nullptr, nullptr};
  bool dist = false;
  std::vector<std::array<int, 5>> bpart;  // per block: G (-1 unset), lo, hi, first, last
  char *xstage = nullptr;                 // pinned staging of exchanged rows (host transport)
  size_t xstage_cap = 0;
  long long exchanges = 0;
  OPS_instance inst;
  OPS_instance *user = nullptr;  // an application-created instance (C++ API)
  bool initialised = false;
  std::vector<ops_block> blocks;
  std::vector<ops_dat> dats;
  std::vector<DatX> datx;
  std::vector<ops_stencil> stencils;
  std::vector<ops_halo> halos;
  std::vector<ops_halo_group> groups;
  std::vector<GroupX> groupx;
  std::vector<ops_reduction> reds;
  std::vector<RedX> redx;
  std::vector<KStat> kstats;
  std::unordered_map<std::string, int> kindex;
  int block_x = 32, block_y = 4, block_z = 1;
  int device = 0;
  int sms = 148;
  // reduction scratch: per-CTA partials + finish counter
  void *partials = nullptr;
  size_t partials_cap = 0;
  unsigned int *counter = nullptr;
  // staging buffer for fetch / set
  char *stage_d = nullptr;
  size_t stage_cap = 0;
  unsigned long long rng_seed = 0, rng_counter = 0;
  ob2_const_fn const_fn = nullptr;
  // per-kernel device timing without host synchronisation: event pairs are
  // recorded around every launch and resolved by ob2_ktime_collect()
  bool ktime = false;
  std::vector<void *> ev_pool;
  struct Pending { void *a, *b; int k; };
  std::vector<Pending> pending;
  long long launches = 0;  // kernels launched by this runtime
  // lazy loop-chain queue (see ob2_launch)
  // lazy queue + graph replay on by default (fewer launch gaps, identical
  // results); OPS_B200_LAZY=0 launches every loop at its call
  bool lazy = true, tiling = false, graphs = true;
  int tile_y = 0, tile_z = 0;  // fixed tile height (OPS_TILESIZE_Y/Z), 0 = from the cache budget
  bool capturing = false;     // recording a loop chain into a graph
  int max_chain = 64;         // queued items that force a flush (0: no limit)
  int red_waves = 1;          // reduction grids: waves of resident CTAs (OPS_B200_RED_WAVES)
  bool autotune = false;      // block-shape autotuning (OPS_B200_AUTOTUNE / OPS_AUTOTUNE)
  std::string tune_file;      // decisions read at ops_init, written at ops_exit
  std::unordered_map<std::string, std::array<int, 3>> tune_known;
  double cache_mb = 40.0;   // L2 budget per tile (OPS_CACHE_SIZE, MB)
  // sx: the stencil's stride per axis (0: the axis of an edge dat, indexed
  // by the stencil offset alone); any: other strides or long stencils (taken
  // to touch everything); sidx: the stencil (index into Runtime::stencils,
  // -1: none)
  struct QAcc { int dat; int acc; int rmin, rmax; int flat; int sx[3]; int any; int sidx; int mg; };  // no padding: hashed as bytes
  struct QItem {
    int kind;               // 0 par_loop, 1 halo group
    ob2_launcher fn;
    ob2_mlauncher mfn;      // multi-instance launcher (NULL: none)
    ob2_flauncher ffn;      // the application's fused launcher (NULL: none)
    int fid, idx32;         // id in ffn; 32-bit offsets
    long long npts;         // points of the range
    std::vector<char> prm;
    unsigned grid[3], block[3];
    int py, ndim, kidx;
    int lo[3], hi[3];
    std::vector<QAcc> acc;
    void *tasks; int ntasks; long long max_pts;  // halo group
    int group;              // halo group index
    ob2_hlauncher hfn;      // halo-folding launcher (NULL: none)
    ob2_tlauncher tfn;      // temporal-blocking launcher (NULL: none)
    const size_t *tb_off;   // view-base offsets of the dat arguments in prm
    const int *tb_role;     // per argument: 1 ping-pong candidate, 2 written dat
    std::vector<int> acc_arg;  // argument index of each entry of acc
  };
  std::vector<QItem> q;
  struct Graph {
    void *exec = nullptr;
    long long kernels = 0;  // kernel launches the graph replays
    std::string params;     // parameter blocks the graph was captured with
    // storage swaps of temporal blocking the chain makes (dat, old, new):
    // repeated on every replay
    std::vector<std::array<long long, 3>> renames;
    // the chain's multi-instance, fused, halo-folding and temporal-blocking
    // launches and sweeps, counted again at every replay
    long long stats[6] = {0, 0, 0, 0, 0, 0};
  };
  std::unordered_map<std::string, Graph> graph_cache;  // key: the chain's shape
  long long chains = 0, graph_hits = 0, graph_updates = 0, tiles_run = 0, multi_launches = 0;
  bool multi = true;          // run independent instances of a loop in one launch
  bool fuse = true;           // run independent small loops in one launch
  long long fuse_pts = 65536; // largest loop (points) that is fused
  long long fused_launches = 0, fused_loops = 0;
  // fold halo transfers into the consuming launch (OPS_B200_HFUSE=1); off by
  // default: C1 (2x2 blocks of 256^2) measured 26.5-27.2 GLUPS folded against
  // 27.3-29.2 unfolded, the CTAs' halo prologue costing more than the launch
  // it saves
  bool hfuse = false;
  long long hfused = 0;       // halo transfers folded
  // temporal blocking of ping-pong sweep chains (OPS_B200_TB=1); off by
  // default: Jacobi 4096^2 (512 sweeps) measured 151 / 203 / 193 GLUPS at
  // depths 2 / 4 / 8 against 272 GLUPS sweep by sweep
  bool tb = false;
  int tb_depth = 8;           // sweeps per temporal-blocking launch (OPS_B200_TB_DEPTH)
  bool tb_auto = false;       // OPS_B200_TB_DEPTH=auto: depth chosen per loop by timing
  long long tb_launches = 0, tb_sweeps = 0;
  std::vector<std::array<long long, 3>> *rename_log = nullptr;  // while capturing
};

Runtime *R = nullptr;

Runtime &rt() {
  if (!R) {
    R = new Runtime();
    memset((void *)&R->inst, 0, sizeof(R->inst));
  }
  return *R;
}

// the instance whose settings apply: the one the application created with
// the C++ object API, else the library's own
OPS_instance &I() {
  Runtime &r = rt();
  return r.user ? *r.user : r.inst;
}

void check(int code, const char *what) {
  if (code != 0) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "Error: CUDA error in " << what << ": " << ob2_error_string(code);
    throw ex;
  }
}

void require_init() {
  if (!rt().initialised) {
    throw OPSException(OPS_RUNTIME_CONFIGURATION_ERROR,
                       "Error: ops_init must be called before other OPS routines");
  }
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
  for (int i = 0; i < OPS_MAX_DIM; i++) n *= (size_t)d->size[i];
  return n;
}

void ensure_host(ops_dat d) {
  if (!d->data) {
    d->data = (char *)calloc(d->mem ? d->mem : 1, 1);
    d->user_managed = 0;
  }
}

/* device -> host when the device copy is newer (ops_lib_core.cpp:2366-2379) */
void dist_unsupported(ops_dat d, const char *what);
void get_data(ops_dat d) {
  if (rt().dist && rt().datx[d->index].split && d->dirty_hd == 2)
    dist_unsupported(d, "a host copy of the whole dat");
  ensure_host(d);
  ob2_flush();
  if (d->dirty_hd == 2) {
    check(ob2_dev_d2h(d->data, d->data_d, d->mem), "ops_get_data");
    d->dirty_hd = 0;
  }
}

/* host -> device when the host copy is newer (ops_lib_core.cpp:2381-2392) */
void put_data(ops_dat d) {
  if (d->dirty_hd == 1 && rt().dist && rt().datx[d->index].split)
    dist_unsupported(d, "uploading a host copy of the whole dat");
  if (d->dirty_hd == 1) {
    ob2_flush();
    check(ob2_dev_h2d(d->data_d, d->data, d->mem), "ops_put_data");
    d->dirty_hd = 0;
  }
}

/* ------------------------------------------------------------------------
 * Slab decomposition over ranks (ops_b200_dist.h).  The partition of a block
 * is fixed by the first dat declared on it; every dat then holds its owned
 * storage rows of the slowest axis plus H rows on each inner side.
 * ---------------------------------------------------------------------- */
void dist_unsupported(ops_dat d, const char *what) {
  OPSException ex(OPS_NOT_IMPLEMENTED);
  ex << "Error: " << what << " (dat " << (d ? d->name : "-")
     << ") is not supported with the slab decomposition over ranks";
  throw ex;
}

std::array<int, 5> &block_part(ops_block b, int G) {
  Runtime &r = rt();
  if ((int)r.bpart.size() <= b->index) r.bpart.resize(b->index + 1, {-1, 0, 0, 0, 0});
  std::array<int, 5> &bp = r.bpart[b->index];
  if (bp[0] < 0 && G > 0) {
    bp[0] = G;
    ob2dist::slab(G, r.comm.size, r.comm.rank, &bp[1], &bp[2]);
    bp[3] = r.comm.rank == 0;
    bp[4] = r.comm.rank == r.comm.size - 1;
    if (bp[2] - bp[1] < 1) {
      OPSException ex(OPS_INVALID_ARGUMENT);
      ex << "Error: block " << b->name << " has " << G << " rows along its slowest axis: too "
         << "few for " << r.comm.size << " ranks";
      throw ex;
    }
  }
  return bp;
}

// decides the held rows of a new dat; returns false when it is not split
bool dist_layout(ops_dat d, DatX &x) {
  Runtime &r = rt();
  if (!r.dist) return false;
  const int ax = d->block->dims - 1;
  if (ax < 0 || ax > 2 || d->size[ax] == 1) return false;  // edge dats: whole on every rank
  if (I().OPS_soa && d->dim > 1) dist_unsupported(d, "a multi-component dat in SoA layout");
  const int n = d->size[ax] + d->d_m[ax] - d->d_p[ax];  // interior extent
  std::array<int, 5> &bp = block_part(d->block, n);
  x.split = true;
  x.axis = ax;
  x.H = std::max(1, std::max(-d->d_m[ax], d->d_p[ax]));
  // block rows -> storage rows: s = y - base - d_m
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
  x.alloc_bytes = (size_t)(x.s_hi - x.s_lo) * rb;
  return true;
}

void xstage_reserve(size_t n) {
  Runtime &r = rt();
  if (n <= r.xstage_cap) return;
  if (r.xstage) ob2_host_free_pinned(r.xstage);
  r.xstage = nullptr;
  check(ob2_host_alloc_pinned((void **)&r.xstage, n), "slab exchange staging");
  r.xstage_cap = n;
}

// refreshes the H inner halo rows of a split dat from its neighbours:
// owned rows [o_lo, o_lo + H) go down into the lower rank's top halo,
// [o_hi - H, o_hi) up into the upper rank's bottom halo
void dist_exchange(ops_dat d) {
  Runtime &r = rt();
  DatX &x = r.datx[d->index];
  ob2_flush();
  const int up = r.comm.rank + 1 < r.comm.size ? r.comm.rank + 1 : -1;
  const int dn = r.comm.rank > 0 ? r.comm.rank - 1 : -1;
  const size_t nb = (size_t)x.H * x.row_bytes;
  char *base = d->data_d;  // global storage row 0
  char *top_own = base + (size_t)(x.o_hi - x.H) * x.row_bytes;
  char *top_halo = base + (size_t)x.o_hi * x.row_bytes;
  char *bot_own = base + (size_t)x.o_lo * x.row_bytes;
  char *bot_halo = base + (size_t)(x.o_lo - x.H) * x.row_bytes;
  int e = 0;
  if (r.comm.device) {  // device buffers, ordered on the work stream
    e = r.comm.sendrecv(r.comm.ctx, top_own, up >= 0 ? nb : 0, up, bot_halo, dn >= 0 ? nb : 0,
                        dn);
    if (!e)
      e = r.comm.sendrecv(r.comm.ctx, bot_own, dn >= 0 ? nb : 0, dn, top_halo,
                          up >= 0 ? nb : 0, up);
  } else {  // host transport: rows staged through pinned memory
    xstage_reserve(2 * nb);
    char *sb = r.xstage, *rb = r.xstage + nb;
    if (up >= 0) check(ob2_dev_d2h(sb, top_own, nb), "slab exchange");
    e = r.comm.sendrecv(r.comm.ctx, sb, up >= 0 ? nb : 0, up, rb, dn >= 0 ? nb : 0, dn);
    if (!e && dn >= 0) check(ob2_dev_h2d(bot_halo, rb, nb), "slab exchange");
    if (!e && dn >= 0) check(ob2_dev_d2h(sb, bot_own, nb), "slab exchange");
    if (!e) e = r.comm.sendrecv(r.comm.ctx, sb, dn >= 0 ? nb : 0, dn, rb, up >= 0 ? nb : 0, up);
    if (!e && up >= 0) check(ob2_dev_h2d(top_halo, rb, nb), "slab exchange");
  }
  if (e) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "Error: slab halo exchange of dat " << d->name << " failed (" << e << ")";
    throw ex;
  }
  x.dirty = false;
  r.exchanges++;
}

// before a loop: clips its range along the slowest axis to this rank's rows
// and refreshes the inner halos of the split dats it reads through a stencil
// reaching along that axis (when written since their last exchange); marks
// the split dats it writes as written
void dist_loop(ops_block block, int dim, int *lo, int *hi, ops_arg *args, int nargs,
               const char *name) {
  Runtime &r = rt();
  if (!r.dist) return;
  const int ax = dim - 1;
  if (ax < 0 || ax > 2) return;
  for (int i = 0; i < nargs; i++) {
    ops_arg &a = args[i];
    if (a.argtype != OPS_ARG_DAT || !a.dat || a.acc == OPS_WRITE) continue;
    DatX &x = r.datx[a.dat->index];
    if (!x.split) continue;
    int reach = 0;
    if (a.stencil) {
      if (a.stencil->type != 0 || (ax < a.stencil->dims && a.stencil->stride[ax] > 1))
        dist_unsupported(a.dat, "a strided or multigrid stencil along the split axis");
      for (int p = 0; p < a.stencil->points; p++)
        if (ax < a.stencil->dims)
          reach = std::max(reach, std::abs(a.stencil->stencil[p * a.stencil->dims + ax]));
    }
    if (reach > x.H) {
      OPSException ex(OPS_NOT_IMPLEMENTED);
      ex << "Error: ops_par_loop " << name << " reads " << a.dat->name << " " << reach
         << " rows along the split axis, beyond its halo depth " << x.H;
      throw ex;
    }
    if (reach > 0 && x.dirty) dist_exchange(a.dat);
  }
  for (int i = 0; i < nargs; i++) {
    ops_arg &a = args[i];
    if (a.argtype == OPS_ARG_DAT && a.dat && a.acc != OPS_READ && r.datx[a.dat->index].split)
      r.datx[a.dat->index].dirty = true;
  }
  const std::array<int, 5> &bp = block_part(block, 0);
  if (bp[0] >= 0) ob2dist::clip(bp[1], bp[2], bp[3], bp[4], &lo[ax], &hi[ax]);
}

int red_type(const char *t) {
  if (!strcmp(t, "double")) return 0;
  if (!strcmp(t, "float")) return 1;
  if (!strcmp(t, "int")) return 2;
  if (!strcmp(t, "long long") || !strcmp(t, "ll")) return 3;
  return -1;
}

int type_code(const char *t) {
  if (!strcmp(t, "double") || !strcmp(t, "real(8)") || !strcmp(t, "double precision")) return 1;
  if (!strcmp(t, "float") || !strcmp(t, "real") || !strcmp(t, "real(4)")) return 2;
  if (!strcmp(t, "int") || !strcmp(t, "integer") || !strcmp(t, "int(4)")) return 3;
  if (!strcmp(t, "long long") || !strcmp(t, "ll")) return 4;
  if (!strcmp(t, "unsigned int") || !strcmp(t, "uint")) return 5;
  if (!strcmp(t, "char")) return 6;
  if (!strcmp(t, "short")) return 7;
  if (!strcmp(t, "long")) return 8;
  if (!strcmp(t, "complexd")) return 9;
  if (!strcmp(t, "complexf")) return 10;
  return 0;
}

/* bytes of one value of type code tc */
int type_bytes(int tc) {
  switch (tc) {
    case 1: case 4: case 8: case 10: return 8;
    case 6: return 1;
    case 7: return 2;
    case 9: return 16;
    default: return 4;
  }
}

/* identity of a reduction / low-dim accumulation (ops_lib_core.cpp:840-965) */
void identity_bytes(int tc, int acc, void *out, bool lowdim) {
  switch (tc) {
    case 1: {
      double v = acc == OPS_MIN ? DBL_MAX : (acc == OPS_MAX ? -DBL_MAX : 0.0);
      if (lowdim && acc == OPS_MAX) v = std::numeric_limits<double>::lowest();
      memcpy(out, &v, 8);
      break;
    }
    case 2: {
      float v = acc == OPS_MIN ? FLT_MAX : (acc == OPS_MAX ? -FLT_MAX : 0.0f);
      memcpy(out, &v, 4);
      break;
    }
    case 3: {
      int v = acc == OPS_MIN ? INT_MAX : (acc == OPS_MAX ? INT_MIN : 0);
      memcpy(out, &v, 4);
      break;
    }
    case 4: {
      long long v = acc == OPS_MIN ? LLONG_MAX : (acc == OPS_MAX ? LLONG_MIN : 0);
      memcpy(out, &v, 8);
      break;
    }
    case 5: {
      unsigned v = acc == OPS_MIN ? UINT_MAX : 0u;
      memcpy(out, &v, 4);
      break;
    }
    case 6: {
      char v = acc == OPS_MIN ? CHAR_MAX : (acc == OPS_MAX ? CHAR_MIN : 0);
      memcpy(out, &v, 1);
      break;
    }
    case 7: {
      short v = acc == OPS_MIN ? SHRT_MAX : (acc == OPS_MAX ? SHRT_MIN : 0);
      memcpy(out, &v, 2);
      break;
    }
    case 8: {
      long v = acc == OPS_MIN ? LONG_MAX : (acc == OPS_MAX ? LONG_MIN : 0);
      memcpy(out, &v, 8);
      break;
    }
    case 9: {  // complexd: (MAX, MAX) for OPS_MIN, zero otherwise (ops_lib_core.cpp:944-952)
      double v[2] = {0.0, 0.0};
      if (acc == OPS_MIN) v[0] = v[1] = DBL_MAX;
      memcpy(out, v, 16);
      break;
    }
    case 10: {  // complexf (ops_lib_core.cpp:935-943)
      float v[2] = {0.0f, 0.0f};
      if (acc == OPS_MIN) v[0] = v[1] = FLT_MAX;
      memcpy(out, v, 8);
      break;
    }
    default:
      throw OPSException(OPS_NOT_IMPLEMENTED, "Error, reduction type not recognised");
  }
}

int kernel_slot(const char *name) {
  Runtime &r = rt();
  auto it = r.kindex.find(name);
  if (it != r.kindex.end()) return it->second;
  int k = (int)r.kstats.size();
  r.kstats.push_back(KStat());
  r.kstats.back().name = name;
  r.kindex[name] = k;
  auto t = r.tune_known.find(name);
  if (t != r.tune_known.end()) {
    KStat &s = r.kstats.back();
    s.tune_state = 2;
    for (int i = 0; i < 3; i++) s.best[i] = t->second[i];
  }
  return k;
}

void *pool_event() {
  Runtime &r = rt();
  void *e = nullptr;
  if (!r.ev_pool.empty()) {
    e = r.ev_pool.back();
    r.ev_pool.pop_back();
  } else {
    check(ob2_event_create(&e), "event");
  }
  return e;
}

/* start / end of one timed launch of kernel slot k (ktime mode) */
void *kt_begin() {
  if (!rt().ktime) return nullptr;
  void *a = pool_event();
  ob2_event_record(a);
  return a;
}
void kt_end(void *a, int k) {
  Runtime &r = rt();
  if (!a) return;
  void *b = pool_event();
  ob2_event_record(b);
  r.pending.push_back({a, b, k});
}

/* ------------------------------------------------------------------------
 * Lazy loop-chain queue.
 *
 * Restates the reference's lazy execution (ops_lazy.cpp:186-276,1248-1446):
 * loops are recorded and run at the next flush point.  Two GPU-specific
 * executions of a recorded chain:
 *  - tiled: the chain runs tile by tile along the slowest axis, tiles sized
 *    so that a tile's rows of every dat the chain touches fit the L2 budget,
 *    so later loops read what earlier loops wrote from L2 instead of HBM.
 *    Tiles are skewed per loop (the scheme of ops_construct_tile_plan,
 *    ops_lazy.cpp:380-1187): walking the chain backwards, a loop's tile edge
 *    is pushed past that of every later loop that depends on it through a
 *    common dat, by that pair's stencil reach, so that each tile of a loop
 *    finds its inputs complete and overwrites nothing a later tile still
 *    reads.  Every point is computed by the same kernel as untiled, so the
 *    results are identical.
 *  - graph: the launches of a flushed chain are captured once into a CUDA
 *    graph keyed by their parameters; a recurring identical chain replays
 *    the graph (one launch instead of one per loop and tile).
 * ---------------------------------------------------------------------- */
void run_item(Runtime::QItem &it, const int *lo_t, const int *hi_t) {
  Runtime &r = rt();
  if (it.kind == 1) {
    void *ev = r.capturing ? nullptr : kt_begin();
    check(ob2_halo_run((const ob2_halo_task *)it.tasks, it.ntasks, it.max_pts),
          "ops_halo_transfer");
    r.launches++;
    kt_end(ev, it.kidx);
    return;
  }
  void *ev = r.capturing ? nullptr : kt_begin();
  if (!lo_t) {
    check(it.fn(it.prm.data(), it.grid, it.block, ob2_dev_stream()), "ops_par_loop launch");
    r.launches++;
    kt_end(ev, it.kidx);
    return;
  }
  // re-range the launch to the tile: the parameter block starts with
  // int lo[3], hi[3]
  std::vector<char> p(it.prm);
  int *lohi = (int *)p.data();
  unsigned g[3] = {it.grid[0], it.grid[1], it.grid[2]};
  const int td = it.ndim - 1;
  lohi[td] = lo_t[td];
  lohi[3 + td] = hi_t[td];
  const unsigned rows = it.block[td] * (td == 1 ? (unsigned)it.py : 1u);
  g[td] = (unsigned)((hi_t[td] - lo_t[td] + (int)rows - 1) / (int)rows);
  check(it.fn(p.data(), g, it.block, ob2_dev_stream()), "ops_par_loop launch (tile)");
  r.launches++;
  r.tiles_run++;
  kt_end(ev, it.kidx);
}

/* Tiled execution of queue items [b, e) (par_loops only, same dimension). */
void run_tiled(std::vector<Runtime::QItem> &q, size_t b, size_t e) {
  Runtime &r = rt();
  const int nd = q[b].ndim;
  const int td = nd - 1;
  const size_t n = e - b;
  // skew per loop: S[k] >= S[j] + reach for every later j depending on k
  std::vector<long long> S(n, 0);
  for (size_t kk = n; kk-- > 0;) {
    Runtime::QItem &K = q[b + kk];
    for (size_t jj = kk + 1; jj < n; jj++) {
      Runtime::QItem &J = q[b + jj];
      for (auto &ka : K.acc)
        for (auto &ja : J.acc) {
          if (ka.dat != ja.dat) continue;
          const bool kw = ka.acc != OPS_READ, jw = ja.acc != OPS_READ;
          long long need = 0;
          bool dep = false;
          if (kw) {  // J reads or writes what K wrote: J's reach above
            dep = true;
            need = std::max(need, (long long)std::max(0, ja.rmax));
          }
          if (jw) {  // J overwrites what K read: K's reach below
            dep = true;
            need = std::max(need, (long long)std::max(0, -ka.rmin));
          }
          if (dep) S[kk] = std::max(S[kk], S[jj] + need);
        }
    }
  }
  // tile height from the L2 budget: rows (planes) of every dat touched
  long long ymin = LLONG_MAX, ymax = LLONG_MIN;
  double row_bytes = 0.0;
  std::vector<int> seen;
  for (size_t k = b; k < e; k++) {
    ymin = std::min(ymin, (long long)q[k].lo[td]);
    ymax = std::max(ymax, (long long)q[k].hi[td]);
    for (auto &a : q[k].acc) {
      if (std::find(seen.begin(), seen.end(), a.dat) != seen.end()) continue;
      seen.push_back(a.dat);
      ops_dat d = r.dats[a.dat];
      double rb = d->elem_size;
      for (int i = 0; i < td; i++) rb *= d->size[i];
      row_bytes += rb;
    }
  }
  long long H = td == 2 ? r.tile_z : r.tile_y;
  if (H <= 0) H = (long long)(r.cache_mb * 1048576.0 / std::max(1.0, row_bytes));
  H = std::max(1LL, H);
  const long long T = std::max(1LL, (ymax - ymin + H - 1) / H);
  for (long long t = 0; t < T; t++) {
    for (size_t kk = 0; kk < n; kk++) {
      Runtime::QItem &K = q[b + kk];
      long long lo = t == 0 ? LLONG_MIN : ymin + t * H + S[kk];
      long long hi = t == T - 1 ? LLONG_MAX : ymin + (t + 1) * H + S[kk];
      lo = std::max(lo, (long long)K.lo[td]);
      hi = std::min(hi, (long long)K.hi[td]);
      if (lo >= hi) continue;
      int lt[3] = {K.lo[0], K.lo[1], K.lo[2]}, ht[3] = {K.hi[0], K.hi[1], K.hi[2]};
      lt[td] = (int)lo;
      ht[td] = (int)hi;
      run_item(K, lt, ht);
    }
  }
}

bool tileable(const Runtime::QItem &it) {
  if (it.kind != 0 || it.ndim < 2 || it.ndim > 3) return false;  // 4D / 5D: untiled
  for (auto &a : it.acc) {
    if (a.flat && a.acc != OPS_READ) return false;  // shared across tiles
    if (a.mg) return false;  // multigrid: the dat's rows are not the loop's
  }
  return true;
}

// two queued loops touch a common dat and one of them writes it
bool conflict(const Runtime::QItem &a, const Runtime::QItem &b) {
  for (auto &x : a.acc)
    for (auto &y : b.acc)
      if (x.dat == y.dat && (x.acc != OPS_READ || y.acc != OPS_READ)) return true;
  return false;
}

// q[i] starts a run of instances of one loop that can share a launch:
// returns the end of the run (at most OB2_MULTI_MAX, no data shared)
size_t multi_run(const std::vector<Runtime::QItem> &q, size_t i) {
  if (!q[i].mfn || !rt().multi) return i + 1;
  size_t j = i + 1;
  while (j < q.size() && j - i < OB2_MULTI_MAX && q[j].kind == 0 && q[j].fn == q[i].fn &&
         q[j].mfn == q[i].mfn && q[j].prm.size() == q[i].prm.size() &&
         q[j].block[0] == q[i].block[0] && q[j].block[1] == q[i].block[1] &&
         q[j].block[2] == q[i].block[2]) {
    bool ok = true;
    for (size_t k = i; k < j && ok; k++) ok = !conflict(q[k], q[j]);
    if (!ok) break;
    j++;
  }
  return j;
}

void run_multi(std::vector<Runtime::QItem> &q, size_t i, size_t j) {
  Runtime &r = rt();
  const void *prm[OB2_MULTI_MAX];
  unsigned g[3] = {0, 0, 0};
  for (size_t k = i; k < j; k++) {
    prm[k - i] = q[k].prm.data();
    for (int d = 0; d < 3; d++) g[d] = std::max(g[d], q[k].grid[d]);
  }
  void *ev = r.capturing ? nullptr : kt_begin();
  check(q[i].mfn(prm, (int)(j - i), g, q[i].block, ob2_dev_stream()),
        "ops_par_loop launch (instances)");
  r.launches++;
  r.multi_launches++;
  kt_end(ev, q[i].kidx);
}

// the points of a dat that loop A touches through access x at stencil
// offset pa and loop B through y at pb intersect (per axis: the loop range
// shifted by the offset, or the offset alone on a stride-0 axis)
bool boxes_meet(const Runtime::QItem &A, const Runtime::QAcc &x, const int *pa,
                const Runtime::QItem &B, const Runtime::QAcc &y, const int *pb) {
  for (int k = 0; k < 3; k++) {
    const int alo = x.sx[k] ? A.lo[k] + pa[k] : pa[k], ahi = x.sx[k] ? A.hi[k] + pa[k] : pa[k] + 1;
    const int blo = y.sx[k] ? B.lo[k] + pb[k] : pb[k], bhi = y.sx[k] ? B.hi[k] + pb[k] : pb[k] + 1;
    if (ahi <= blo || bhi <= alo) return false;
  }
  return true;
}

// loop A writes (at the centre point, the only point an OPS kernel may
// write) a point of the dat that loop B touches at its centre or at one of
// its stencil points
bool writes_into(const Runtime::QItem &A, const Runtime::QAcc &x, const Runtime::QItem &B,
                 const Runtime::QAcc &y) {
  static const int zero[3] = {0, 0, 0};
  if (boxes_meet(A, x, zero, B, y, zero)) return true;
  if (y.sidx < 0) return false;
  const ops_stencil_core *st = rt().stencils[y.sidx];
  for (int p = 0; p < st->points; p++) {
    int o[3] = {0, 0, 0};
    for (int k = 0; k < 3 && k < st->dims; k++) o[k] = st->stencil[p * st->dims + k];
    if (boxes_meet(A, x, zero, B, y, o)) return true;
  }
  return false;
}

// two queued loops touch a common point of a dat that one of them writes
bool footprint_conflict(const Runtime::QItem &a, const Runtime::QItem &b) {
  for (auto &x : a.acc)
    for (auto &y : b.acc) {
      if (x.dat != y.dat || (x.acc == OPS_READ && y.acc == OPS_READ)) continue;
      if (x.any || y.any) return true;
      if (x.acc != OPS_READ && writes_into(a, x, b, y)) return true;
      if (y.acc != OPS_READ && writes_into(b, y, a, x)) return true;
    }
  return false;
}

bool fusable(const Runtime::QItem &a) {
  const Runtime &r = rt();
  return r.fuse && !r.ktime && a.kind == 0 && a.ffn && a.fid >= 0 && a.npts <= r.fuse_pts &&
         a.prm.size() <= OB2_FUSE_BLOB;
}

// q[i] starts a run of small loops that can share one fused launch: returns
// the end of the run (at most OB2_FUSE_MAX loops, parameter blocks within
// OB2_FUSE_BLOB, one CTA shape, no footprint conflict between any two)
size_t fuse_run(const std::vector<Runtime::QItem> &q, size_t i) {
  const Runtime::QItem &a = q[i];
  if (!fusable(a)) return i + 1;
  size_t bytes = (a.prm.size() + 15) & ~(size_t)15;
  size_t j = i + 1;
  while (j < q.size() && j - i < OB2_FUSE_MAX) {
    const Runtime::QItem &b = q[j];
    if (!fusable(b) || b.ffn != a.ffn || b.idx32 != a.idx32 || b.block[0] != a.block[0] ||
        b.block[1] != a.block[1] || b.block[2] != a.block[2])
      break;
    const size_t nb = (b.prm.size() + 15) & ~(size_t)15;
    if (bytes + nb > OB2_FUSE_BLOB) break;
    bool ok = true;
    for (size_t k = i; k < j && ok; k++) ok = !footprint_conflict(q[k], b);
    if (!ok) break;
    bytes += nb;
    j++;
  }
  return j;
}

void run_fused(std::vector<Runtime::QItem> &q, size_t i, size_t j) {
  Runtime &r = rt();
  const int n = (int)(j - i);
  int ids[OB2_FUSE_MAX];
  const void *prm[OB2_FUSE_MAX];
  size_t psz[OB2_FUSE_MAX];
  unsigned grids[3 * OB2_FUSE_MAX];
  for (int k = 0; k < n; k++) {
    const Runtime::QItem &it = q[i + k];
    ids[k] = it.fid;
    prm[k] = it.prm.data();
    psz[k] = it.prm.size();
    for (int d = 0; d < 3; d++) grids[3 * k + d] = it.grid[d];
  }
  check(q[i].ffn(n, ids, prm, psz, grids, q[i].block, q[i].idx32, ob2_dev_stream()),
        "ops_par_loop launch (fused)");
  r.launches++;
  r.fused_launches++;
  r.fused_loops += n;
}

// Folding the halo group q[h] into the launch of loop items [b, e) (one
// loop, its instances on several blocks): legal when every task's
// destination dat is read (OPS_READ) by one of the instances, every cell the
// task fills lies inside that instance's range widened by the loop's stencil
// reach (so some CTA's footprint holds it), and no instance writes a dat the
// group reads or fills.  Fills h and returns true when legal.
bool hfuse_plan(const std::vector<Runtime::QItem> &q, size_t hi, size_t b, size_t e,
                ob2_hfuse &h) {
  Runtime &r = rt();
  const Runtime::QItem &H = q[hi];
  if (!r.hfuse || H.kind != 1 || H.group < 0 || b >= e) return false;
  const GroupX &gx = r.groupx[H.group];
  if (gx.ntasks <= 0 || gx.ntasks > OB2_HFUSE_MAX || (int)gx.dst_dat.size() != gx.ntasks)
    return false;
  for (size_t k = b; k < e; k++)
    if (q[k].kind != 0 || !q[k].hfn || q[k].hfn != q[b].hfn) return false;
  memset(&h, 0, sizeof(h));
  // stencil reach of every read argument, per axis
  for (size_t k = b; k < e; k++)
    for (auto &a : q[k].acc) {
      if (a.any || a.flat || a.mg) return false;
      if (a.acc != OPS_READ) {
        for (int t = 0; t < gx.ntasks; t++)
          if (a.dat == gx.src_dat[t] || a.dat == gx.dst_dat[t]) return false;
        continue;
      }
      if (a.sidx < 0) continue;
      const ops_stencil_core *st = r.stencils[a.sidx];
      for (int p = 0; p < st->points; p++)
        for (int d = 0; d < st->dims && d < 3; d++) {
          const int o = st->stencil[p * st->dims + d];
          h.mlo[d] = std::max(h.mlo[d], -o);
          h.mhi[d] = std::max(h.mhi[d], o);
        }
    }
  h.tasks = (const ob2_halo_task *)H.tasks;
  h.n = gx.ntasks;
  for (int t = 0; t < gx.ntasks; t++) {
    int inst = -1;
    for (size_t k = b; k < e && inst < 0; k++)
      for (auto &a : q[k].acc)
        if (a.dat == gx.dst_dat[t] && a.acc == OPS_READ) {
          inst = (int)(k - b);
          break;
        }
    if (inst < 0) return false;
    const Runtime::QItem &L = q[b + inst];
    for (int d = 0; d < 3; d++) {
      const int lo = d < L.ndim ? L.lo[d] - h.mlo[d] : 0;
      const int hi = d < L.ndim ? L.hi[d] + h.mhi[d] : 1;
      if (gx.dlo[t][d] < lo || gx.dhi[t][d] > hi) return false;
      h.org[t][d] = gx.org[t][d];
    }
    h.task[t] = t;
    h.inst[t] = inst;
  }
  for (int d = 0; d < 3; d++)
    if (d >= q[b].ndim) h.mlo[d] = h.mhi[d] = 0;
  return true;
}

void run_hfused(std::vector<Runtime::QItem> &q, size_t b, size_t e, const ob2_hfuse &h) {
  Runtime &r = rt();
  const void *prm[OB2_MULTI_MAX];
  unsigned g[3] = {0, 0, 0};
  for (size_t k = b; k < e; k++) {
    prm[k - b] = q[k].prm.data();
    for (int d = 0; d < 3; d++) g[d] = std::max(g[d], q[k].grid[d]);
  }
  void *ev = r.capturing ? nullptr : kt_begin();
  check(q[b].hfn(prm, (int)(e - b), g, q[b].block, &h, ob2_dev_stream()),
        "ops_par_loop launch (with halo transfer)");
  r.launches++;
  r.hfused++;
  if (e - b > 1) r.multi_launches++;
  kt_end(ev, q[b].kidx);
}

// ---- temporal blocking of ping-pong sweep chains (ob2_tblock) ----
// the stencil of an access stays within +-r along x and y (r = 0: the
// centre only)
bool tb_stencil_within(const Runtime::QAcc &a, int r) {
  if (a.any || a.flat || a.mg || a.sidx < 0) return false;
  const ops_stencil_core *st = rt().stencils[a.sidx];
  if (st->dims != 2 || st->stride[0] != 1 || st->stride[1] != 1) return false;
  for (int p = 0; p < st->points; p++)
    for (int d = 0; d < 2; d++)
      if (std::abs(st->stencil[2 * p + d]) > r) return false;
  return true;
}

// the written dat of an item (entry index in acc), -1: not one
int tb_written(const Runtime::QItem &it) {
  int w = -1;
  for (size_t k = 0; k < it.acc.size(); k++)
    if (it.acc[k].acc != OPS_READ) {
      if (w >= 0 || it.acc[k].acc != OPS_WRITE) return -1;
      w = (int)k;
    }
  return w;
}

bool tb_same_shape(ops_dat a, ops_dat b) {
  if (a->elem_size != b->elem_size || a->dim != 1 || b->dim != 1) return false;
  for (int i = 0; i < 2; i++)
    if (a->size[i] != b->size[i] || a->d_m[i] != b->d_m[i] || a->base[i] != b->base[i])
      return false;
  return true;
}

// items a, b are consecutive sweeps of a ping-pong chain: one loop, a reads
// dat X through a stencil of reach <= 1 (entry ks) and writes dat Y at the
// centre (entry kw), b reads Y at entry ks and writes X at entry kw,
// everything else equal; sets ks and kw
bool tb_pair(const Runtime::QItem &a, const Runtime::QItem &b, int *ks, int *kw) {
  Runtime &r = rt();
  if (a.kind != 0 || b.kind != 0 || !a.tfn || a.tfn != b.tfn || a.fn != b.fn || !a.idx32 ||
      a.ndim != 2 || a.prm.size() != b.prm.size() || a.acc.size() != b.acc.size() ||
      a.lo[0] != b.lo[0] || a.hi[0] != b.hi[0] || a.lo[1] != b.lo[1] || a.hi[1] != b.hi[1] ||
      !a.tb_off || !a.tb_role || r.dist)
    return false;
  const int w = tb_written(a);
  if (w < 0 || tb_written(b) != w) return false;
  int k = -1;
  for (size_t e = 0; e < a.acc.size() && k < 0; e++)
    if ((int)e != w && a.acc[e].acc == OPS_READ && a.acc[e].dat == b.acc[w].dat) k = (int)e;
  if (k < 0 || b.acc[k].dat != a.acc[w].dat || b.acc[k].acc != OPS_READ) return false;
  const int argS = a.acc_arg[k], argW = a.acc_arg[w];
  if (a.tb_role[argS] != 1 || a.tb_role[argW] != 2) return false;
  if (!tb_stencil_within(a.acc[k], 1) || !tb_stencil_within(a.acc[w], 0) ||
      !tb_stencil_within(b.acc[k], 1) || !tb_stencil_within(b.acc[w], 0))
    return false;
  const int X = a.acc[k].dat, Y = a.acc[w].dat;
  if (X == Y || !tb_same_shape(r.dats[X], r.dats[Y])) return false;
  for (size_t e = 0; e < a.acc.size(); e++) {  // every other entry: the same read-only dat
    if ((int)e == w || (int)e == k) continue;
    if (a.acc[e].dat != b.acc[e].dat || a.acc[e].acc != OPS_READ || a.acc[e].dat == X ||
        a.acc[e].dat == Y)
      return false;
  }
  // parameter blocks equal except the two ping-pong view bases
  const size_t os = a.tb_off[argS], ow = a.tb_off[argW];
  for (size_t e = 0; e < a.prm.size(); e++)
    if ((e < os || e >= os + 8) && (e < ow || e >= ow + 8) && a.prm[e] != b.prm[e]) return false;
  *ks = k;
  *kw = w;
  return true;
}

// end of the ping-pong chain starting at q[i] (i + 1: none); the chain
// must reach the end of the queue (later items hold the dats' addresses)
size_t tb_chain(const std::vector<Runtime::QItem> &q, size_t i) {
  if (!rt().tb || rt().tiling || i + 1 >= q.size()) return i + 1;
  size_t j = i + 1;
  int ks, kw;
  while (j < q.size() && tb_pair(q[j - 1], q[j], &ks, &kw)) j++;
  if (j != q.size() || j - i < 2) return i + 1;
  return j;
}

void tb_spare(ops_dat d) {
  DatX &x = rt().datx[d->index];
  if (!x.spare) check(ob2_dev_malloc((void **)&x.spare, d->mem), "temporal blocking");
}

// allocations before a graph capture (none may happen inside one)
void tb_prepare(std::vector<Runtime::QItem> &q) {
  for (size_t i = 0; i < q.size(); i++) {
    const size_t j = tb_chain(q, i);
    if (j - i < 2) continue;
    int ks, kw;
    if (!tb_pair(q[i], q[i + 1], &ks, &kw)) continue;
    tb_spare(rt().dats[q[i].acc[ks].dat]);
    tb_spare(rt().dats[q[i].acc[kw].dat]);
    i = j - 1;
  }
}

void tb_rename(ops_dat d, char *now) {
  DatX &x = rt().datx[d->index];
  char *old = d->data_d;
  d->data_d = now;
  x.spare = old;
}

/* Temporal-blocking depth autotuner (OPS_B200_TB_DEPTH=auto).  The first
 * chains of a loop's ping-pong sweeps run outside graphs, each with one of
 * the candidate depths (1: plain sweeps, no blocking) and bracketed by
 * events, kTbReps times per candidate; at the next flush the depth with the
 * least device time per sweep is kept for the rest of the run, and chains of
 * that loop are captured into graphs again.  Every depth computes every
 * point with the same code on the same values, so the choice changes no
 * result. */
constexpr int kTbDepths[] = {1, 2, 4, 8};
constexpr int kTbCands = (int)(sizeof kTbDepths / sizeof kTbDepths[0]);
constexpr int kTbReps = 2;

void tb_decide(KStat &k) {
  std::vector<double> best(kTbCands, 1e300);
  for (int c = 0; c < kTbCands * kTbReps && 2 * c + 1 < (int)k.tb_ev.size(); c++) {
    float ms = 0.f;
    if (!k.tb_ev[2 * c] || ob2_event_elapsed_ms(k.tb_ev[2 * c], k.tb_ev[2 * c + 1], &ms)) continue;
    best[c % kTbCands] =
        std::min(best[c % kTbCands], ms / (double)std::max(1LL, k.tb_sw[c]));
  }
  int bi = 0;
  for (int c = 1; c < kTbCands; c++)
    if (best[c] < best[bi]) bi = c;
  k.tb_best = kTbDepths[bi];
  for (void *e : k.tb_ev)
    if (e) rt().ev_pool.push_back(e);
  k.tb_ev.clear();
  k.tb_sw.clear();
  k.tb_state = 2;
}

// true when the queue holds a ping-pong chain whose depth is still being
// tuned (the flush then runs it outside a graph, timed); decides the loops
// whose candidates have all been timed
bool tb_tuning(std::vector<Runtime::QItem> &q) {
  Runtime &r = rt();
  if (!r.tb_auto) return false;
  for (size_t i = 0; i < q.size(); i++) {
    if (q[i].kind != 0 || !q[i].tfn) continue;
    const size_t j = tb_chain(q, i);
    if (j - i < 2) continue;
    KStat &k = r.kstats[q[i].kidx];
    if (k.tb_state == 1) {
      check(ob2_dev_sync(), "temporal-blocking depth tuning");
      tb_decide(k);
    }
    if (k.tb_state == 0) return true;
    i = j - 1;
  }
  return false;
}

int tb_depth_of(const Runtime::QItem &F) {
  Runtime &r = rt();
  if (!r.tb_auto) return r.tb_depth;
  const KStat &k = r.kstats[F.kidx];
  return k.tb_state == 2 ? k.tb_best : kTbDepths[k.tb_next % kTbCands];
}

void run_tb_sweeps(std::vector<Runtime::QItem> &q, size_t i, size_t j, int depth);

void run_tb(std::vector<Runtime::QItem> &q, size_t i, size_t j) {
  Runtime &r = rt();
  const int depth = tb_depth_of(q[i]);
  KStat &k = r.kstats[q[i].kidx];
  const bool timed = r.tb_auto && k.tb_state == 0 && !r.capturing;
  void *e0 = nullptr;
  if (timed) {
    e0 = pool_event();
    check(ob2_event_record(e0), "event");
  }
  run_tb_sweeps(q, i, j, depth);
  if (timed) {
    void *e1 = pool_event();
    check(ob2_event_record(e1), "event");
    k.tb_ev.push_back(e0);
    k.tb_ev.push_back(e1);
    k.tb_sw.push_back((long long)(j - i));
    if (++k.tb_next == kTbCands * kTbReps) k.tb_state = 1;
  }
}

void run_tb_sweeps(std::vector<Runtime::QItem> &q, size_t i, size_t j, int depth) {
  Runtime &r = rt();
  if (depth < 2) {  // plain sweeps: every item as queued
    for (size_t a = i; a < j; a++) run_item(q[a], nullptr, nullptr);
    return;
  }
  size_t a = i;
  while (a < j) {
    int ks = -1, kw = -1;
    // the pair relation of a piece's first sweep with its successor (or,
    // for the last item, with its predecessor read backwards)
    if (a + 1 < j) {
      tb_pair(q[a], q[a + 1], &ks, &kw);
    } else {
      run_item(q[a], nullptr, nullptr);  // one sweep left: as it is
      break;
    }
    const size_t b = std::min(j, a + (size_t)depth);
    Runtime::QItem &F = q[a];
    ops_dat X = r.dats[F.acc[ks].dat];
    DatX &xx = r.datx[X->index];
    const int argS = F.acc_arg[ks];
    char *vs;
    memcpy(&vs, F.prm.data() + F.tb_off[argS], sizeof vs);
    ob2_tblock t;
    memset(&t, 0, sizeof t);
    t.steps = (int)(b - a);
    t.s = argS;
    t.spare = xx.spare + (vs - X->data_d);
    t.sx0 = X->base[0] + X->d_m[0];
    t.sx1 = t.sx0 + X->size[0];
    t.sy0 = X->base[1] + X->d_m[1];
    t.sy1 = t.sy0 + X->size[1];
    void *ev = r.capturing ? nullptr : kt_begin();
    check(F.tfn(F.prm.data(), &t, ob2_dev_stream()), "ops_par_loop launch (temporal blocking)");
    kt_end(ev, F.kidx);
    r.launches++;
    r.tb_launches++;
    r.tb_sweeps += t.steps;
    // X's storage is now the spare; later sweeps of the chain address it there
    char *old = X->data_d, *now = xx.spare;
    tb_rename(X, now);
    if (r.rename_log) r.rename_log->push_back({(long long)X->index, (long long)old, (long long)now});
    for (size_t k = b; k < j; k++) {
      Runtime::QItem &K = q[k];
      for (size_t e = 0; e < K.acc.size(); e++) {
        if (K.acc[e].dat != X->index) continue;
        char *v;
        memcpy(&v, K.prm.data() + K.tb_off[K.acc_arg[e]], sizeof v);
        v = now + (v - old);
        memcpy(K.prm.data() + K.tb_off[K.acc_arg[e]], &v, sizeof v);
      }
    }
    a = b;
  }
}

void run_queue(std::vector<Runtime::QItem> &q) {
  Runtime &r = rt();
  size_t i = 0;
  while (i < q.size()) {
    if (q[i].kind == 0 && q[i].tfn) {
      const size_t j = tb_chain(q, i);
      if (j - i >= 2) {
        run_tb(q, i, j);
        i = j;
        continue;
      }
    }
    if (q[i].kind == 1 && i + 1 < q.size() && q[i + 1].kind == 0 && !r.tiling) {
      const size_t j = multi_run(q, i + 1);
      ob2_hfuse h;
      if (hfuse_plan(q, i, i + 1, j, h)) {
        run_hfused(q, i + 1, j, h);
        i = j;
        continue;
      }
    }
    if (r.tiling && tileable(q[i])) {
      size_t j = i + 1;
      while (j < q.size() && tileable(q[j]) && q[j].ndim == q[i].ndim) j++;
      if (j - i >= 2) {
        run_tiled(q, i, j);
        i = j;
        continue;
      }
    }
    if (q[i].kind == 0) {
      size_t j = multi_run(q, i);
      if (j - i >= 2) {
        run_multi(q, i, j);
        i = j;
        continue;
      }
      j = fuse_run(q, i);
      if (j - i >= 2) {
        run_fused(q, i, j);
        i = j;
        continue;
      }
    }
    run_item(q[i], nullptr, nullptr);
    i++;
  }
}

}  // namespace

/* run everything queued (no-op in eager mode) */
OPS_API void ob2_flush(void) {
  if (!R) return;
  Runtime &r = rt();
  if (r.q.empty()) return;
  std::vector<Runtime::QItem> q;
  q.swap(r.q);
  r.chains++;
  // per-kernel event timing and depth tuning need plain launches
  if (!r.graphs || r.ktime || tb_tuning(q)) {
    tb_prepare(q);
    run_queue(q);
    return;
  }
  // shape: everything that fixes the graph's topology and launch shapes;
  // exact: the shape plus every kernel parameter block (gbl values, dat
  // pointers, ranges).  Same exact key: replay.  Same shape only (typically
  // new ops_arg_gbl values such as a time step): re-capture and update the
  // executable graph in place, which skips instantiation.
  std::string shape, params;
  auto put = [&shape](const void *p, size_t n) { shape.append((const char *)p, n); };
  put(&r.tiling, sizeof r.tiling);
  put(&r.tile_y, sizeof r.tile_y);
  put(&r.tile_z, sizeof r.tile_z);
  put(&r.cache_mb, sizeof r.cache_mb);
  for (auto &it : q) {
    put(&it.kind, sizeof it.kind);
    put(&it.fn, sizeof it.fn);
    put(&it.mfn, sizeof it.mfn);
    put(&it.ffn, sizeof it.ffn);
    put(&it.fid, sizeof it.fid);
    put(&it.hfn, sizeof it.hfn);
    put(&it.group, sizeof it.group);
    const size_t np = it.prm.size();
    put(&np, sizeof np);
    put(it.grid, sizeof it.grid);
    put(it.block, sizeof it.block);
    put(&it.py, sizeof it.py);
    put(it.lo, sizeof it.lo);
    put(it.hi, sizeof it.hi);
    put(&it.tasks, sizeof it.tasks);
    put(&it.ntasks, sizeof it.ntasks);
    put(&it.max_pts, sizeof it.max_pts);
    for (auto &a : it.acc) put(&a, sizeof a);
    params.append(it.prm.data(), np);
  }
  auto f = r.graph_cache.find(shape);
  if (f != r.graph_cache.end() && f->second.params == params) {
    r.graph_hits++;
    check(ob2_graph_launch(f->second.exec), "loop-chain graph launch");
    r.launches += f->second.kernels;
    const long long *st = f->second.stats;
    r.multi_launches += st[0];
    r.fused_launches += st[1];
    r.fused_loops += st[2];
    r.hfused += st[3];
    r.tb_launches += st[4];
    r.tb_sweeps += st[5];
    for (auto &rn : f->second.renames) {  // the storage swaps the chain makes
      ops_dat d = r.dats[rn[0]];
      if (d->data_d != (char *)rn[1])
        throw OPSException(OPS_RUNTIME_ERROR, "Error: temporal blocking replay out of step");
      tb_rename(d, (char *)rn[2]);
    }
    return;
  }
  tb_prepare(q);
  if (f == r.graph_cache.end() && r.graph_cache.size() >= 256) {
    check(ob2_dev_sync(), "graph cache");
    for (auto &kv : r.graph_cache) ob2_graph_destroy(kv.second.exec);
    r.graph_cache.clear();
  }
  Runtime::Graph &G = r.graph_cache[shape];  // exec == nullptr when new
  if (G.exec) r.graph_updates++;
  check(ob2_graph_begin_capture(), "loop-chain capture");
  const long long l0 = r.launches;
  const long long s0[6] = {r.multi_launches, r.fused_launches, r.fused_loops, r.hfused,
                           r.tb_launches, r.tb_sweeps};
  r.capturing = true;
  std::vector<std::array<long long, 3>> renames;
  r.rename_log = &renames;
  try {
    run_queue(q);
  } catch (...) {
    r.rename_log = nullptr;
    r.capturing = false;
    void *dummy = nullptr;
    ob2_graph_end_capture(&dummy);
    if (dummy) ob2_graph_destroy(dummy);
    if (!G.exec) r.graph_cache.erase(shape);
    throw;
  }
  r.capturing = false;
  r.rename_log = nullptr;
  G.renames.swap(renames);
  int e = ob2_graph_end_capture(&G.exec);
  if (e) {
    r.graph_cache.erase(shape);
    check(e, "loop-chain capture");
  }
  G.kernels = r.launches - l0;
  const long long s1[6] = {r.multi_launches, r.fused_launches, r.fused_loops, r.hfused,
                           r.tb_launches, r.tb_sweeps};
  for (int k = 0; k < 6; k++) G.stats[k] = s1[k] - s0[k];
  G.params.swap(params);
  check(ob2_graph_launch(G.exec), "loop-chain graph launch");
}

OPS_API void ob2_launch(ob2_loop *L, ob2_launcher fn, ob2_mlauncher mfn, const void *params,
                        size_t psize, const unsigned *grid, const unsigned *block,
                        int rows_per_thread) {
  Runtime &r = rt();
  bool reduce = false;
  for (int i = 0; i < L->nargs; i++)
    if (L->red[i].acc) reduce = true;
  if (!r.lazy || reduce || L->tune >= 0) {
    ob2_flush();
    void *ev = kt_begin();
    void *t0 = nullptr, *t1 = nullptr;
    if (L->tune >= 0) {
      t0 = pool_event();
      ob2_event_record(t0);
    }
    int e = fn(params, grid, block, L->stream);
    if (L->tune >= 0) {
      t1 = pool_event();
      ob2_event_record(t1);
      KStat &k = r.kstats[L->kernel_index];
      k.tune_ev[2 * L->tune] = t0;
      k.tune_ev[2 * L->tune + 1] = t1;
    }
    kt_end(ev, L->kernel_index);
    if (e) {
      OPSException ex(OPS_RUNTIME_ERROR);
      ex << "Error: kernel launch of ops_par_loop " << L->name
         << " failed: " << ob2_error_string(e);
      throw ex;
    }
    r.launches++;
    return;
  }
  Runtime::QItem it;
  it.kind = 0;
  it.fn = fn;
  it.mfn = mfn;
  it.ffn = L->ffn;
  it.fid = L->fuse_id;
  it.idx32 = L->idx32;
  it.npts = L->npoints;
  it.prm.assign((const char *)params, (const char *)params + psize);
  for (int i = 0; i < 3; i++) {
    it.grid[i] = grid[i];
    it.block[i] = block[i];
    it.lo[i] = L->lo[i];
    it.hi[i] = L->hi[i];
  }
  it.py = rows_per_thread;
  it.ndim = L->dim;
  it.kidx = L->kernel_index;
  it.tasks = nullptr;
  it.ntasks = 0;
  it.max_pts = 0;
  it.group = -1;
  it.hfn = L->hfn;
  it.tfn = L->tfn;
  it.tb_off = L->tb_off;
  it.tb_role = L->tb_role;
  const int td = L->dim - 1;
  for (int i = 0; i < L->nargs; i++) {
    ops_arg &a = L->args[i];
    if (a.argtype != OPS_ARG_DAT || !a.dat) continue;
    Runtime::QAcc qa;
    qa.dat = a.dat->index;
    qa.acc = a.acc;
    qa.rmin = qa.rmax = 0;
    qa.flat = (a.stencil && a.stencil->stride[td] == 0) ? 1 : 0;
    if (a.stencil)
      for (int p = 0; p < a.stencil->points; p++) {
        const int o = td < a.stencil->dims ? a.stencil->stencil[p * a.stencil->dims + td] : 0;
        qa.rmin = std::min(qa.rmin, o);
        qa.rmax = std::max(qa.rmax, o);
      }
    // for the footprint test of fused launches: the stencil and its strides
    qa.any = 0;
    qa.sidx = a.stencil ? a.stencil->index : -1;
    for (int k = 0; k < 3; k++) {
      const int st = a.stencil ? a.stencil->stride[k] : 1;
      qa.sx[k] = st;
      if (st != 0 && st != 1) qa.any = 1;
    }
    if (a.stencil && a.stencil->points > 32) qa.any = 1;  // keeps the test short
    qa.mg = (a.stencil && a.stencil->type != 0) ? 1 : 0;  // restrict / prolong
    if (qa.mg) qa.any = 1;
    it.acc.push_back(qa);
    it.acc_arg.push_back(i);
  }
  r.q.push_back(std::move(it));
  if (r.max_chain > 0 && (int)r.q.size() >= r.max_chain) ob2_flush();
}

OPS_instance *OPS_instance::getOPSInstance() { return &I(); }

OPS_API void ob2_adopt_instance(OPS_instance *inst, int argc, const char *const *argv,
                                int diags) {
  Runtime &r = rt();
  if (r.user && r.user != inst)
    throw OPSException(OPS_INVALID_ARGUMENT, "Error: only one OPS_instance per process");
  r.user = inst;
  ops_init(argc, argv, diags);
}

OPS_API void ob2_release_instance(OPS_instance *inst) {
  if (!R || rt().user != inst) return;
  ops_exit();
  rt().user = nullptr;
}

/* ------------------------------------------------------------------------
 * init / exit  (ops_lib_core.cpp:100-275; ops_cuda_common.cu:68-182)
 * ---------------------------------------------------------------------- */
/* ------------------------------------------------------------------------
 * Communicator registration and the runtime's own NCCL transport
 * (OPS_B200_DIST=nccl: RANK / WORLD_SIZE from the launcher, NCCL loaded at
 * run time, its unique id passed through a file named after MASTER_ADDR /
 * MASTER_PORT; rows go GPU to GPU with ncclSend / ncclRecv and reduction
 * results are combined with ncclAllReduce, all on the work stream).
 * ---------------------------------------------------------------------- */
OPS_API int ob2_dist_init(const ob2_dist_comm *c) {
  Runtime &r = rt();
  if (!c || c->size < 1 || c->rank < 0 || c->rank >= c->size ||
      (c->size > 1 && (!c->sendrecv || !c->allreduce)))
    return OPS_INVALID_ARGUMENT;
  if (r.initialised && !r.dats.empty()) return OPS_INVALID_ARGUMENT;  // before any dat
  r.comm = *c;
  r.dist = c->size > 1;
  return 0;
}
OPS_API int ob2_dist_rank(void) { return rt().comm.rank; }
OPS_API int ob2_dist_size(void) { return rt().comm.size; }

namespace {
struct NcclApi {  // the few NCCL entry points used, resolved with dlsym
  void *h = nullptr;
  void *comm = nullptr;
  int (*get_id)(void *id) = nullptr;
  int (*init_rank)(void **comm, int n, char id[128], int rank) = nullptr;
  int (*group_start)() = nullptr;
  int (*group_end)() = nullptr;
  int (*send)(const void *, size_t, int, int, void *, void *) = nullptr;
  int (*recv)(void *, size_t, int, int, void *, void *) = nullptr;
  int (*allreduce)(const void *, void *, size_t, int, int, void *, void *) = nullptr;
};
NcclApi g_nccl;

// NCCL's enum values (nccl.h): ncclChar 0, ncclInt32 2, ncclInt64 4,
// ncclFloat32 7, ncclFloat64 8; ncclSum 0, ncclMax 2, ncclMin 3
int nccl_sendrecv(void *, const void *sbuf, size_t sb, int sp, void *rbuf, size_t rbn, int rp) {
  NcclApi &n = g_nccl;
  void *st = ob2_dev_stream();
  int e = n.group_start();
  if (!e && sb && sp >= 0) e = n.send(sbuf, sb, 0, sp, n.comm, st);
  if (!e && rbn && rp >= 0) e = n.recv(rbuf, rbn, 0, rp, n.comm, st);
  const int e2 = n.group_end();
  return e ? e : e2;
}
int nccl_allreduce(void *, void *buf, int count, int type, int op) {
  static const int types[4] = {8, 7, 2, 4};
  const int o = op == OPS_MAX ? 2 : (op == OPS_MIN ? 3 : 0);
  if (type < 0 || type > 3) return -1;
  return g_nccl.allreduce(buf, buf, (size_t)count, types[type], o, g_nccl.comm, ob2_dev_stream());
}

int nccl_setup() {
  const char *rk = getenv("RANK"), *ws = getenv("WORLD_SIZE");
  if (!rk || !ws) return -1;
  const int rank = atoi(rk), size = atoi(ws);
  NcclApi &n = g_nccl;
  n.h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!n.h) return -2;
  n.get_id = (int (*)(void *))dlsym(n.h, "ncclGetUniqueId");
  n.init_rank = (int (*)(void **, int, char *, int))dlsym(n.h, "ncclCommInitRank");
  n.group_start = (int (*)())dlsym(n.h, "ncclGroupStart");
  n.group_end = (int (*)())dlsym(n.h, "ncclGroupEnd");
  n.send = (int (*)(const void *, size_t, int, int, void *, void *))dlsym(n.h, "ncclSend");
  n.recv = (int (*)(void *, size_t, int, int, void *, void *))dlsym(n.h, "ncclRecv");
  n.allreduce = (int (*)(const void *, void *, size_t, int, int, void *, void *))dlsym(
      n.h, "ncclAllReduce");
  if (!n.get_id || !n.init_rank || !n.group_start || !n.group_end || !n.send || !n.recv ||
      !n.allreduce)
    return -3;
  const char *ma = getenv("MASTER_ADDR"), *mp = getenv("MASTER_PORT");
  std::string path = std::string("/tmp/ob2_nccl_id_") + (ma ? ma : "local") + "_" + (mp ? mp : "0");
  char id[128];
  if (rank == 0) {  // written whole, then renamed into place
    if (n.get_id(id)) return -4;
    std::string tmp = path + ".tmp";
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f || fwrite(id, 1, 128, f) != 128) return -5;
    fclose(f);
    if (rename(tmp.c_str(), path.c_str())) return -5;
  } else {  // bounded wait for rank 0's id
    bool ok = false;
    for (int t = 0; t < 1200 && !ok; t++) {
      FILE *f = fopen(path.c_str(), "rb");
      if (f) {
        ok = fread(id, 1, 128, f) == 128;
        fclose(f);
      }
      if (!ok) usleep(100000);
    }
    if (!ok) return -6;
  }
  if (n.init_rank(&n.comm, size, id, rank)) return -7;
  ob2_dist_comm c = {rank, size, 1, nullptr, nccl_sendrecv, nccl_allreduce};
  return ob2_dist_init(&c);
}
}  // namespace

OPS_API void ops_init(const int argc, const char *const argv[], const int diags) {
  Runtime &r = rt();
  I().OPS_diags = diags;
  I().OPS_hybrid_gpu = 1;
  for (int i = 0; i < argc; i++) {
    if (!argv || !argv[i]) continue;
    const char *a = argv[i];
    const char *p;
    if ((p = strstr(a, "-OPS_DIAGS="))) I().OPS_diags = atoi(p + 11);
    if ((p = strstr(a, "OPS_BLOCK_SIZE_X="))) r.block_x = atoi(p + 17);
    if ((p = strstr(a, "OPS_BLOCK_SIZE_Y="))) r.block_y = atoi(p + 17);
    if ((p = strstr(a, "OPS_BLOCK_SIZE_Z="))) r.block_z = atoi(p + 17);
    if ((p = strstr(a, "OPS_DEVICE="))) r.device = atoi(p + 11);
    // loop-chain tiling (ops_lib_core.cpp:132-180): lazy queue + tiles
    if (strstr(a, "OPS_TILING")) r.lazy = r.tiling = true;
    if ((p = strstr(a, "OPS_TILESIZE_Y="))) r.tile_y = atoi(p + 15);
    if ((p = strstr(a, "OPS_TILESIZE_Z="))) r.tile_z = atoi(p + 15);
    if ((p = strstr(a, "OPS_CACHE_SIZE="))) r.cache_mb = atof(p + 15);
    if (strstr(a, "OPS_AUTOTUNE")) r.autotune = true;
  }
  const char *e;
  if ((e = getenv("OPS_B200_LAZY"))) r.lazy = atoi(e) != 0;
  if ((e = getenv("OPS_B200_TILING"))) r.tiling = atoi(e) != 0;
  if (r.tiling) r.lazy = true;
  if ((e = getenv("OPS_B200_GRAPHS"))) r.graphs = atoi(e) != 0;
  if ((e = getenv("OPS_B200_TILESIZE_Y"))) r.tile_y = atoi(e);
  if ((e = getenv("OPS_B200_TILESIZE_Z"))) r.tile_z = atoi(e);
  if ((e = getenv("OPS_B200_CACHE_MB"))) r.cache_mb = atof(e);
  if ((e = getenv("OPS_B200_MAX_CHAIN"))) r.max_chain = atoi(e);
  if ((e = getenv("OPS_B200_RED_WAVES"))) r.red_waves = std::max(1, atoi(e));
  if ((e = getenv("OPS_B200_AUTOTUNE"))) r.autotune = atoi(e) != 0;
  if ((e = getenv("OPS_B200_MULTI"))) r.multi = atoi(e) != 0;
  if ((e = getenv("OPS_B200_FUSE"))) r.fuse = atoi(e) != 0;
  if ((e = getenv("OPS_B200_HFUSE"))) r.hfuse = atoi(e) != 0;
  if ((e = getenv("OPS_B200_TB"))) r.tb = atoi(e) != 0;
  if ((e = getenv("OPS_B200_TB_DEPTH"))) {
    if (!strcmp(e, "auto"))
      r.tb_auto = true;
    else
      r.tb_depth = std::max(2, std::min(OB2_TB_MAX, atoi(e)));
  }
  if ((e = getenv("OPS_B200_FUSE_PTS"))) r.fuse_pts = atoll(e);
  if ((e = getenv("OPS_B200_TUNE_FILE")) && *e) {
    r.tune_file = e;
    if (FILE *f = fopen(e, "r")) {  // decisions of an earlier run
      char nm[256];
      int bx, by, bz;
      while (fscanf(f, "%255s %d %d %d", nm, &bx, &by, &bz) == 4)
        if (bx > 0 && by > 0 && bz > 0 && bx * by * bz <= 1024)
          r.tune_known[nm] = {bx, by, bz};
      fclose(f);
    }
  }
  if (r.cache_mb <= 0.0) r.cache_mb = 40.0;
  if ((e = getenv("OPS_B200_DEVICE"))) r.device = atoi(e);
  else if ((e = getenv("OPS_B200_DIST")) && !strcmp(e, "nccl") && getenv("LOCAL_RANK"))
    r.device = atoi(getenv("LOCAL_RANK"));  // one process per GPU
  if ((e = getenv("OPS_B200_BLOCK"))) sscanf(e, "%d,%d,%d", &r.block_x, &r.block_y, &r.block_z);
  if (r.block_x < 1) r.block_x = 32;
  if (r.block_y < 1) r.block_y = 1;
  if (r.block_z < 1) r.block_z = 1;
  // diagnostics above 1: per-kernel device times in the timing table
  if (I().OPS_diags > 1) r.ktime = true;
  if (r.initialised) return;
  check(ob2_dev_init(r.device), "ops_init (no usable CUDA device)");
  if ((e = getenv("OPS_B200_DIST")) && !strcmp(e, "nccl") && !r.dist) {
    const int ne = nccl_setup();  // one process per GPU, rank and size from the launcher
    if (ne) {
      OPSException ex(OPS_RUNTIME_ERROR);
      ex << "Error: OPS_B200_DIST=nccl: NCCL communicator set-up failed (" << ne << ")";
      throw ex;
    }
  }
  check(ob2_dev_sm_count(&r.sms), "ops_init");
  check(ob2_dev_malloc((void **)&r.counter, 4096), "ops_init");
  check(ob2_dev_memset(r.counter, 0, 4096), "ops_init");
  r.initialised = true;
}

OPS_API void ops_dump_dats(const char *path);

OPS_API void ops_exit(void) {
  if (!R || !R->initialised) return;
  ob2_flush();
  Runtime &r = rt();
  if (r.autotune && !r.tune_file.empty()) {
    ob2_dev_sync();
    if (FILE *f = fopen(r.tune_file.c_str(), "w")) {
      for (auto &k : r.kstats) {
        if (k.tune_state == 1) tune_decide(k, k.tune_dim);
        if (k.tune_state == 2)
          fprintf(f, "%s %d %d %d\n", k.name.c_str(), k.best[0], k.best[1], k.best[2]);
      }
      fclose(f);
    }
  }
  const char *dump = getenv("OPS_DUMP_FILE");
  if (dump && *dump) ops_dump_dats(dump);
  ob2_dev_sync();
}

OPS_API void ops_set_soa(const int soa) { I().OPS_soa = soa; }

OPS_API ops_block ops_decl_block(int dims, const char *name) {
  if (dims < 1 || dims > OPS_MAX_DIM)
    throw OPSException(OPS_INVALID_ARGUMENT,
                       "Error: ops_decl_block -- this backend supports 1D to 5D blocks");
  ops_block b = (ops_block)calloc(1, sizeof(ops_block_core));
  b->dims = dims;
  b->name = copy_str(name);
  b->instance = &I();
  b->index = (int)rt().blocks.size();
  rt().blocks.push_back(b);
  return b;
}

/* ------------------------------------------------------------------------
 * dats (ops_lib_core.cpp:445-601; ops_device_singlenode_common.cpp:45-106)
 * ---------------------------------------------------------------------- */
OPS_API ops_dat ops_decl_dat_char(ops_block block, int dim, int *size, int *base, int *d_m,
                                  int *d_p, int *stride, char *data, int type_size,
                                  char const *type, char const *name) {
  require_init();
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
    if (d_m[n] > 0) {
      OPSException ex(OPS_INVALID_ARGUMENT);
      ex << "Error: ops_decl_dat -- Non negative d_m during declaration of: " << name;
      throw ex;
    }
    if (d_p[n] < 0) {
      OPSException ex(OPS_INVALID_ARGUMENT);
      ex << "Error: ops_decl_dat -- Non positive d_p during declaration of: " << name;
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
  DatX dxn;
  d->index = (int)rt().dats.size();
  if (dist_layout(d, dxn)) {  // this rank's rows only; data_d addresses them globally
    check(ob2_dev_malloc((void **)&dxn.alloc, dxn.alloc_bytes), "ops_decl_dat (device allocation)");
    d->data_d = dxn.alloc - (size_t)dxn.s_lo * dxn.row_bytes;
    if (data) {
      d->data = data;
      d->user_managed = 1;
      check(ob2_dev_h2d(dxn.alloc, data + (size_t)dxn.s_lo * dxn.row_bytes, dxn.alloc_bytes),
            "ops_decl_dat (upload)");
    } else {
      d->data = nullptr;
      d->user_managed = 0;
      check(ob2_dev_memset(dxn.alloc, 0, dxn.alloc_bytes), "ops_decl_dat (zero)");
    }
  } else {
  check(ob2_dev_malloc((void **)&d->data_d, d->mem), "ops_decl_dat (device allocation)");
  if (data) {
    d->data = data;
    d->user_managed = 1;
    check(ob2_dev_h2d(d->data_d, data, d->mem), "ops_decl_dat (upload)");
  } else {
    d->data = nullptr;
    d->user_managed = 0;
    check(ob2_dev_memset(d->data_d, 0, d->mem), "ops_decl_dat (zero)");
  }
  }
  d->dirty_hd = data ? 0 : 2;
  long long off = 0, cum = 1;
  for (int i = 0; i < block->dims; i++) {
    off += (long long)(I().OPS_soa ? d->type_size : d->elem_size) * cum *
           (-d->base[i] - d->d_m[i]);
    cum *= d->size[i];
  }
  d->base_offset = (size_t)off;
  rt().dats.push_back(d);
  rt().datx.push_back(dxn);
  return d;
}

OPS_API void ops_free_dat(ops_dat d) {
  if (!d) return;
  ob2_flush();
  ob2_dev_sync();
  for (auto &p : rt().dats)
    if (p == d) p = nullptr;
  {
    DatX &x = rt().datx[d->index];
    ob2_dev_free(x.split ? x.alloc : d->data_d);
    if (x.spare) ob2_dev_free(x.spare);
  }
  if (!d->user_managed) free(d->data);
  free(d);
}

OPS_API void ops_dat_deep_copy(ops_dat target, ops_dat src) {
  if (rt().dist && (rt().datx[src->index].split || rt().datx[target->index].split))
    dist_unsupported(src, "ops_dat_deep_copy");
  require_init();
  ob2_flush();
  if (target->data_d && target->mem != src->mem) {
    ob2_dev_sync();
    ob2_dev_free(target->data_d);
    target->data_d = nullptr;
  }
  if (!target->data_d) check(ob2_dev_malloc((void **)&target->data_d, src->mem), "deep copy");
  if (target->data && !target->user_managed) free(target->data);
  char *dd = target->data_d;
  int idx = target->index;
  ops_block blk = target->block ? target->block : src->block;
  memcpy(target, src, sizeof(ops_dat_core));
  target->data_d = dd;
  target->data = nullptr;
  target->user_managed = 0;
  target->index = idx;
  target->block = blk;
  // the copy is renamed to the source name + "_copy", cut to strlen(name) + 4
  // characters as in ops_lib_core.cpp:2280-2281 (so "u" becomes "u_cop")
  {
    size_t nl = strlen(src->name) + 5;
    char *nm = (char *)malloc(nl + 1);
    snprintf(nm, nl, "%s_copy", src->name);
    target->name = nm;
  }
  target->type = copy_str(src->type);
  put_data(src);
  check(ob2_dev_d2d(target->data_d, src->data_d, src->mem), "deep copy");
  target->dirty_hd = 2;
  target->locked_hd = 0;
}

OPS_API ops_dat ops_dat_copy(ops_dat src) {
  ops_dat d = (ops_dat)calloc(1, sizeof(ops_dat_core));
  d->block = src->block;
  d->index = (int)rt().dats.size();
  rt().dats.push_back(d);
  rt().datx.push_back(DatX());
  ops_dat_deep_copy(d, src);
  return d;
}

/* ------------------------------------------------------------------------
 * args (ops_lib_core.cpp:856-1105)
 * ---------------------------------------------------------------------- */
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
    a.data_d = dat->data_d;
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
    int tc = type_code(type);
    int ts = type_bytes(tc);
    for (int off = 0; off + ts <= h->size; off += ts) identity_bytes(tc, acc, h->data + off, false);
    rt().redx[h->index].pending_first = 1;
  } else if (h->acc != acc) {
    OPSException ex(OPS_INVALID_ARGUMENT);
    ex << "Error: ops_reduction handle " << h->name
       << " was already used with a different access type";
    throw ex;
  }
  return a;
}

OPS_API ops_reduction ops_decl_reduction_handle(int size, const char *type, const char *name) {
  require_init();
  ops_reduction r = (ops_reduction)calloc(1, sizeof(ops_reduction_core));
  r->size = size;
  r->data = (char *)calloc(size, 1);
  r->type = copy_str(type);
  r->name = copy_str(name);
  r->instance = &I();
  r->index = (int)rt().reds.size();
  rt().reds.push_back(r);
  RedX x;
  check(ob2_dev_malloc(&x.acc_d, size > 0 ? size : 8), "ops_decl_reduction_handle");
  check(ob2_host_alloc_pinned(&x.host_pinned, size > 0 ? size : 8), "ops_decl_reduction_handle");
  rt().redx.push_back(x);
  return r;
}

/* ops_lib_core.cpp:1143-1149: forces execution, returns, resets the handle */
OPS_API void ops_reduction_result_char(ops_reduction h, int, char *ptr) {
  Runtime &r = rt();
  RedX &x = r.redx[h->index];
  if (!x.pending_first) {
    check(ob2_dev_d2h_async(x.host_pinned, x.acc_d, h->size), "ops_reduction_result");
    check(ob2_dev_sync(), "ops_reduction_result");
    memcpy(h->data, x.host_pinned, h->size);
  } else if (r.dist && h->initialized) {
    // no point of this rank's rows fed the handle: its part is the identity
    const int tc = type_code(h->type);
    const int ts = type_bytes(tc);
    for (int k = 0; k + ts <= h->size; k += ts) identity_bytes(tc, h->acc, h->data + k, false);
  }
  if (r.dist) {  // combined over the ranks (the reference's MPI_Allreduce)
    const int t = red_type(h->type);
    const int ts = t == 0 || t == 3 ? 8 : 4;
    if (t < 0) dist_unsupported(nullptr, "a reduction of this type");
    int e;
    if (r.comm.device) {
      check(ob2_dev_h2d(x.acc_d, h->data, h->size), "ops_reduction_result");
      e = r.comm.allreduce(r.comm.ctx, x.acc_d, h->size / ts, t, h->acc);
      if (!e) check(ob2_dev_d2h(h->data, x.acc_d, h->size), "ops_reduction_result");
    } else {
      e = r.comm.allreduce(r.comm.ctx, h->data, h->size / ts, t, h->acc);
    }
    if (e) throw OPSException(OPS_RUNTIME_ERROR, "Error: reduction over the ranks failed");
  }
  memcpy(ptr, h->data, h->size);
  x.pending_first = 0;
  h->initialized = 0;
}

/* ------------------------------------------------------------------------
 * stencils (ops_lib_core.cpp:640-836)
 * ---------------------------------------------------------------------- */
static ops_stencil make_stencil(int dims, int points, int *sten, int *stride, const char *name,
                                int type) {
  ops_stencil s = (ops_stencil)calloc(1, sizeof(ops_stencil_core));
  s->dims = dims;
  s->points = points;
  s->name = copy_str(name);
  s->stencil = (int *)malloc(sizeof(int) * (size_t)(dims * points > 0 ? dims * points : 1));
  if (dims * points > 0) memcpy(s->stencil, sten, sizeof(int) * dims * points);
  s->stride = (int *)malloc(sizeof(int) * OPS_MAX_DIM);
  s->mgrid_stride = (int *)malloc(sizeof(int) * OPS_MAX_DIM);
  for (int i = 0; i < OPS_MAX_DIM; i++) {
    s->stride[i] = (stride && i < dims) ? stride[i] : 1;
    s->mgrid_stride[i] = 1;
  }
  s->type = type;
  s->index = (int)rt().stencils.size();
  rt().stencils.push_back(s);
  return s;
}
OPS_API ops_stencil ops_decl_stencil(int dims, int points, int *sten, char const *name) {
  return make_stencil(dims, points, sten, nullptr, name, 0);
}
OPS_API ops_stencil ops_decl_strided_stencil(int dims, int points, int *sten, int *stride,
                                             char const *name) {
  return make_stencil(dims, points, sten, stride, name, 0);
}
// multigrid stencils (ops_lib_core.cpp:736-831): the stride is kept as the
// multigrid stride; type 2 restrict (the dat is read at index * stride, a
// finer dat from a coarser loop), type 1 prolong (at index / stride, a
// coarser dat from a finer loop); offsets are in the dat's own index space
static ops_stencil make_mgrid_stencil(int dims, int points, int *sten, int *stride,
                                      const char *name, int type) {
  if (!stride) throw OPSException(OPS_INVALID_ARGUMENT, "Error: multigrid stencil without stride");
  ops_stencil s = make_stencil(dims, points, sten, nullptr, name, type);
  for (int i = 0; i < dims && i < OPS_MAX_DIM; i++) {
    if (stride[i] < 1)
      throw OPSException(OPS_INVALID_ARGUMENT, "Error: multigrid stencil stride must be >= 1");
    s->mgrid_stride[i] = stride[i];
  }
  return s;
}
OPS_API ops_stencil ops_decl_restrict_stencil(int dims, int points, int *sten, int *stride,
                                              char const *name) {
  return make_mgrid_stencil(dims, points, sten, stride, name, 2);
}
OPS_API ops_stencil ops_decl_prolong_stencil(int dims, int points, int *sten, int *stride,
                                             char const *name) {
  return make_mgrid_stencil(dims, points, sten, stride, name, 1);
}

/* ------------------------------------------------------------------------
 * halos (ops_lib_core.cpp:967-1045; ops_device_singlenode_common.cpp:262-346)
 * ---------------------------------------------------------------------- */
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
  h->index = (int)rt().halos.size();
  rt().halos.push_back(h);
  return h;
}

OPS_API ops_halo_group ops_decl_halo_group(int nhalos, ops_halo *halos) {
  ops_halo_group g = (ops_halo_group)calloc(1, sizeof(ops_halo_group_core));
  g->nhalos = nhalos;
  g->halos = (ops_halo *)malloc(sizeof(ops_halo) * (nhalos > 0 ? nhalos : 1));
  for (int i = 0; i < nhalos; i++) g->halos[i] = halos[i];
  g->instance = &I();
  g->index = (int)rt().groups.size();
  rt().groups.push_back(g);
  rt().groupx.push_back(GroupX());
  return g;
}

static void build_halo_tasks(ops_halo_group g, GroupX &gx) {
  std::vector<ob2_halo_task> tasks;
  gx.key.clear();
  gx.max_pts = 0;
  gx.src_dat.clear();
  gx.dst_dat.clear();
  gx.org.clear();
  gx.dlo.clear();
  gx.dhi.clear();
  for (int hh = 0; hh < g->nhalos; hh++) {
    ops_halo h = g->halos[hh];
    // 4D / 5D blocks: the box is cut into 3D boxes, one per index along the
    // 4th and 5th axes, which must map onto themselves (flips allowed)
    int hi_iter[2] = {1, 1};
    for (int i = 3; i < OPS_MAX_DIM; i++) {
      hi_iter[i - 3] = h->iter_size[i];
      if (h->iter_size[i] != 1 &&
          (abs(h->from_dir[i]) != i + 1 || abs(h->to_dir[i]) != i + 1))
        throw OPSException(OPS_NOT_IMPLEMENTED,
                           "Error: a halo whose 4th or 5th axis maps onto another axis");
    }
    if (h->from->dim != h->to->dim)
      throw OPSException(OPS_INVALID_ARGUMENT,
                         "Error: ops_halo_transfer between dats of different dim");
    ob2_halo_task t;
    memset(&t, 0, sizeof(t));
    t.src = h->from->data_d;
    t.dst = h->to->data_d;
    t.src_type = h->from->type_size;
    t.dst_type = h->to->type_size;
    if (t.src_type != t.dst_type) {
      // mixed float / double / half transfers convert each value to the
      // destination type (ops_host_singlenode.cpp:224-228, through the
      // smaller of the two types, which equals the direct conversion)
      auto fp = [](const char *t) {
        return !strcmp(t, "double") || !strcmp(t, "float") || !strcmp(t, "half");
      };
      bool okf = fp(h->from->type) && fp(h->to->type);
      if (!okf)
        throw OPSException(OPS_NOT_IMPLEMENTED, "Error: unsupported mixed-type halo transfer");
      t.float_kind = 1;
    }
    t.ncomp = h->from->dim;
    t.src_soa = t.dst_soa = I().OPS_soa;
    t.npts = 1;
    for (int a = 0; a < 3; a++) {
      t.iter[a] = h->iter_size[a];
      t.npts *= h->iter_size[a];
    }
    long long fc = 1, tc = 1;
    for (int i = 0; i < 3; i++) {
      t.src_axis[i] = abs(h->from_dir[i]) - 1;
      t.src_flip[i] = h->from_dir[i] < 0;
      t.src_start[i] = h->from_base[i] - h->from->d_m[i] - h->from->base[i];
      t.src_cum[i] = fc;
      fc *= h->from->size[i];
      t.dst_axis[i] = abs(h->to_dir[i]) - 1;
      t.dst_flip[i] = h->to_dir[i] < 0;
      t.dst_start[i] = h->to_base[i] - h->to->d_m[i] - h->to->base[i];
      t.dst_cum[i] = tc;
      tc *= h->to->size[i];
      if (t.src_axis[i] < 0 || t.src_axis[i] > 2 || t.dst_axis[i] < 0 || t.dst_axis[i] > 2)
        throw OPSException(OPS_INVALID_ARGUMENT, "Error: invalid halo direction");
    }
    t.src_npts_total = fc;
    t.dst_npts_total = tc;
    // bounds: every touched storage index must lie inside the dats
    for (int i = 0; i < 3; i++) {
      int fl = t.iter[t.src_axis[i]], tl = t.iter[t.dst_axis[i]];
      if (t.src_start[i] < 0 || t.src_start[i] + fl > h->from->size[i] || t.dst_start[i] < 0 ||
          t.dst_start[i] + tl > h->to->size[i]) {
        OPSException ex(OPS_INVALID_ARGUMENT);
        ex << "Error: halo " << hh << " of group " << g->index << " reaches outside dat "
           << h->from->name << " or " << h->to->name;
        throw ex;
      }
    }
    if (t.npts > gx.max_pts) gx.max_pts = t.npts;
    // storage index and point offset along the 4th and 5th axes
    long long hstart[2][2], hcum[2][2];
    for (int i = 3; i < OPS_MAX_DIM; i++) {
      hstart[0][i - 3] = h->from_base[i] - h->from->d_m[i] - h->from->base[i];
      hstart[1][i - 3] = h->to_base[i] - h->to->d_m[i] - h->to->base[i];
      hcum[0][i - 3] = fc;
      hcum[1][i - 3] = tc;
      fc *= h->from->size[i];
      tc *= h->to->size[i];
      if (hi_iter[i - 3] != 1 &&
          (hstart[0][i - 3] < 0 || hstart[0][i - 3] + hi_iter[i - 3] > h->from->size[i] ||
           hstart[1][i - 3] < 0 || hstart[1][i - 3] + hi_iter[i - 3] > h->to->size[i]))
        throw OPSException(OPS_INVALID_ARGUMENT, "Error: halo reaches outside its dats");
    }
    t.src_npts_total = fc;  // all axes: the component stride of SoA dats
    t.dst_npts_total = tc;
    for (int a4 = 0; a4 < hi_iter[1]; a4++)
      for (int a3 = 0; a3 < hi_iter[0]; a3++) {
        ob2_halo_task u = t;
        const int hi_a[2] = {a3, a4};
        long long soff = 0, doff = 0;
        for (int k = 0; k < 2; k++) {
          if (hi_iter[k] == 1 && h->iter_size[3 + k] == 1 &&
              h->from->block->dims <= 3 + k)
            continue;
          const int fi = h->from_dir[3 + k] < 0 ? hi_iter[k] - 1 - hi_a[k] : hi_a[k];
          const int ti = h->to_dir[3 + k] < 0 ? hi_iter[k] - 1 - hi_a[k] : hi_a[k];
          soff += (hstart[0][k] + fi) * hcum[0][k];
          doff += (hstart[1][k] + ti) * hcum[1][k];
        }
        // AoS: ncomp values per point; SoA: components npts_total apart
        u.src += soff * (u.src_soa ? 1 : u.ncomp) * u.src_type;
        u.dst += doff * (u.dst_soa ? 1 : u.ncomp) * u.dst_type;
        std::array<int, 3> og, lo, hi;
        for (int i = 0; i < 3; i++) {
          og[i] = h->to->d_m[i] + h->to->base[i];
          lo[i] = og[i] + u.dst_start[i];
          hi[i] = lo[i] + u.iter[u.dst_axis[i]];
        }
        gx.org.push_back(og);
        gx.dlo.push_back(lo);
        gx.dhi.push_back(hi);
        gx.src_dat.push_back(h->from->index);
        gx.dst_dat.push_back(h->to->index);
        tasks.push_back(u);
      }
    gx.key.push_back(h->from->data_d);
    gx.key.push_back(h->to->data_d);
  }
  if (gx.tasks_d) {
    ob2_dev_sync();
    ob2_dev_free(gx.tasks_d);
    gx.tasks_d = nullptr;
  }
  gx.ntasks = (int)tasks.size();
  if (gx.ntasks) {
    size_t bytes = sizeof(ob2_halo_task) * tasks.size();
    check(ob2_dev_malloc(&gx.tasks_d, bytes), "ops_halo_transfer");
    check(ob2_dev_h2d(gx.tasks_d, tasks.data(), bytes), "ops_halo_transfer");
  }
}

OPS_API void ops_halo_transfer(ops_halo_group g) {
  require_init();
  if (rt().dist) dist_unsupported(nullptr, "ops_halo_transfer between blocks");
  GroupX &gx = rt().groupx[g->index];
  bool stale = gx.key.size() != (size_t)2 * g->nhalos;
  for (int hh = 0; !stale && hh < g->nhalos; hh++)
    stale = gx.key[2 * hh] != g->halos[hh]->from->data_d ||
            gx.key[2 * hh + 1] != g->halos[hh]->to->data_d;
  if (stale) {
    ob2_flush();  // queued transfers may still use the old task table
    build_halo_tasks(g, gx);
  }
  for (int hh = 0; hh < g->nhalos; hh++) {
    put_data(g->halos[hh]->from);
    put_data(g->halos[hh]->to);
  }
  Runtime &r = rt();
  int k = kernel_slot("ops_halo_transfer");
  double t0 = wall();
  if (r.lazy && gx.ntasks) {
    // part of the loop chain: ordered with the queued loops, captured with
    // them into the chain's graph
    Runtime::QItem it;
    it.kind = 1;
    it.fn = nullptr;
    it.mfn = nullptr;
    for (int i = 0; i < 3; i++) it.grid[i] = it.block[i] = 1, it.lo[i] = it.hi[i] = 0;
    it.py = 1;
    it.ndim = 0;
    it.kidx = k;
    it.tasks = gx.tasks_d;
    it.ntasks = gx.ntasks;
    it.max_pts = gx.max_pts;
    it.group = g->index;
    it.hfn = nullptr;
    it.tfn = nullptr;
    it.tb_off = nullptr;
    it.tb_role = nullptr;
    it.ffn = nullptr;
    it.fid = -1;
    it.idx32 = 0;
    it.npts = 0;
    r.q.push_back(std::move(it));
    if (r.max_chain > 0 && (int)r.q.size() >= r.max_chain) ob2_flush();
  } else {
    ob2_flush();
    void *ev = kt_begin();
    check(ob2_halo_run((const ob2_halo_task *)gx.tasks_d, gx.ntasks, gx.max_pts),
          "ops_halo_transfer");
    kt_end(ev, k);
    r.launches++;
  }
  KStat &s = r.kstats[k];
  s.count++;
  s.host_s += wall() - t0;
  for (int hh = 0; hh < g->nhalos; hh++) {
    ops_halo h = g->halos[hh];
    h->to->dirty_hd = 2;
    s.transfer += 2.0 * (double)h->from->elem_size * h->iter_size[0] * h->iter_size[1] *
                  h->iter_size[2];
  }
}

/* ------------------------------------------------------------------------
 * constants (ops_decl_const_char: cudaMemcpyToSymbol in the reference,
 * master_kernel.cpp.j2:40-70).  The generated kernels file registers the
 * copier for its __constant__ symbols.
 * ---------------------------------------------------------------------- */
OPS_API void ob2_register_const_handler(ob2_const_fn fn) { rt().const_fn = fn; }

OPS_API void ops_decl_const_char(OPS_instance *, int dim, char const *, int type_size, char *data,
                                 char const *name) {
  require_init();
  if (!rt().const_fn) return;  // no generated kernel uses constants
  ob2_flush();                 // queued loops read the old value
  int rc = rt().const_fn(name, dim, type_size, data, ob2_dev_stream());
  if (rc < 0) {
    OPSException ex(OPS_INVALID_ARGUMENT);
    ex << "Error: ops_decl_const " << name << " larger than its device symbol";
    throw ex;
  }
  check(rc, "ops_decl_const");
}

/* runs the lazy loop-chain queue (ops_lazy.cpp:1248-1446); work is
 * stream ordered, so this does not wait for the device */
OPS_API void ops_execute(OPS_instance *) { ob2_flush(); }

/* ------------------------------------------------------------------------
 * par_loop support for generated stubs (loop_host.cpp.j2:13-780)
 * ---------------------------------------------------------------------- */
/* Block-shape autotuner.  After one untimed launch with the default shape,
 * each candidate shape is launched kTuneReps times, eagerly and bracketed by
 * events; at the kernel's next launch the shape with the smallest device
 * time per point (best of its repetitions) is kept for the rest of the run
 * (and written to OPS_B200_TUNE_FILE at ops_exit). */
namespace {
constexpr int kTuneReps = 2;

int tune_count(int dim) {
  return dim == 2 ? (int)(sizeof kTune2 / sizeof kTune2[0]) : (int)(sizeof kTune3 / sizeof kTune3[0]);
}

void tune_decide(KStat &k, int dim) {
  const int nc = tune_count(dim);
  std::vector<double> best_per(nc, 1e300);
  for (int j = 0; j < nc * kTuneReps && 2 * j + 1 < (int)k.tune_ev.size(); j++) {
    float ms = 0.f;
    if (!k.tune_ev[2 * j] || ob2_event_elapsed_ms(k.tune_ev[2 * j], k.tune_ev[2 * j + 1], &ms))
      continue;
    const double per = ms / (double)std::max(1LL, k.tune_pts[j]);
    best_per[j % nc] = std::min(best_per[j % nc], per);
  }
  int bi = 0;
  for (int c = 1; c < nc; c++)
    if (best_per[c] < best_per[bi]) bi = c;
  const int(*t)[3] = dim == 2 ? kTune2 : kTune3;
  for (int i = 0; i < 3; i++) k.best[i] = t[bi][i];
  for (void *e : k.tune_ev)
    if (e) rt().ev_pool.push_back(e);
  k.tune_ev.clear();
  k.tune_state = 2;
}

void tune_pick(ob2_loop *L) {
  Runtime &r = rt();
  KStat &k = r.kstats[L->kernel_index];
  const int dim = L->dim > 3 ? 3 : L->dim;
  const int nc = tune_count(dim);
  const int(*t)[3] = dim == 2 ? kTune2 : kTune3;
  if (k.tune_state == 1) {
    ob2_flush();
    tune_decide(k, dim);
  }
  if (k.tune_state == 2) {
    for (int i = 0; i < 3; i++) L->block[i] = k.best[i];
    return;
  }
  k.tune_dim = dim;
  if (k.tune_next++ == 0) return;  // first launch: default shape, untimed
  const int j = k.tune_next - 2;  // timed launch index
  const int c = j % nc;
  for (int i = 0; i < 3; i++) L->block[i] = t[c][i];
  L->tune = j;
  if ((int)k.tune_ev.size() < 2 * nc * kTuneReps) k.tune_ev.resize(2 * nc * kTuneReps, nullptr);
  if ((int)k.tune_pts.size() < nc * kTuneReps) k.tune_pts.resize(nc * kTuneReps, 0);
  k.tune_pts[j] = L->npoints;
  if (j + 1 == nc * kTuneReps) k.tune_state = 1;
}
}  // namespace

OPS_API int ob2_loop_begin(ob2_loop *L, const char *name, ops_block block, int dim,
                           const int *range, ops_arg *args, int nargs) {
  require_init();
  Runtime &r = rt();
  if (nargs > OB2_MAX_ARGS)
    throw OPSException(OPS_NOT_IMPLEMENTED, "Error: too many arguments in ops_par_loop");
  L->name = name;
  L->dim = dim;
  L->nargs = nargs;
  L->args = args;
  L->stream = ob2_dev_stream();
  L->npoints = 1;
  if (dim < 1 || dim > OPS_MAX_DIM)
    throw OPSException(OPS_INVALID_ARGUMENT, "Error: ops_par_loop dimension out of range");
  for (int i = 0; i < 3; i++) {
    L->lo[i] = i < dim ? range[2 * i] : 0;
    L->hi[i] = i < dim ? range[2 * i + 1] : 1;
  }
  for (int i = 0; i < 2; i++) {  // the 4th and 5th axes of 4D / 5D blocks
    L->lo4[i] = 3 + i < dim ? range[2 * (3 + i)] : 0;
    L->hi4[i] = 3 + i < dim ? range[2 * (3 + i) + 1] : 1;
  }
  if (r.dist) dist_loop(block, dim, L->lo, L->hi, args, nargs, name);
  // a loop launched at once (reductions, autotuning) runs the queue first:
  // a temporally blocked chain in it may move a dat's storage, and the
  // views below must see where the dats are
  if (r.autotune || !r.lazy) ob2_flush();
  else
    for (int i = 0; i < nargs; i++)
      if (args[i].argtype == OPS_ARG_GBL && args[i].acc != OPS_READ) {
        ob2_flush();
        break;
      }
  for (int i = 0; i < 3; i++) {
    L->n[i] = std::max(0, L->hi[i] - L->lo[i]);
    L->npoints *= L->n[i];
  }
  // 4D / 5D: the generated kernel walks the 3rd to 5th axes as one folded
  // index, so the grid's z extent covers their product
  long long nfold = L->n[2];
  for (int i = 0; i < 2; i++) {
    const long long e = std::max(0, L->hi4[i] - L->lo4[i]);
    L->npoints *= e;
    nfold *= e;
  }
  if (nfold > 0x7fffffffLL)
    throw OPSException(OPS_NOT_IMPLEMENTED, "Error: ops_par_loop range too large");
  L->kernel_index = kernel_slot(name);
  L->block[0] = r.block_x;
  L->block[1] = dim > 1 ? r.block_y : 1;
  L->block[2] = dim > 2 ? r.block_z : 1;
  L->host_t0 = wall();
  L->ev_start = L->ev_end = nullptr;
  L->fuse_id = -1;  // the stub names its fused launcher after this call
  L->ffn = nullptr;
  L->hfn = nullptr;
  L->tfn = nullptr;
  L->tb_off = nullptr;
  L->tb_role = nullptr;
  if (L->npoints == 0) return 0;

  size_t red_bytes = 0;
  int nred = 0;
  L->idx32 = 1;
  const int soa = I().OPS_soa;
  for (int i = 0; i < nargs; i++) {
    ops_arg &a = args[i];
    ob2_view &v = L->view[i];
    memset(&v, 0, sizeof(v));
    L->red[i].acc = nullptr;
    L->red[i].first = 0;
    L->red[i].op = 0;
    if (a.argtype == OPS_ARG_DAT) {
      // a disabled optional argument (ops_arg_dat_opt, flag 0) still gets
      // its dat's view when it names one, as in the reference's generated
      // code, where the flag only matters to distributed halo exchanges
      if (!a.dat) continue;
      ops_dat d = a.dat;
      if (d->locked_hd) {
        OPSException ex(OPS_INVALID_ARGUMENT);
        ex << "Error: ops_par_loop " << name << " called with dat " << d->name
           << " whose raw pointer was not released";
        throw ex;
      }
      put_data(d);
      // low-dim accumulation: first INC/MIN/MAX since another access fills
      // the dat with the identity (ops_dummy_singlenode.cpp:235-391)
      DatX &dx = r.datx[d->index];
      if (a.opt && d->e_dat && (a.acc == OPS_INC || a.acc == OPS_MIN || a.acc == OPS_MAX) &&
          dx.edat_prev_acc != a.acc) {
        dx.edat_prev_acc = a.acc;
        ob2_flush();
        unsigned char idv[16];
        int tc = type_code(d->type);
        identity_bytes(tc, a.acc, idv, true);
        check(ob2_fill_value(d->data_d, idv, d->type_size, d->mem / d->type_size),
              "low-dim init");
      }
      if (d->block->dims != block->dims && !d->e_dat) {
        // dats of other blocks are allowed as long as the dims agree
      }
      if ((double)dat_points(d) * d->dim >= 2147483647.0) L->idx32 = 0;
      const int md = d->dim;
      const int *st = a.stencil ? a.stencil->stride : nullptr;
      // a prolong stencil needs generated code that divides the loop index
      // (the stub marks those arguments in prolong_mask)
      const int stype = a.stencil ? a.stencil->type : 0;
      if ((stype == 1) != (((L->prolong_mask >> i) & 1u) != 0)) {
        OPSException ex(OPS_NOT_IMPLEMENTED);
        ex << "Error: ops_par_loop " << name << " argument " << i
           << (stype == 1 ? " has a prolong stencil that its generated code does not divide by"
                          : " is marked as prolong but its stencil is not a prolong stencil")
           << " (pass the stencil variable declared by ops_decl_prolong_stencil directly)";
        throw ex;
      }
      long long cum = 1, off = 0;
      long long step[OPS_MAX_DIM] = {0, 0, 0, 0, 0};
      long long cums[OPS_MAX_DIM + 1] = {1, 1, 1, 1, 1, 1};  // points before axis k
      for (int k = 0; k < block->dims && k < OPS_MAX_DIM; k++) {
        int sk = st ? st[k] : 1;
        if (stype == 2) sk *= a.stencil->mgrid_stride[k];  // restrict: index * stride
        off += cum * (long long)(-d->base[k] - d->d_m[k]);
        step[k] = cum * sk;
        cums[k] = cum;
        cum *= d->size[k];
      }
      if (soa) {
        v.ex = 1;
        v.ey = d->size[0];
        v.ez = d->size[0] * d->size[1];
        v.eu = (int)cums[3];
        v.ev = (int)cums[4];
        v.ed = (int)cum;
        v.base = d->data_d + off * d->type_size;
        v.wx = step[0];
        v.wy = step[1];
        v.wz = step[2];
        v.wu = step[3];
        v.wv = step[4];
      } else {
        v.ex = md;
        v.ey = d->size[0] * md;
        v.ez = d->size[0] * d->size[1] * md;
        v.eu = (int)(cums[3] * md);
        v.ev = (int)(cums[4] * md);
        v.ed = 1;
        v.base = d->data_d + off * d->elem_size;
        v.wx = step[0] * md;
        v.wy = step[1] * md;
        v.wz = step[2] * md;
        v.wu = step[3] * md;
        v.wv = step[4] * md;
      }
    } else if (a.argtype == OPS_ARG_GBL && a.acc != OPS_READ) {
      ops_reduction h = (ops_reduction)a.data;
      RedX &x = r.redx[h->index];
      if (!h->initialized) {
        OPSException ex(OPS_INVALID_ARGUMENT);
        ex << "Error: reduction handle " << h->name << " used without ops_arg_reduce";
        throw ex;
      }
      L->red[i].acc = x.acc_d;
      L->red[i].first = x.pending_first;
      L->red[i].op = a.acc;
      x.pending_first = 0;
      red_bytes += (size_t)h->size;
      nred++;
    }
  }
  // scratch for per-CTA partials (grid = ceil(n/block) per axis); each
  // reduction argument's region is rounded up to 256 bytes by the stub
  // grid: x covers the range; y and z are capped so that the grid is about
  // one wave of resident CTAs (SMs x CTAs per SM), threads loop over the rest
  L->tune = -1;
  if (r.autotune && nred == 0 && dim >= 2 && dim <= 3) tune_pick(L);
  {
    long long tpb = (long long)L->block[0] * L->block[1] * L->block[2];
    long long per_sm = std::max(1LL, 2048 / tpb);
    long long target = (long long)r.sms * per_sm * r.red_waves;
    long long gx = (L->n[0] + L->block[0] - 1) / L->block[0];
    long long gy = (L->n[1] + L->block[1] - 1) / L->block[1];
    long long gz = (nfold + L->block[2] - 1) / L->block[2];
    if (nred > 0) {  // reduction kernels stride over y/z (see the generated kernel)
      long long cy = std::max(1LL, target / std::max(1LL, gx));
      if (gy > cy) gy = cy;
      long long cz = std::max(1LL, target / std::max(1LL, gx * gy));
      if (gz > cz) gz = cz;
    }
    if (nred == 0 && (gy > 65535 || gz > 65535))
      throw OPSException(OPS_NOT_IMPLEMENTED,
                         "Error: ops_par_loop range too large along y or z for one launch");
    if (gz > 65535) gz = 65535;
    if (gy > 65535) gy = 65535;
    L->grid[0] = (int)gx;
    L->grid[1] = (int)gy;
    L->grid[2] = (int)gz;
  }
  long long nblk = (long long)L->grid[0] * L->grid[1] * L->grid[2];
  size_t need = red_bytes * (size_t)nblk + 256 * (size_t)nred;
  if (need > r.partials_cap) {
    if (r.partials) {
      ob2_dev_sync();
      ob2_dev_free(r.partials);
    }
    size_t cap = std::max(need, (size_t)1 << 20);
    check(ob2_dev_malloc(&r.partials, cap), "reduction scratch");
    r.partials_cap = cap;
  }
  L->partials = r.partials;
  L->partials_bytes = r.partials_cap;
  L->counter = r.counter;
  L->ev_start = nullptr;  // launches are timed in ob2_launch / run_item
  return 1;
}

OPS_API int ob2_args_alias(const ops_arg *args, int nargs) {
  for (int i = 0; i < nargs; i++) {
    if (args[i].argtype != OPS_ARG_DAT || !args[i].dat) continue;
    for (int j = i + 1; j < nargs; j++) {
      if (args[j].argtype != OPS_ARG_DAT || args[j].dat != args[i].dat) continue;
      if (args[i].acc != OPS_READ || args[j].acc != OPS_READ) return 1;
    }
  }
  return 0;
}

OPS_API void ob2_loop_check_launch(ob2_loop *L) {
  int e = ob2_last_launch_error();
  if (e) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "Error: kernel launch of ops_par_loop " << L->name << " failed: " << ob2_error_string(e);
    throw ex;
  }
}

OPS_API void ob2_loop_end(ob2_loop *L) {
  Runtime &r = rt();
  KStat &s = r.kstats[L->kernel_index];
  s.count++;
  if (L->ev_start) {
    kt_end(L->ev_start, L->kernel_index);
    L->ev_start = nullptr;
  }
  s.host_s += wall() - L->host_t0;
  for (int i = 0; i < L->nargs; i++) {
    ops_arg &a = L->args[i];
    if (a.argtype != OPS_ARG_DAT || !a.dat) continue;
    ops_dat d = a.dat;
    if (a.acc != OPS_READ) d->dirty_hd = 2;
    if (d->e_dat && (a.acc == OPS_READ || a.acc == OPS_WRITE || a.acc == OPS_RW))
      r.datx[d->index].edat_prev_acc = a.acc;
    // transfer model (ops_lib_core.cpp:1687-1697)
    s.transfer += (double)L->npoints * d->elem_size *
                  ((a.acc == OPS_RW || a.acc == OPS_INC) ? 2.0 : 1.0);
  }
}

/* ------------------------------------------------------------------------
 * per-kernel device timing (see ops_b200_loop.h)
 * ---------------------------------------------------------------------- */
static void ktime_collect() {
  Runtime &r = rt();
  ob2_flush();
  if (r.pending.empty()) return;
  check(ob2_dev_sync(), "ob2_ktime");
  for (auto &p : r.pending) {
    float ms = 0.f;
    check(ob2_event_elapsed_ms(p.a, p.b, &ms), "ob2_ktime");
    r.kstats[p.k].dev_ms += ms;
    r.ev_pool.push_back(p.a);
    r.ev_pool.push_back(p.b);
  }
  r.pending.clear();
}
OPS_API void ob2_ktime_enable(int on) {
  ktime_collect();
  rt().ktime = on != 0;
}
OPS_API void ob2_ktime_reset(void) {
  ktime_collect();
  for (auto &k : rt().kstats) {
    k.count = 0;
    k.dev_ms = 0.0;
    k.host_s = 0.0;
    k.transfer = 0.0;
  }
}
OPS_API size_t ob2_ktime_report(char *buf, size_t n) {
  ktime_collect();
  std::string s;
  char line[512];
  for (auto &k : rt().kstats) {
    if (!k.count) continue;
    snprintf(line, sizeof line, "%s %ld %.6f %.0f\n", k.name.c_str(), k.count, k.dev_ms,
             k.transfer);
    s += line;
  }
  if (buf && n) {
    size_t m = std::min(n - 1, s.size());
    memcpy(buf, s.data(), m);
    buf[m] = 0;
  }
  return s.size();
}
OPS_API long long ob2_launch_count(void) { return rt().launches; }

/* ------------------------------------------------------------------------
 * output / timing (ops_lib_core.cpp:1468-1647)
 * ---------------------------------------------------------------------- */
OPS_API void ops_printf(const char *fmt, ...) {
  if (R && R->comm.rank != 0) return;  // rank 0 prints, as in the reference's MPI build
  va_list ap;
  va_start(ap, fmt);
  vprintf(fmt, ap);
  va_end(ap);
}
OPS_API void ops_fprintf(FILE *f, const char *fmt, ...) {
  if (R && R->comm.rank != 0) return;
  va_list ap;
  va_start(ap, fmt);
  vfprintf(f, fmt, ap);
  va_end(ap);
}
OPS_API void ops_diagnostic_output(void) {
  Runtime &r = rt();
  if (I().OPS_diags <= 1) return;
  printf("\n OPS diagnostic output (B200 backend)\n --------------------------------\n");
  printf(" blocks %zu, dats %zu, stencils %zu, halos %zu\n", r.blocks.size(), r.dats.size(),
         r.stencils.size(), r.halos.size());
  size_t tot = 0;
  for (ops_dat d : r.dats)
    if (d) tot += d->mem;
  printf(" total device memory in dats: %.3f MB\n", tot / 1e6);
}
OPS_API size_t ops_timing_output_str(char *buf, size_t n) {
  Runtime &r = rt();
  ob2_flush();
  ob2_dev_sync();
  ktime_collect();
  std::string s;
  char line[320];
  snprintf(line, sizeof line, "\n  %-40s %8s %14s %14s %10s\n", "Timings (B200 backend)", "count",
           "time(s)", "device(ms)", "GB/s");
  s += line;
  double tt = 0.0;
  for (auto &k : r.kstats) {
    double t = k.dev_ms > 0 ? k.dev_ms * 1e-3 : k.host_s;
    tt += k.host_s;
    snprintf(line, sizeof line, "  %-40s %8ld %14.6f %14.4f %10.2f\n", k.name.c_str(), k.count,
             k.host_s, k.dev_ms, t > 0 ? k.transfer / t / 1e9 : 0.0);
    s += line;
  }
  snprintf(line, sizeof line, "  Total kernel time (host): %f\n", tt);
  s += line;
  if (r.autotune) {
    s += "  Autotuned block shapes:";
    for (auto &k : r.kstats)
      if (k.tune_state == 2) {
        snprintf(line, sizeof line, " %s=%dx%dx%d", k.name.c_str(), k.best[0], k.best[1],
                 k.best[2]);
        s += line;
      }
    s += "\n";
  }
  if (r.tb_auto) {
    s += "  Temporal-blocking depths (1: plain sweeps):";
    for (auto &k : r.kstats)
      if (k.tb_state == 2) {
        snprintf(line, sizeof line, " %s=%d", k.name.c_str(), k.tb_best);
        s += line;
      }
    s += "\n";
  }
  if (r.lazy) {
    snprintf(line, sizeof line,
             "  Lazy execution: %lld chains, %lld graph replays, %lld graph updates, "
             "%lld tile launches, %lld multi-instance launches, %lld fused launches "
             "(%lld loops), %lld halo transfers folded into loop launches, "
             "%lld temporal-blocking launches (%lld sweeps)\n",
             r.chains, r.graph_hits, r.graph_updates, r.tiles_run, r.multi_launches,
             r.fused_launches, r.fused_loops, r.hfused, r.tb_launches, r.tb_sweeps);
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
/* like the reference CUDA backend's ops_timers: device work is complete at
 * the returned time stamp */
OPS_API void ops_timers(double *cpu, double *et) {
  if (R && R->initialised) {
    ob2_flush();
    ob2_dev_sync();
  }
  ops_timers_core(cpu, et);
}
OPS_API int ops_is_root(void) { return rt().comm.rank == 0; }
OPS_API int ops_get_proc(void) { return rt().comm.rank; }
OPS_API int ops_num_procs(void) { return rt().comm.size; }
OPS_API void ops_NaNcheck(ops_dat d) {
  require_init();
  ops_printf("ops_NaNcheck_core called for %s \n", d->name);
  if (strcmp(d->type, "double") && strcmp(d->type, "float")) return;
  ob2_flush();
  put_data(d);
  long long first = -1;
  check(ob2_nan_find(d->data_d, d->type_size, d->dim, I().OPS_soa, d->mem / d->type_size,
                     &first),
        "ops_NaNcheck");
  if (first < 0) return;
  const int comp = (int)(first % d->dim);
  long long pt = first / d->dim;
  int idx[OPS_MAX_DIM] = {0};
  for (int i = 0; i < OPS_MAX_DIM; i++) {
    const int sz = std::max(1, d->size[i]);
    idx[i] = (int)(pt % sz) + d->d_m[i];
    pt /= sz;
  }
  printf("Error: NaN detected at element dim:%d,index:(%d", comp, idx[0]);
  for (int i = 1; i < d->block->dims; i++) printf(",%d", idx[i]);
  printf(")\n");
  fflush(stdout);
  exit(2);
}
OPS_API void ops_partition(const char *) {}
OPS_API void ops_partition_opts_c(const char *) {}
OPS_API void ops_get_data(ops_dat d) { get_data(d); }
OPS_API void ops_put_data(ops_dat d) { put_data(d); }
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
OPS_API void *xmalloc(size_t n) {
  void *p = malloc(n);
  if (!p && n) throw OPSException(OPS_RUNTIME_ERROR, "Error: xmalloc failed");
  return p;
}
OPS_API void *xrealloc(void *p, size_t n) {
  void *q = realloc(p, n);
  if (!q && n) throw OPSException(OPS_RUNTIME_ERROR, "Error: xrealloc failed");
  return q;
}
OPS_API void *xcalloc(size_t k, size_t n) {
  void *p = calloc(k, n);
  if (!p && k != 0 && n != 0) throw OPSException(OPS_RUNTIME_ERROR, "Error: xcalloc failed");
  return p;
}

OPS_API void ops_print_dat_to_txtfile(ops_dat d, const char *file) {
  get_data(d);
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
static void no_hdf5(const char *what, const char *file) {
  fprintf(stderr, "OPS B200 backend: %s(%s) skipped: built without HDF5\n", what,
          file ? file : "");
}
OPS_API void ops_fetch_dat_hdf5_file(ops_dat, char const *f) { no_hdf5("ops_fetch_dat_hdf5_file", f); }
OPS_API void ops_fetch_block_hdf5_file(ops_block, char const *f) {
  no_hdf5("ops_fetch_block_hdf5_file", f);
}
OPS_API void ops_fetch_stencil_hdf5_file(ops_stencil, char const *f) {
  no_hdf5("ops_fetch_stencil_hdf5_file", f);
}
OPS_API void ops_fetch_halo_hdf5_file(ops_halo, char const *f) {
  no_hdf5("ops_fetch_halo_hdf5_file", f);
}
OPS_API void ops_print_dat_to_txtfile_core(ops_dat d, const char *file) {
  ops_print_dat_to_txtfile(d, file);
}

/* ------------------------------------------------------------------------
 * external access (ops_dummy_singlenode.cpp:630-850)
 * ---------------------------------------------------------------------- */
OPS_API int ops_dat_get_local_npartitions(ops_dat) { return 1; }
OPS_API int ops_dat_get_global_npartitions(ops_dat) { return 1; }
OPS_API void ops_dat_get_extents(ops_dat d, int, int *disp, int *size) {
  for (int i = 0; i < d->block->dims; i++) {
    if (disp) disp[i] = 0;
    if (size) size[i] = d->size[i] + d->d_m[i] - d->d_p[i];
  }
  const DatX &x = rt().datx[d->index];
  if (rt().dist && x.split) {  // this rank's interior rows (as the reference's MPI backend)
    const int ax = x.axis, sh = -d->d_m[ax];  // storage row of interior row 0
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
    if (slab[2 * i] < 0 || slab[2 * i + 1] > ext[i]) {
      OPSException ex(OPS_RUNTIME_ERROR);
      ex << "Error: ops_dat_get_slab_extents() called on " << d->name
         << " with slab ranges in dimension " << i << ": " << slab[2 * i] << "-"
         << slab[2 * i + 1] << " beyond data size 0-" << ext[i];
      throw ex;
    }
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
/* ops_dummy_singlenode.cpp:662-707 */
OPS_API char *ops_dat_get_raw_pointer(ops_dat d, int, ops_stencil, ops_memspace *ms) {
  if (rt().dist && rt().datx[d->index].split) dist_unsupported(d, "a raw pointer");
  require_init();
  ob2_flush();
  if (ms && *ms == OPS_HOST) {
    get_data(d);
    d->locked_hd = OPS_HOST;
    return d->data + d->base_offset;
  }
  put_data(d);
  if (ms) *ms = OPS_DEVICE;
  d->locked_hd = OPS_DEVICE;
  return d->data_d + d->base_offset;
}
/* ops_dummy_singlenode.cpp:709-735 */
OPS_API void ops_dat_release_raw_data(ops_dat d, int, ops_access acc) {
  if (!d->locked_hd) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "Error: ops_dat_release_raw_data() called, but with no matching "
          "ops_dat_get_raw_pointer() beforehand: "
       << d->name;
    throw ex;
  }
  if (acc != OPS_READ) d->dirty_hd = d->locked_hd == OPS_HOST ? 1 : 2;
  d->locked_hd = 0;
}
OPS_API void ops_dat_release_raw_data_memspace(ops_dat d, int part, ops_access acc,
                                               ops_memspace *ms) {
  if (ms && d->locked_hd) d->locked_hd = *ms;
  ops_dat_release_raw_data(d, part, acc);
}

static void stage_reserve(size_t n) {
  Runtime &r = rt();
  if (n > r.stage_cap) {
    if (r.stage_d) {
      ob2_dev_sync();
      ob2_dev_free(r.stage_d);
    }
    check(ob2_dev_malloc((void **)&r.stage_d, n), "staging buffer");
    r.stage_cap = n;
  }
}

/* packed AoS slab <-> dat: dir 0 fetch, 1 set (ops_util.cpp:353-500) */
static void slab_io(ops_dat d, char *data, const int *range, ops_memspace ms, int dir) {
  require_init();
  if (d->block->dims > 3)
    throw OPSException(OPS_NOT_IMPLEMENTED,
                       "Error: slab fetch / set of a dat of a 4D or 5D block");
  int start[3] = {0, 0, 0}, count[3] = {1, 1, 1}, size3[3] = {1, 1, 1};
  size_t pts = 1;
  for (int i = 0; i < 3; i++) size3[i] = d->size[i];
  for (int i = 0; i < d->block->dims && i < 3; i++) {
    start[i] = range[2 * i] - d->d_m[i];
    count[i] = range[2 * i + 1] - range[2 * i];
    if (count[i] < 0 || start[i] < 0 || start[i] + count[i] > d->size[i])
      throw OPSException(OPS_RUNTIME_ERROR, "Error: slab range outside the dat");
    pts *= (size_t)count[i];
  }
  size_t bytes = pts * d->elem_size;
  if (bytes == 0) return;
  ob2_flush();
  put_data(d);
  char *buf = data;
  if (ms != OPS_DEVICE) {
    stage_reserve(bytes);
    buf = rt().stage_d;
    if (dir == 1) check(ob2_dev_h2d(buf, data, bytes), "ops_dat_set_data");
  }
  check(ob2_box_copy(d->data_d, d->type_size, d->dim, I().OPS_soa, size3, start, count,
                     buf, dir),
        dir == 0 ? "ops_dat_fetch_data" : "ops_dat_set_data");
  if (ms != OPS_DEVICE && dir == 0) check(ob2_dev_d2h(data, buf, bytes), "ops_dat_fetch_data");
  if (ms == OPS_DEVICE) check(ob2_dev_sync(), "slab copy");
  if (dir == 1) d->dirty_hd = 2;
}
static void full_range(ops_dat d, int *r) {
  int ext[OPS_MAX_DIM], disp[OPS_MAX_DIM] = {0, 0, 0, 0, 0};
  ops_dat_get_extents(d, 0, disp, ext);
  for (int i = 0; i < OPS_MAX_DIM; i++) {
    r[2 * i] = i < d->block->dims ? disp[i] : 0;
    r[2 * i + 1] = i < d->block->dims ? disp[i] + ext[i] : 1;
  }
}
OPS_API void ops_dat_fetch_data_memspace(ops_dat d, int, char *data, ops_memspace ms) {
  int r[2 * OPS_MAX_DIM];
  full_range(d, r);
  slab_io(d, data, r, ms, 0);
}
OPS_API void ops_dat_fetch_data(ops_dat d, int part, char *data) {
  ops_dat_fetch_data_memspace(d, part, data, OPS_HOST);
}
OPS_API void ops_dat_fetch_data_slab_memspace(ops_dat d, int, char *data, int *range,
                                              ops_memspace ms) {
  slab_io(d, data, range, ms, 0);
}
OPS_API void ops_dat_set_data_memspace(ops_dat d, int, char *data, ops_memspace ms) {
  int r[2 * OPS_MAX_DIM];
  full_range(d, r);
  slab_io(d, data, r, ms, 1);
}
OPS_API void ops_dat_set_data(ops_dat d, int part, char *data) {
  ops_dat_set_data_memspace(d, part, data, OPS_HOST);
}
OPS_API void ops_dat_set_data_slab_memspace(ops_dat d, int, char *data, int *range,
                                            ops_memspace ms) {
  slab_io(d, data, range, ms, 1);
}

/* ------------------------------------------------------------------------
 * random fills: counter-based stream generated on the device
 * (replaces cuRAND in ops_cuda_common.cu:184-283)
 * ---------------------------------------------------------------------- */
OPS_API void ops_randomgen_init(unsigned int seed, int) {
  rt().rng_seed = seed;
  rt().rng_counter = 0;
}
OPS_API void ops_randomgen_exit(void) {}
static void fill_rand(ops_dat d, int normal) {
  require_init();
  if (d->type_size != 8 && d->type_size != 4)
    throw OPSException(OPS_NOT_IMPLEMENTED, "Error: random fill needs a float or double dat");
  size_t n = dat_points(d) * d->dim;
  ob2_flush();
  check(ob2_fill_random(d->data_d, d->type_size, n, rt().rng_seed, rt().rng_counter, normal),
        "ops_fill_random");
  rt().rng_counter += n;
  d->dirty_hd = 2;
}
OPS_API void ops_fill_random_uniform(ops_dat d) { fill_rand(d, 0); }
OPS_API void ops_fill_random_normal(ops_dat d) { fill_rand(d, 1); }

/* ------------------------------------------------------------------------
 * tridiagonal (ops_tridiag_cuda.cpp:96-251: size/type checks, raw pointers
 * at the range origin, solve along solvedim)
 * ---------------------------------------------------------------------- */
static void trid_dist_check(int ndim, int solvedim, ops_dat d) {
  if (rt().dist && rt().datx[d->index].split && solvedim == ndim - 1)
    dist_unsupported(d, "a tridiagonal solve along the split axis");
}
static void trid(int ndim, int solvedim, int *range, ops_dat a, ops_dat b, ops_dat c, ops_dat d,
                 ops_dat u) {
  require_init();
  if (ndim < 1 || ndim > 3 || solvedim < 0 || solvedim >= ndim)
    throw OPSException(OPS_INVALID_ARGUMENT, "Tridsolver error: bad ndim or solvedim");
  for (int i = 0; i < ndim; i++)
    if (a->size[i] != b->size[i] || b->size[i] != c->size[i] || c->size[i] != d->size[i] ||
        (u && u->size[i] != d->size[i]))
      throw OPSException(OPS_RUNTIME_ERROR,
                         "Tridsolver error: the a,b,c,d datasets all need to be the same size");
  if (strcmp(a->type, b->type) || strcmp(b->type, c->type) || strcmp(c->type, d->type) ||
      (u && strcmp(d->type, u->type)))
    throw OPSException(OPS_RUNTIME_ERROR,
                       "Tridsolver error: the a,b,c,d datasets must all be of the same type");
  if (strcmp(a->type, "double") && strcmp(a->type, "float"))
    throw OPSException(OPS_RUNTIME_ERROR,
                       "Tridsolver error: unsupported type. Dataset type must either be "
                       "\"double\" or \"float\"");
  ops_dat all[5] = {a, b, c, d, u};
  for (int i = 0; i < 5; i++)
    if (all[i]) {
      if (all[i]->locked_hd)
        throw OPSException(OPS_INVALID_ARGUMENT, "Tridsolver error: dat raw pointer not released");
      put_data(all[i]);
    }
  int dims[3] = {1, 1, 1};
  long long strides[3] = {1, a->size[0], (long long)a->size[0] * a->size[1]};
  long long off = 0;
  int rng[6] = {0, 1, 0, 1, 0, 1};
  for (int i = 0; i < 2 * ndim; i++) rng[i] = range[i];
  if (rt().dist && rt().datx[d->index].split) {  // lines across the split axis: this rank's
    trid_dist_check(ndim, solvedim, d);
    const std::array<int, 5> &bp = block_part(d->block, 0);
    ob2dist::clip(bp[1], bp[2], bp[3], bp[4], &rng[2 * (ndim - 1)], &rng[2 * ndim - 1]);
    rt().datx[(u ? u : d)->index].dirty = true;
  }
  range = rng;
  for (int i = 0; i < ndim; i++) {
    dims[i] = range[2 * i + 1] - range[2 * i];
    long long s0 = (long long)range[2 * i] - a->d_m[i] - a->base[i];
    if (dims[i] < 0 || s0 < 0 || s0 + dims[i] > a->size[i])
      throw OPSException(OPS_INVALID_ARGUMENT, "Tridsolver error: range outside the datasets");
    off += s0 * strides[i];
  }
  size_t ts = a->type_size;
  static const char *names[2][3] = {
      {"ops_tridMultiDimBatch_x", "ops_tridMultiDimBatch_y", "ops_tridMultiDimBatch_z"},
      {"ops_tridMultiDimBatch_Inc_x", "ops_tridMultiDimBatch_Inc_y",
       "ops_tridMultiDimBatch_Inc_z"}};
  int k = kernel_slot(names[u ? 1 : 0][solvedim]);
  double t0 = wall();
  ob2_flush();
  void *ev = kt_begin();
  int rc = ob2_trid_batch((int)ts, ndim, solvedim, dims, strides, a->data_d + off * ts,
                          b->data_d + off * ts, c->data_d + off * ts, d->data_d + off * ts,
                          u ? u->data_d + off * ts : nullptr);
  kt_end(ev, k);
  rt().launches++;
  if (rc) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "Tridsolver error: " << ob2_error_string(rc) << " (line length "
       << dims[solvedim] << ", max 4096)";
    throw ex;
  }
  KStat &s = rt().kstats[k];
  s.count++;
  s.host_s += wall() - t0;
  double pts = (double)dims[0] * dims[1] * dims[2];
  s.transfer += pts * ts * (u ? 6.0 : 5.0);
  (u ? u : d)->dirty_hd = 2;
}
OPS_API void ops_tridMultiDimBatch(int ndim, int solvedim, int *range, ops_dat a, ops_dat b,
                                   ops_dat c, ops_dat d, ops_tridsolver_params *) {
  trid(ndim, solvedim, range, a, b, c, d, nullptr);
}
OPS_API void ops_tridMultiDimBatch_Inc(int ndim, int solvedim, int *range, ops_dat a,
                                       ops_dat b, ops_dat c, ops_dat d, ops_dat u,
                                       ops_tridsolver_params *) {
  trid(ndim, solvedim, range, a, b, c, d, u);
}

/* ------------------------------------------------------------------------
 * dump hook (same format as the oracle): every live dat, halos included
 * ---------------------------------------------------------------------- */
OPS_API void ops_dump_dats(const char *path) {
  Runtime &r = rt();
  std::string fp(path);
  if (r.dist) fp += ".r" + std::to_string(r.comm.rank);  // one file per rank
  FILE *f = fopen(fp.c_str(), "wb");
  if (!f) return;
  for (ops_dat d : r.dats) {
    if (!d) continue;
    const DatX &x = r.datx[d->index];
    if (r.dist && x.split) {  // this rank's owned storage rows of the slowest axis
      ob2_flush();
      const size_t nb = (size_t)(x.o_hi - x.o_lo) * x.row_bytes;
      std::vector<char> h(nb ? nb : 1);
      if (nb) check(ob2_dev_d2h(h.data(), d->data_d + (size_t)x.o_lo * x.row_bytes, nb), "dump");
      int nl = (int)strlen(d->name), tl = (int)strlen(d->type);
      fwrite("DAT0", 1, 4, f);
      fwrite(&nl, 4, 1, f);
      fwrite(d->name, 1, nl, f);
      fwrite(&tl, 4, 1, f);
      fwrite(d->type, 1, tl, f);
      int meta[4] = {d->dim, d->type_size, d->block->dims, I().OPS_soa};
      fwrite(meta, 4, 4, f);
      int sz[OPS_MAX_DIM];
      for (int i = 0; i < OPS_MAX_DIM; i++) sz[i] = d->size[i];
      sz[x.axis] = x.o_hi - x.o_lo;
      fwrite(sz, 4, OPS_MAX_DIM, f);
      fwrite(d->d_m, 4, OPS_MAX_DIM, f);
      fwrite(d->d_p, 4, OPS_MAX_DIM, f);
      unsigned long long nbl = nb;
      fwrite(&nbl, 8, 1, f);
      fwrite(h.data(), 1, nb, f);
      continue;
    }
    if (r.dist && r.comm.rank != 0) continue;  // whole on every rank: rank 0 writes it
    get_data(d);
    int nl = (int)strlen(d->name);
    fwrite("DAT0", 1, 4, f);
    fwrite(&nl, 4, 1, f);
    fwrite(d->name, 1, nl, f);
    int tl = (int)strlen(d->type);
    fwrite(&tl, 4, 1, f);
    fwrite(d->type, 1, tl, f);
    int meta[4] = {d->dim, d->type_size, d->block->dims, I().OPS_soa};
    fwrite(meta, 4, 4, f);
    fwrite(d->size, 4, OPS_MAX_DIM, f);
    fwrite(d->d_m, 4, OPS_MAX_DIM, f);
    fwrite(d->d_p, 4, OPS_MAX_DIM, f);
    unsigned long long nb = d->mem;
    fwrite(&nb, 8, 1, f);
    fwrite(d->data, 1, d->mem, f);
  }
  fclose(f);
}
