// capi.cu -- the native C ABI: context, device-resident state and the step
// driver.  The call structure mirrors the reference driver (step.cpp:13-147
// -> sph_accelerations.cpp:3-121 -> CUDA_calls.cpp / CUDA_gravity.cpp), but
// every phase is a stream-ordered launch on device-resident FP64 state and
// nothing is copied to the host inside a step.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"

namespace sph {
// kernels (launchers) from the other translation units
size_t radix_scratch_bytes(int n);
int radix_sort_u64(int n, uint64_t *keys, uint32_t *vals, void *scratch, cudaStream_t st);
int morton_keys(int n, const double4 *pos, const double *x, const double *y, const double *z, double *part,
                double *box4, uint64_t *keys, uint32_t *vals, cudaStream_t st);
int peano_keys(int n, const double4 *pos, const double *x, const double *y, const double *z, double *part,
               double *box4, uint64_t *keys, uint32_t *vals, cudaStream_t st);
int tree_layout(int n, TreeView *t);
int build_tree(const TreeView &t, const double4 *pos, float4 *lo, float4 *hi, cudaStream_t st);
int launch_solve_range(const TreeView &t, double4 *pos, int *nevals, unsigned *flags, const sph_params &p,
                       int *n_ngb, int *list, double *dcache, int cap, void *work, int leaf0, int leaf1,
                       cudaStream_t st);
size_t solve_work_bytes(int n, int nleaf);
int launch_find_ngb(const TreeView &t, const double4 *pos, int *n_ngb, int *list, int cap, unsigned *flags,
                    int leaf0, int leaf1, cudaStream_t st);
int launch_density(const HydroArgs &a, cudaStream_t st);
int launch_pressure(int n, double4 *hyd, int eos_mode, double gamma, unsigned *flags, cudaStream_t st);
int launch_hydro(const HydroArgs &a, cudaStream_t st);
int launch_density_mixed(const HydroArgs &a, cudaStream_t st);
int launch_hydro_mixed(const HydroArgs &a, cudaStream_t st);
int launch_gravity(int n, const double4 *src, const double *h2src, double4 *out, int soft_mode, double eps, double G,
                   int precision, const int *mass_mixed, int rank, int world, cudaStream_t st);
int launch_tree_gravity(const TreeView &t, const uint64_t *keys, const double4 *src, void *ws, double4 *out,
                        unsigned *flags, double eps, double theta, double G, int rank, int world, cudaStream_t st);
size_t tree_gravity_workspace_bytes(int n);
int launch_shard_pack(int n, int s0, int s1, const double4 *pos, const double4 *hyd, const double4 *dd,
                      const int *n_ngb, double4 *xbuf, cudaStream_t st);
int launch_shard_unpack(int n, const double4 *xbuf, double4 *pos, double4 *hyd, double4 *dd, int *n_ngb,
                        cudaStream_t st);
int launch_pack_sources(int n, const double4 *pos, const double4 *vel, double4 *src, double *h2, int *mass_mixed,
                        cudaStream_t st);
int launch_predict(int n, double4 *pos, double4 *vel, double4 *hyd, const double4 *dots, double4 *old,
                   const double *sc, cudaStream_t st);
int finish_partial_doubles(int n);
int launch_finish(int n, const double4 *pos, const double4 *vel, const double4 *hyd, double4 *dots,
                  const double4 *grav, const double *vsig, const int *n_ngb, int add_gravity, double cn1, double cn2,
                  double *part, double *sc, unsigned *flags, cudaStream_t st);
int launch_kick(int n, double4 *vel, double4 *hyd, const double4 *dots, const double4 *old, const double *sc,
                cudaStream_t st);
int launch_permute(int n, const uint32_t *order, const Fields &src, const Fields &dst, cudaStream_t st);
int launch_invert(int n, const int *id, int *slot_of, cudaStream_t st);
int launch_field_io(int n, double *arr, int stride, int comp, const int *id, double *flat, int to_state,
                    cudaStream_t st);
int launch_iota(int n, int *id, cudaStream_t st);
int adjoint_part_doubles(int n);
int launch_adjoint(AdjArgs a, const double4 *src, const int *mass_mixed, double eps, double G, int precision,
                   cudaStream_t st);
}  // namespace sph

using namespace sph;

static thread_local std::string g_last_error;

void sph_internal_set_error(const char *msg) { g_last_error = msg ? msg : ""; }

int sph_internal_cuda_fail(cudaError_t err, const char *what, const char *file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(err), file, line);
  g_last_error = buf;
  return SPH_ERR_CUDA;
}

extern "C" const char *cudasph_last_error(void) { return g_last_error.c_str(); }

struct sph_ctx {
  sph_params p;
  int n = 0;
  int device = 0;
  cudaStream_t st = nullptr;
  Fields f[2];
  int cur = 0;
  double4 *old = nullptr;
  int *n_ngb = nullptr, *nevals = nullptr, *list = nullptr;
  int list_cap = 0;  // per particle
  double *dcache = nullptr;  // candidate squared distances of the h solve, layout of list
  char *solve_work = nullptr;  // queue and saved lane states between the h solve's two kernels
  TreeView tree;
  float4 *tlo = nullptr, *thi = nullptr;
  void *tgws = nullptr;  // tree-gravity workspace (radix tree + node moments)
  uint64_t *keys = nullptr;
  uint32_t *vals = nullptr;
  void *sort_scratch = nullptr;
  double *bbox_part = nullptr, *box4 = nullptr;
  double4 *aux = nullptr;  // per-particle factors of the hydro pair loop (scratch)
  double4 *gsrc = nullptr;
  double *gh2 = nullptr;
  int *mass_mixed = nullptr;  // 0 when all masses are equal (set with the gravity sources)
  unsigned *flags = nullptr;
  double *sc = nullptr;  // StepScalars
  double *fin_part = nullptr;
  double *flat = nullptr;  // n doubles: field exchange staging
  int *slot_of = nullptr;
  long long iteration = 0;
  bool need_sort = true;
  bool tree_ok = false, lists_ok = false, density_ok = false;
  long long launches = 0;
  bool profiling = false;
  std::vector<cudaEvent_t> ev[SPH_NPHASES];
  std::vector<cudaEvent_t> pool;
  // CUDA graphs of one whole step, one per parity of the double-buffered
  // state (the sort flips the buffers every step)
  bool use_graph = false;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  long long glaunches[2] = {0, 0};
  // adjoint (allocated on the first cudasph_set_keep(ctx, 1))
  bool keep = false, kept = false;
  double4 *pre_acc = nullptr, *xb = nullptr, *vb = nullptr, *ab = nullptr, *vpb = nullptr, *vpup = nullptr;
  double4 *dsum = nullptr;  // the density loop's raw sums of the kept step (FP64 density only)
  bool dsum_ok = false;
  double *rhob = nullptr, *Pb = nullptr, *omb = nullptr, *psib = nullptr, *divb = nullptr, *curlb = nullptr;
  double *cb = nullptr, *bb = nullptr, *prb = nullptr, *rho_ext = nullptr, *asc = nullptr, *apart = nullptr;
  // sharding (cudasph_set_shard): this context computes shard `rank` of
  // `world` of the leaf-parallel SPH loops and of the gravity work; xbuf is
  // the exchange buffer of the SPH results (2 double4 per particle)
  int rank = 0, world = 1;
  double4 *xbuf = nullptr;
};

static void drop_graphs(sph_ctx *c);

namespace {

// Every phase is an NVTX range on the host thread (names below; a profiler
// attached to the process shows the step's structure) and, with profiling
// on, a pair of CUDA events on the context's stream (cudasph_phase_times).
const char *const kPhaseNames[SPH_NPHASES] = {"sph:sort",    "sph:predict", "sph:tree",     "sph:solve_range",
                                              "sph:find_ngb", "sph:density", "sph:pressure", "sph:hydro",
                                              "sph:gravity", "sph:finish",  "sph:kick",     "sph:adjoint"};

struct PhaseScope {
  sph_ctx *c;
  int ph;
  cudaEvent_t b = nullptr;
  PhaseScope(sph_ctx *c_, int ph_) : c(c_), ph(ph_) {
    nvtxRangePushA(kPhaseNames[ph]);
    if (!c->profiling) return;
    b = take();
    cudaEventRecord(b, c->st);
  }
  cudaEvent_t take() {
    cudaEvent_t e;
    if (!c->pool.empty()) {
      e = c->pool.back();
      c->pool.pop_back();
    } else {
      cudaEventCreate(&e);
    }
    return e;
  }
  ~PhaseScope() {
    nvtxRangePop();
    if (!c->profiling) return;
    cudaEvent_t e = take();
    cudaEventRecord(e, c->st);
    c->ev[ph].push_back(b);
    c->ev[ph].push_back(e);
  }
};

template <class T>
int dalloc(T **p, size_t count) {
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * count);
  if (e != cudaSuccess) {
    sph_internal_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    return SPH_ERR_ALLOC;
  }
  return SPH_OK;
}

int alloc_lists(sph_ctx *c) {
  int cap = c->p.ngb_cap > 0 ? c->p.ngb_cap : (int)(4 * c->p.n_target) + 32;
  if (cap == c->list_cap && c->list) return SPH_OK;
  if (c->list) cudaFree(c->list);
  if (c->dcache) cudaFree(c->dcache);
  c->list = nullptr;
  c->dcache = nullptr;
  c->list_cap = cap;
  size_t entries = (size_t)c->tree.count[0] * kLeaf * (size_t)cap;
  c->lists_ok = false;
  int rc = dalloc(&c->list, entries);
  if (!rc) rc = dalloc(&c->dcache, entries);
  return rc;
}

int check_params(const sph_params *p) {
  if (!p) return SPH_ERR_ARG;
  if (!(p->n_target > 0) || !(p->rel_err > 0) || p->max_iter < 0 || !(p->f_scale > 0)) return SPH_ERR_ARG;
  if (p->eos_mode != SPH_EOS_IDEAL && p->eos_mode != SPH_EOS_GAS_RADIATION) return SPH_ERR_ARG;
  if (p->soft_mode != SPH_SOFT_SPLINE && p->soft_mode != SPH_SOFT_PLUMMER) return SPH_ERR_ARG;
  if (p->soft_mode == SPH_SOFT_PLUMMER && !(p->eps > 0)) return SPH_ERR_ARG;
  if (p->precision != SPH_PREC_FP64 && p->precision != SPH_PREC_MIXED) return SPH_ERR_ARG;
  if (p->ngb_cap < 0 || p->sort_every < 0 || p->mixed_sph < 0 || p->mixed_sph > 3) return SPH_ERR_ARG;
  if (!(p->gamma > 1)) return SPH_ERR_ARG;
  if (p->grav_mode != SPH_GRAV_DIRECT && p->grav_mode != SPH_GRAV_TREE) return SPH_ERR_ARG;
  if (p->key_mode != SPH_KEY_MORTON && p->key_mode != SPH_KEY_PEANO) return SPH_ERR_ARG;
  if (p->grav_mode == SPH_GRAV_TREE && (p->soft_mode != SPH_SOFT_PLUMMER || !(p->theta >= 0) || !(p->theta < 1)))
    return SPH_ERR_ARG;
  return SPH_OK;
}

int use_psi(const sph_params &p) { return p.use_psi < 0 ? (p.soft_mode == SPH_SOFT_SPLINE) : p.use_psi; }

struct FieldRef {
  double *base;
  int stride, comp;
};

FieldRef field_ref(sph_ctx *c, int field) {
  Fields &F = c->f[c->cur];
  FieldRef r{nullptr, 4, field & 3};
  switch (field >> 2) {
    case 0: r.base = (double *)F.pos; break;
    case 1: r.base = (double *)F.vel; break;
    case 2: r.base = (double *)F.hyd; break;
    case 3: r.base = (double *)F.dd; break;
    case 4: r.base = (double *)F.dots; break;
    case 5: r.base = (double *)F.grav; break;
    case 6: r.base = F.vsig; r.stride = 1; r.comp = 0; break;
  }
  return r;
}

// this context's leaves: all of them, or its shard's contiguous range
void shard_leaves(const sph_ctx *c, int &leaf0, int &leaf1) {
  long long lo, hi;
  shard_range(c->tree.count[0], c->rank, c->world, lo, hi);
  leaf0 = (int)lo;
  leaf1 = (int)hi;
}

HydroArgs hydro_args(sph_ctx *c) {
  Fields &F = c->f[c->cur];
  HydroArgs a;
  a.n = c->n;
  a.nleaf = c->tree.count[0];
  a.cap = c->list_cap;
  a.pos = F.pos; a.vel = F.vel; a.hyd = F.hyd; a.dd = F.dd; a.dots = F.dots; a.vsig = F.vsig;
  a.n_ngb = c->n_ngb; a.list = c->list; a.ngb_acc = nullptr; a.aux = c->aux; a.dsum = nullptr;
  a.alpha = c->p.av_alpha; a.beta = c->p.av_beta; a.gamma = c->p.gamma;
  a.use_psi = use_psi(c->p);
  a.jside = 1;
  shard_leaves(c, a.leaf0, a.leaf1);
  return a;
}

}  // namespace

extern "C" sph_params cudasph_default_params(void) {
  sph_params p;
  memset(&p, 0, sizeof(p));
  p.n_target = 24.0;   // DESIRED_NGB, dev_solve_range.cu:14
  p.rel_err = 1e-3;    // CUDA_calls.cpp:4
  p.max_iter = 20;     // MAX_ITER, dev_solve_range.cu:15
  p.f_scale = 0.1;     // dev_solve_range.cu:92
  p.av_alpha = 1.0;    // CUDA_calls.cpp:13
  p.av_beta = 2.0;     // CUDA_calls.cpp:14
  p.gamma = 5.0 / 3.0;
  p.eos_mode = SPH_EOS_GAS_RADIATION;
  p.soft_mode = SPH_SOFT_SPLINE;
  p.eps = 0.0;
  p.use_psi = -1;
  p.cn1 = 0.3;         // compute_timestep.cpp:4
  p.cn2 = 0.2;         // compute_timestep.cpp:5
  p.G = 1.0;
  p.precision = SPH_PREC_FP64;
  p.ngb_cap = 0;
  p.sort_every = 1;
  p.mixed_sph = 0;
  p.grav_mode = SPH_GRAV_DIRECT;
  p.theta = 0.5;
  p.key_mode = SPH_KEY_MORTON;
  return p;
}

extern "C" int cudasph_destroy(sph_ctx *c) {
  if (!c) return SPH_OK;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  for (int b = 0; b < 2; b++) {
    Fields &F = c->f[b];
    cudaFree(F.pos); cudaFree(F.vel); cudaFree(F.hyd); cudaFree(F.dd); cudaFree(F.dots); cudaFree(F.grav);
    cudaFree(F.vsig); cudaFree(F.id);
  }
  cudaFree(c->old); cudaFree(c->n_ngb); cudaFree(c->nevals); cudaFree(c->list); cudaFree(c->dcache);
  cudaFree(c->tlo); cudaFree(c->thi); cudaFree(c->tgws); cudaFree(c->keys); cudaFree(c->vals); cudaFree(c->sort_scratch);
  cudaFree(c->bbox_part); cudaFree(c->box4); cudaFree(c->aux); cudaFree(c->solve_work); cudaFree(c->gsrc); cudaFree(c->gh2); cudaFree(c->mass_mixed); cudaFree(c->xbuf); cudaFree(c->flags);
  cudaFree(c->sc); cudaFree(c->fin_part); cudaFree(c->flat); cudaFree(c->slot_of);
  cudaFree(c->pre_acc); cudaFree(c->dsum); cudaFree(c->xb); cudaFree(c->vb); cudaFree(c->ab); cudaFree(c->vpb); cudaFree(c->vpup);
  cudaFree(c->rhob); cudaFree(c->Pb); cudaFree(c->omb); cudaFree(c->psib); cudaFree(c->divb); cudaFree(c->curlb);
  cudaFree(c->cb); cudaFree(c->bb); cudaFree(c->prb); cudaFree(c->rho_ext); cudaFree(c->asc); cudaFree(c->apart);
  for (int ph = 0; ph < SPH_NPHASES; ph++)
    for (cudaEvent_t e : c->ev[ph]) cudaEventDestroy(e);
  for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
  drop_graphs(c);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return SPH_OK;
}

extern "C" int cudasph_create(const sph_params *params, int n, int device, sph_ctx **out) {
  if (!out || n <= 0) return SPH_ERR_ARG;
  *out = nullptr;
  int rc = check_params(params);
  if (rc) {
    sph_internal_set_error("invalid sph_params");
    return rc;
  }
  SPH_CUDA_TRY(cudaSetDevice(device));
  sph_ctx *c = new sph_ctx();
  c->p = *params;
  c->n = n;
  c->device = device;
  tree_layout(n, &c->tree);
  int nodes = 0;
  for (int l = 0; l < c->tree.levels; l++) nodes += c->tree.count[l];
#define TRY_ALLOC(expr)        \
  do {                         \
    int r__ = (expr);          \
    if (r__) {                 \
      cudasph_destroy(c);      \
      return r__;              \
    }                          \
  } while (0)
  cudaError_t e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return sph_internal_cuda_fail(e, "cudaStreamCreate", __FILE__, __LINE__);
  }
  for (int b = 0; b < 2; b++) {
    Fields &F = c->f[b];
    TRY_ALLOC(dalloc(&F.pos, n)); TRY_ALLOC(dalloc(&F.vel, n)); TRY_ALLOC(dalloc(&F.hyd, n));
    TRY_ALLOC(dalloc(&F.dd, n)); TRY_ALLOC(dalloc(&F.dots, n)); TRY_ALLOC(dalloc(&F.grav, n));
    TRY_ALLOC(dalloc(&F.vsig, n)); TRY_ALLOC(dalloc(&F.id, n));
  }
  TRY_ALLOC(dalloc(&c->old, n));
  TRY_ALLOC(dalloc(&c->n_ngb, n));
  TRY_ALLOC(dalloc(&c->nevals, n));
  TRY_ALLOC(dalloc(&c->tlo, nodes));
  TRY_ALLOC(dalloc(&c->thi, nodes));
  TRY_ALLOC(dalloc((char **)&c->tgws, tree_gravity_workspace_bytes(n)));
  TRY_ALLOC(dalloc(&c->keys, n));
  TRY_ALLOC(dalloc(&c->vals, n));
  TRY_ALLOC(dalloc((char **)&c->sort_scratch, radix_scratch_bytes(n)));
  TRY_ALLOC(dalloc(&c->bbox_part, 148 * 2 * 6));
  TRY_ALLOC(dalloc(&c->box4, 4));
  TRY_ALLOC(dalloc(&c->aux, n));
  TRY_ALLOC(dalloc(&c->solve_work, solve_work_bytes(n, c->tree.count[0])));
  TRY_ALLOC(dalloc(&c->gsrc, n));
  TRY_ALLOC(dalloc(&c->gh2, n));
  TRY_ALLOC(dalloc(&c->mass_mixed, 1));
  TRY_ALLOC(dalloc(&c->flags, 1));
  TRY_ALLOC(dalloc(&c->sc, 4 + SPH_NSTATS));
  TRY_ALLOC(dalloc(&c->fin_part, finish_partial_doubles(n)));
  TRY_ALLOC(dalloc(&c->flat, n));
  TRY_ALLOC(dalloc(&c->slot_of, n));
  TRY_ALLOC(alloc_lists(c));
#undef TRY_ALLOC
  for (int b = 0; b < 2; b++) {
    Fields &F = c->f[b];
    cudaMemsetAsync(F.pos, 0, sizeof(double4) * n, c->st);
    cudaMemsetAsync(F.vel, 0, sizeof(double4) * n, c->st);
    cudaMemsetAsync(F.hyd, 0, sizeof(double4) * n, c->st);
    cudaMemsetAsync(F.dd, 0, sizeof(double4) * n, c->st);
    cudaMemsetAsync(F.dots, 0, sizeof(double4) * n, c->st);
    cudaMemsetAsync(F.grav, 0, sizeof(double4) * n, c->st);
    cudaMemsetAsync(F.vsig, 0, sizeof(double) * n, c->st);
  }
  cudaMemsetAsync(c->n_ngb, 0, sizeof(int) * n, c->st);
  cudaMemsetAsync(c->nevals, 0, sizeof(int) * n, c->st);
  cudaMemsetAsync(c->old, 0, sizeof(double4) * n, c->st);
  cudaMemsetAsync(c->flags, 0, sizeof(unsigned), c->st);
  cudaMemsetAsync(c->sc, 0, sizeof(double) * (4 + SPH_NSTATS), c->st);
  launch_iota(n, c->f[0].id, c->st);
  e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) {
    int r = sph_internal_cuda_fail(e, "cudasph_create", __FILE__, __LINE__);
    cudasph_destroy(c);
    return r;
  }
  *out = c;
  return SPH_OK;
}

extern "C" int cudasph_set_params(sph_ctx *c, const sph_params *p) {
  if (!c) return SPH_ERR_ARG;
  int rc = check_params(p);
  if (rc) return rc;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  drop_graphs(c);  // parameters are baked into captured launches
  c->p = *p;
  return alloc_lists(c);
}

extern "C" int cudasph_get_params(const sph_ctx *c, sph_params *out) {
  if (!c || !out) return SPH_ERR_ARG;
  *out = c->p;
  return SPH_OK;
}

extern "C" int cudasph_num_particles(const sph_ctx *c) { return c ? c->n : 0; }

// ------------------------------ state exchange ------------------------------
static int copy_in(sph_ctx *c, const void *src, size_t bytes, int on_device, void *dst) {
  SPH_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->st));
  return SPH_OK;
}

static void mark_changed(sph_ctx *c, int field) {
  if (field <= SPH_Z) {
    c->need_sort = true;
    c->tree_ok = false;
    c->lists_ok = false;
    c->density_ok = false;
  } else if (field == SPH_RANGE) {
    c->lists_ok = false;
    c->density_ok = false;
  }
}

// One field in or out through the staging buffer `flat`, stream ordered: a
// later copy into `flat` waits for the kernel that read it, so a run of
// fields needs one host synchronisation at the end (for host memory).
static int put_field(sph_ctx *c, int field, const double *src, int on_device) {
  int rc = copy_in(c, src, sizeof(double) * c->n, on_device, c->flat);
  if (rc) return rc;
  FieldRef r = field_ref(c, field);
  launch_field_io(c->n, r.base, r.stride, r.comp, c->f[c->cur].id, c->flat, 1, c->st);
  c->launches++;
  mark_changed(c, field);
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

static int take_field(sph_ctx *c, int field, double *dst, int on_device) {
  FieldRef r = field_ref(c, field);
  launch_field_io(c->n, r.base, r.stride, r.comp, c->f[c->cur].id, c->flat, 0, c->st);
  c->launches++;
  SPH_CUDA_TRY(cudaMemcpyAsync(dst, c->flat, sizeof(double) * c->n,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->st));
  return SPH_OK;
}

extern "C" int cudasph_set_field(sph_ctx *c, int field, const double *src, int on_device) {
  if (!c || !src || field < 0 || field >= SPH_NFIELDS) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  int rc = put_field(c, field, src, on_device);
  if (rc) return rc;
  if (!on_device) SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_get_field(sph_ctx *c, int field, double *dst, int on_device) {
  if (!c || !dst || field < 0 || field >= SPH_NFIELDS) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  int rc = take_field(c, field, dst, on_device);
  if (rc) return rc;
  if (!on_device) SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_set_state(sph_ctx *c, const double *const *fields, int on_device) {
  if (!c || !fields) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  for (int k = 0; k < SPH_NFIELDS; k++) {
    if (!fields[k]) continue;
    int rc = put_field(c, k, fields[k], on_device);
    if (rc) return rc;
  }
  if (!on_device) SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_get_state(sph_ctx *c, double *const *fields, int on_device) {
  if (!c || !fields) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  for (int k = 0; k < SPH_NFIELDS; k++) {
    if (!fields[k]) continue;
    int rc = take_field(c, k, fields[k], on_device);
    if (rc) return rc;
  }
  if (!on_device) SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_get_n_ngb(sph_ctx *c, int *dst, int on_device) {
  if (!c || !dst) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  // reuse the double staging buffer as int scratch
  launch_field_io(c->n, (double *)c->n_ngb, -1, 0, c->f[c->cur].id, c->flat, 0, c->st);
  c->launches++;
  SPH_CUDA_TRY(cudaMemcpyAsync(dst, c->flat, sizeof(int) * c->n,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->st));
  if (!on_device) SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_get_solve_evals(sph_ctx *c, int *dst) {
  if (!c || !dst) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  launch_field_io(c->n, (double *)c->nevals, -1, 0, c->f[c->cur].id, c->flat, 0, c->st);
  c->launches++;
  SPH_CUDA_TRY(cudaMemcpyAsync(dst, c->flat, sizeof(int) * c->n, cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_get_order(sph_ctx *c, int *sorted_ids_host) {
  if (!c || !sorted_ids_host) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaMemcpyAsync(sorted_ids_host, c->f[c->cur].id, sizeof(int) * c->n, cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_set_time(sph_ctx *c, double time, double dt) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  double v[3] = {dt, dt, time};
  SPH_CUDA_TRY(cudaMemcpyAsync(c->sc, v, sizeof(v), cudaMemcpyHostToDevice, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_get_time(sph_ctx *c, double *time, double *dt) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  double v[3];
  SPH_CUDA_TRY(cudaMemcpyAsync(v, c->sc, sizeof(v), cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  if (time) *time = v[2];
  if (dt) *dt = v[1];
  return SPH_OK;
}

extern "C" int cudasph_get_neighbours(sph_ctx *c, int *counts, int64_t *offsets, int *list) {
  if (!c || !counts || !offsets) return SPH_ERR_ARG;
  if (!c->lists_ok) return SPH_ERR_STATE;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  const int n = c->n, cap = c->list_cap, nleaf = c->tree.count[0];
  std::vector<int> ids(n), cnt(n);
  SPH_CUDA_TRY(cudaMemcpyAsync(ids.data(), c->f[c->cur].id, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaMemcpyAsync(cnt.data(), c->n_ngb, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  for (int s = 0; s < n; s++) counts[ids[s]] = cnt[s];
  offsets[0] = 0;
  for (int i = 0; i < n; i++) offsets[i + 1] = offsets[i] + counts[i];
  if (!list) return SPH_OK;
  std::vector<int> lst((size_t)nleaf * kLeaf * cap);
  SPH_CUDA_TRY(cudaMemcpyAsync(lst.data(), c->list, sizeof(int) * lst.size(), cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  for (int s = 0; s < n; s++) {
    const int leaf = s / kLeaf, lane = s % kLeaf;
    const int m = cnt[s] < cap ? cnt[s] : cap;
    int64_t o = offsets[ids[s]];
    for (int k = 0; k < m; k++) list[o + k] = ids[lst[((size_t)leaf * cap + k) * kLeaf + lane]];
  }
  return SPH_OK;
}

// ------------------------------- the phases --------------------------------
#define LAUNCHED(expr) (c->launches += (expr))

extern "C" int cudasph_sort(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_SORT);
  const int n = c->n;
  Fields &S = c->f[c->cur];
  Fields &D = c->f[1 - c->cur];
  if (c->p.key_mode == SPH_KEY_PEANO)
    LAUNCHED(peano_keys(n, S.pos, nullptr, nullptr, nullptr, c->bbox_part, c->box4, c->keys, c->vals, c->st));
  else
    LAUNCHED(morton_keys(n, S.pos, nullptr, nullptr, nullptr, c->bbox_part, c->box4, c->keys, c->vals, c->st));
  LAUNCHED(radix_sort_u64(n, c->keys, c->vals, c->sort_scratch, c->st));
  LAUNCHED(launch_permute(n, c->vals, S, D, c->st));
  c->cur = 1 - c->cur;
  c->need_sort = false;
  c->tree_ok = c->lists_ok = c->density_ok = false;
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_predict(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_PREDICT);
  Fields &F = c->f[c->cur];
  LAUNCHED(launch_predict(c->n, F.pos, F.vel, F.hyd, F.dots, c->old, c->sc, c->st));
  c->tree_ok = c->lists_ok = c->density_ok = false;
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_build_tree(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  if (c->need_sort) {
    int rc = cudasph_sort(c);
    if (rc) return rc;
  }
  PhaseScope ps(c, SPH_PH_TREE);
  LAUNCHED(build_tree(c->tree, c->f[c->cur].pos, c->tlo, c->thi, c->st));
  c->tree.lo = c->tlo;
  c->tree.hi = c->thi;
  c->tree_ok = true;
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_solve_range(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (!c->tree_ok) {
    int rc = cudasph_build_tree(c);
    if (rc) return rc;
  }
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_SOLVE);
  int leaf0, leaf1;
  shard_leaves(c, leaf0, leaf1);
  LAUNCHED(launch_solve_range(c->tree, c->f[c->cur].pos, c->nevals, c->flags, c->p, c->n_ngb, c->list, c->dcache,
                              c->list_cap, c->solve_work, leaf0, leaf1, c->st));
  // the solve writes the neighbour lists at the final ranges (find_ngb fused)
  c->lists_ok = true;
  c->density_ok = false;
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_find_ngb(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (!c->tree_ok) {
    int rc = cudasph_build_tree(c);
    if (rc) return rc;
  }
  if (c->lists_ok) return SPH_OK;  // already written by the h solve at these ranges
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_FIND);
  int leaf0, leaf1;
  shard_leaves(c, leaf0, leaf1);
  LAUNCHED(launch_find_ngb(c->tree, c->f[c->cur].pos, c->n_ngb, c->list, c->list_cap, c->flags, leaf0, leaf1, c->st));
  c->lists_ok = true;
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_density(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (!c->lists_ok) return SPH_ERR_STATE;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_DENSITY);
  HydroArgs a = hydro_args(c);
  const bool fp32 = c->p.precision == SPH_PREC_MIXED && (c->p.mixed_sph & 1);
  // a kept step records the FP64 loop's raw sums for the density VJP
  a.dsum = (c->keep && !fp32) ? c->dsum : nullptr;
  c->dsum_ok = a.dsum != nullptr;
  if (fp32) LAUNCHED(launch_density_mixed(a, c->st));
  else LAUNCHED(launch_density(a, c->st));
  c->density_ok = true;
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_pressure(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_PRESSURE);
  LAUNCHED(launch_pressure(c->n, c->f[c->cur].hyd, c->p.eos_mode, c->p.gamma, c->flags, c->st));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_hydro(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (!c->lists_ok) return SPH_ERR_STATE;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_HYDRO);
  Fields &F = c->f[c->cur];
  SPH_CUDA_TRY(cudaMemsetAsync(F.dots, 0, sizeof(double4) * c->n, c->st));
  // a shard writes the signal speeds of its own particles only; zeros elsewhere make the sum over shards exact
  if (c->world > 1) SPH_CUDA_TRY(cudaMemsetAsync(F.vsig, 0, sizeof(double) * c->n, c->st));
  HydroArgs a = hydro_args(c);
  if (c->p.precision == SPH_PREC_MIXED && (c->p.mixed_sph & 2)) LAUNCHED(launch_hydro_mixed(a, c->st));
  else LAUNCHED(launch_hydro(a, c->st));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_sph_accelerations(sph_ctx *c) {
  int rc;
  if ((rc = cudasph_build_tree(c))) return rc;
  if ((rc = cudasph_solve_range(c))) return rc;
  if ((rc = cudasph_find_ngb(c))) return rc;
  if ((rc = cudasph_density(c))) return rc;
  if ((rc = cudasph_pressure(c))) return rc;
  if ((rc = cudasph_hydro(c))) return rc;
  return SPH_OK;
}

extern "C" int cudasph_gravity(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (c->p.grav_mode == SPH_GRAV_TREE && !c->tree_ok) {
    int rc = cudasph_build_tree(c);
    if (rc) return rc;
  }
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_GRAVITY);
  Fields &F = c->f[c->cur];
  if (c->p.grav_mode == SPH_GRAV_TREE) {
    LAUNCHED(launch_pack_sources(c->n, F.pos, F.vel, c->gsrc, c->gh2, c->mass_mixed, c->st));
    // the radix tree is built from the sort's keys, which match the current order
    LAUNCHED(launch_tree_gravity(c->tree, c->keys, c->gsrc, c->tgws, F.grav, c->flags, c->p.eps, c->p.theta, c->p.G,
                                 c->rank, c->world, c->st));
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
  }
  LAUNCHED(launch_pack_sources(c->n, F.pos, F.vel, c->gsrc, c->gh2, c->mass_mixed, c->st));
  LAUNCHED(launch_gravity(c->n, c->gsrc, c->gh2, F.grav, c->p.soft_mode, c->p.eps, c->p.G, c->p.precision,
                          c->mass_mixed, c->rank, c->world, c->st));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_finish(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_FINISH);
  Fields &F = c->f[c->cur];
  LAUNCHED(launch_finish(c->n, F.pos, F.vel, F.hyd, F.dots, F.grav, F.vsig, c->n_ngb, 1, c->p.cn1, c->p.cn2,
                         c->fin_part, c->sc, c->flags, c->st));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_kick(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  PhaseScope ps(c, SPH_PH_KICK);
  Fields &F = c->f[c->cur];
  LAUNCHED(launch_kick(c->n, F.vel, F.hyd, F.dots, c->old, c->sc, c->st));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

static void drop_graphs(sph_ctx *c) {
  for (int k = 0; k < 2; k++) {
    if (c->gexec[k]) cudaGraphExecDestroy(c->gexec[k]);
    c->gexec[k] = nullptr;
    c->glaunches[k] = 0;
  }
}

static int step_body(sph_ctx *c);

// One step, replayed from a captured CUDA graph when the step is the steady
// kind (sorted every step, no profiling events, no adjoint bookkeeping): the
// ~45 launches of a step then cost one graph launch.  The first step of each
// buffer parity runs under stream capture; the host bookkeeping it performs
// (buffer flip, phase validity) is then repeated by hand on every replay.
extern "C" int cudasph_step(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (c->world > 1) {
    sph_internal_set_error("cudasph_step: a sharded context is stepped phase by phase with the exchanges "
                           "between them (cudasph_shard_pack / unpack, sums of dots, vsig and grav)");
    return SPH_ERR_STATE;
  }
  const bool graphable = c->use_graph && !c->need_sort && c->p.sort_every == 1 && !c->profiling && !c->keep;
  if (!graphable) return step_body(c);
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  const int par = c->cur;
  if (c->gexec[par]) {
    SPH_CUDA_TRY(cudaGraphLaunch(c->gexec[par], c->st));
    c->iteration++;
    c->cur = 1 - c->cur;
    c->tree_ok = c->lists_ok = c->density_ok = true;
    c->kept = false;
    c->launches += c->glaunches[par];
    return SPH_OK;
  }
  const long long l0 = c->launches;
  SPH_CUDA_TRY(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  int rc = step_body(c);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->st, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return sph_internal_cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  e = cudaGraphInstantiate(&c->gexec[par], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    c->gexec[par] = nullptr;
    return sph_internal_cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
  }
  c->glaunches[par] = c->launches - l0;
  SPH_CUDA_TRY(cudaGraphLaunch(c->gexec[par], c->st));
  return SPH_OK;
}

extern "C" int cudasph_set_graph(sph_ctx *c, int on) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  if (!on) drop_graphs(c);
  c->use_graph = on != 0;
  return SPH_OK;
}

extern "C" int cudasph_begin_step(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  c->iteration++;
  if (c->need_sort || (c->p.sort_every > 0 && c->iteration % c->p.sort_every == 0)) return cudasph_sort(c);
  return SPH_OK;
}

static int step_body(sph_ctx *c) {
  int rc;
  if ((rc = cudasph_begin_step(c))) return rc;
  if (c->keep) {
    // the adjoint needs the accelerations the predictor uses (a0, du0)
    SPH_CUDA_TRY(cudaSetDevice(c->device));
    SPH_CUDA_TRY(cudaMemcpyAsync(c->pre_acc, c->f[c->cur].dots, sizeof(double4) * c->n, cudaMemcpyDeviceToDevice,
                                 c->st));
  }
  c->kept = false;
  if ((rc = cudasph_predict(c))) return rc;
  if ((rc = cudasph_sph_accelerations(c))) return rc;
  if ((rc = cudasph_gravity(c))) return rc;
  if ((rc = cudasph_finish(c))) return rc;
  if ((rc = cudasph_kick(c))) return rc;
  c->kept = c->keep;
  return SPH_OK;
}

extern "C" int cudasph_steps(sph_ctx *c, int k) {
  for (int i = 0; i < k; i++) {
    int rc = cudasph_step(c);
    if (rc) return rc;
  }
  return SPH_OK;
}

extern "C" int cudasph_step_host(sph_ctx *c, const double *const *fields_in, double *const *fields_out) {
  int rc;
  if (fields_in && (rc = cudasph_set_state(c, fields_in, 0))) return rc;
  if ((rc = cudasph_step(c))) return rc;
  if (fields_out && (rc = cudasph_get_state(c, fields_out, 0))) return rc;
  return SPH_OK;
}

extern "C" int cudasph_synchronize(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_statistics(sph_ctx *c, double *stats) {
  if (!c || !stats) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaMemcpyAsync(stats, c->sc + 4, sizeof(double) * SPH_NSTATS, cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_device_status(sph_ctx *c, unsigned *flags) {
  if (!c || !flags) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaMemcpyAsync(flags, c->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaMemsetAsync(c->flags, 0, sizeof(unsigned), c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_set_profiling(sph_ctx *c, int on) {
  if (!c) return SPH_ERR_ARG;
  c->profiling = on != 0;
  return SPH_OK;
}

extern "C" int cudasph_phase_times(sph_ctx *c, double *ms, int *launches) {
  if (!c) return SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  for (int ph = 0; ph < SPH_NPHASES; ph++) {
    double t = 0;
    auto &v = c->ev[ph];
    for (size_t k = 0; k + 1 < v.size(); k += 2) {
      float x = 0;
      cudaEventElapsedTime(&x, v[k], v[k + 1]);
      t += x;
    }
    if (ms) ms[ph] = t;
    if (launches) launches[ph] = (int)(v.size() / 2);
  }
  return SPH_OK;
}

extern "C" int cudasph_reset_counters(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->st);
  for (int ph = 0; ph < SPH_NPHASES; ph++) {
    for (cudaEvent_t e : c->ev[ph]) c->pool.push_back(e);
    c->ev[ph].clear();
  }
  c->launches = 0;
  return SPH_OK;
}

extern "C" long long cudasph_kernel_launches(const sph_ctx *c) { return c ? c->launches : 0; }

// ------------------------------- the adjoint --------------------------------
extern "C" int cudasph_set_keep(sph_ctx *c, int on) {
  if (!c) return SPH_ERR_ARG;
  if (on && c->world > 1) {
    sph_internal_set_error("cudasph_set_keep: the adjoint runs on an unsharded context");
    return SPH_ERR_STATE;
  }
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  if (on && !c->pre_acc) {
    const int n = c->n;
    int rc = SPH_OK;
    double4 **d4[] = {&c->pre_acc, &c->xb, &c->vb, &c->ab, &c->vpb, &c->vpup, &c->dsum};
    for (double4 **p : d4)
      if (!rc) rc = dalloc(p, n);
    double **d1[] = {&c->rhob, &c->Pb, &c->omb, &c->psib, &c->divb, &c->curlb, &c->cb, &c->bb, &c->prb, &c->rho_ext};
    for (double **p : d1)
      if (!rc) rc = dalloc(p, n);
    if (!rc) rc = dalloc(&c->asc, 8);
    if (!rc) rc = dalloc(&c->apart, adjoint_part_doubles(n));
    if (rc) return rc;
    SPH_CUDA_TRY(cudaMemsetAsync(c->xb, 0, sizeof(double4) * n, c->st));
    SPH_CUDA_TRY(cudaMemsetAsync(c->vb, 0, sizeof(double4) * n, c->st));
    SPH_CUDA_TRY(cudaMemsetAsync(c->ab, 0, sizeof(double4) * n, c->st));
    SPH_CUDA_TRY(cudaMemsetAsync(c->rho_ext, 0, sizeof(double) * n, c->st));
    SPH_CUDA_TRY(cudaMemsetAsync(c->asc, 0, sizeof(double) * 8, c->st));
  }
  c->keep = on != 0;
  return SPH_OK;
}

static int adj_ref(sph_ctx *c, int field, double **base, int *stride, int *comp) {
  if (!c->pre_acc) return SPH_ERR_STATE;
  *stride = 4;
  if (field >= SPH_ADJ_X && field <= SPH_ADJ_Z) { *base = (double *)c->xb; *comp = field - SPH_ADJ_X; }
  else if (field >= SPH_ADJ_VX && field <= SPH_ADJ_U) { *base = (double *)c->vb; *comp = field - SPH_ADJ_VX; }
  else if (field >= SPH_ADJ_AX && field <= SPH_ADJ_DU) { *base = (double *)c->ab; *comp = field - SPH_ADJ_AX; }
  else if (field == SPH_ADJ_RHO) { *base = c->rho_ext; *stride = 1; *comp = 0; }
  else return SPH_ERR_ARG;
  return SPH_OK;
}

extern "C" int cudasph_adjoint_set_field(sph_ctx *c, int field, const double *src, int on_device) {
  if (!c || !src) return SPH_ERR_ARG;
  double *base;
  int stride, comp;
  int rc = adj_ref(c, field, &base, &stride, &comp);
  if (rc) return rc;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  rc = copy_in(c, src, sizeof(double) * c->n, on_device, c->flat);
  if (rc) return rc;
  launch_field_io(c->n, base, stride, comp, c->f[c->cur].id, c->flat, 1, c->st);
  c->launches++;
  SPH_CUDA_TRY(cudaGetLastError());
  if (!on_device) SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_adjoint_get_field(sph_ctx *c, int field, double *dst, int on_device) {
  if (!c || !dst) return SPH_ERR_ARG;
  double *base;
  int stride, comp;
  int rc = adj_ref(c, field, &base, &stride, &comp);
  if (rc) return rc;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  launch_field_io(c->n, base, stride, comp, c->f[c->cur].id, c->flat, 0, c->st);
  c->launches++;
  SPH_CUDA_TRY(cudaMemcpyAsync(dst, c->flat, sizeof(double) * c->n,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->st));
  if (!on_device) SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_adjoint_set_dt(sph_ctx *c, double dtbar) {
  if (!c || !c->asc) return c ? SPH_ERR_STATE : SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaMemcpyAsync(c->asc, &dtbar, sizeof(double), cudaMemcpyHostToDevice, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_adjoint_get_dt(sph_ctx *c, double *dtbar) {
  if (!c || !dtbar || !c->asc) return c ? SPH_ERR_STATE : SPH_ERR_ARG;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaMemcpyAsync(dtbar, c->asc + 1, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return SPH_OK;
}

extern "C" int cudasph_adjoint(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (!c->kept) {
    sph_internal_set_error("cudasph_adjoint: the last step was not taken with cudasph_set_keep(ctx, 1)");
    return SPH_ERR_STATE;
  }
  if (c->p.soft_mode != SPH_SOFT_PLUMMER || c->p.grav_mode != SPH_GRAV_DIRECT) {
    sph_internal_set_error("cudasph_adjoint: implemented for direct Plummer gravity");
    return SPH_ERR_ARG;
  }
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  Fields &F = c->f[c->cur];
  AdjArgs a;
  memset(&a, 0, sizeof(a));
  a.n = c->n;
  a.nleaf = c->tree.count[0];
  a.cap = c->list_cap;
  a.pos = F.pos; a.vel = F.vel; a.hyd = F.hyd; a.dd = F.dd; a.dots = F.dots; a.vsig = F.vsig;
  a.old = c->old; a.pre_acc = c->pre_acc; a.x0 = nullptr; a.vpup = c->vpup;
  a.n_ngb = c->n_ngb; a.list = c->list; a.sc = c->sc;
  a.xb = c->xb; a.vb = c->vb; a.ab = c->ab; a.vpb = c->vpb;
  a.rhob = c->rhob; a.Pb = c->Pb; a.omb = c->omb; a.psib = c->psib; a.divb = c->divb; a.curlb = c->curlb;
  a.cb = c->cb; a.bb = c->bb; a.prb = c->prb; a.rho_ext = c->rho_ext; a.aux = c->aux;
  a.dsum = c->dsum_ok ? c->dsum : nullptr;
  a.asc = c->asc; a.part = c->apart;
  a.alpha = c->p.av_alpha; a.beta = c->p.av_beta; a.gamma = c->p.gamma; a.cn1 = c->p.cn1; a.cn2 = c->p.cn2;
  a.eos_mode = c->p.eos_mode; a.use_psi = use_psi(c->p);
  PhaseScope ps(c, SPH_PH_ADJOINT);
  c->launches += launch_adjoint(a, c->gsrc, c->mass_mixed, c->p.eps, c->p.G, c->p.precision, c->st);
  // the density injection is per step
  SPH_CUDA_TRY(cudaMemsetAsync(c->rho_ext, 0, sizeof(double) * c->n, c->st));
  SPH_CUDA_TRY(cudaGetLastError());
  c->kept = false;
  return SPH_OK;
}

// ------------------------------- sharding ------------------------------------
extern "C" int cudasph_shard_range(long long count, int rank, int world, long long *lo, long long *hi) {
  if (!lo || !hi || count < 0 || world < 1 || rank < 0 || rank >= world) return SPH_ERR_ARG;
  shard_range(count, rank, world, *lo, *hi);
  return SPH_OK;
}

extern "C" int cudasph_set_shard(sph_ctx *c, int rank, int world) {
  if (!c || world < 1 || rank < 0 || rank >= world) return SPH_ERR_ARG;
  if (c->keep && world > 1) {
    sph_internal_set_error("cudasph_set_shard: the adjoint runs on an unsharded context");
    return SPH_ERR_STATE;
  }
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  SPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  if (!c->xbuf) {
    int rc = dalloc(&c->xbuf, 2 * (size_t)c->n);
    if (rc) return rc;
  }
  drop_graphs(c);
  c->rank = rank;
  c->world = world;
  c->lists_ok = c->density_ok = false;
  return SPH_OK;
}

extern "C" int cudasph_get_shard(sph_ctx *c, int *rank, int *world, int *leaf0, int *leaf1) {
  if (!c) return SPH_ERR_ARG;
  if (rank) *rank = c->rank;
  if (world) *world = c->world;
  int l0, l1;
  shard_leaves(c, l0, l1);
  if (leaf0) *leaf0 = l0;
  if (leaf1) *leaf1 = l1;
  return SPH_OK;
}

extern "C" int cudasph_shard_pack(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (!c->xbuf || !c->density_ok) return SPH_ERR_STATE;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  Fields &F = c->f[c->cur];
  int l0, l1;
  shard_leaves(c, l0, l1);
  const int s0 = l0 * kLeaf, s1 = min(l1 * kLeaf, c->n);
  LAUNCHED(launch_shard_pack(c->n, s0, s1, F.pos, F.hyd, F.dd, c->n_ngb, c->xbuf, c->st));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_shard_unpack(sph_ctx *c) {
  if (!c) return SPH_ERR_ARG;
  if (!c->xbuf) return SPH_ERR_STATE;
  SPH_CUDA_TRY(cudaSetDevice(c->device));
  Fields &F = c->f[c->cur];
  LAUNCHED(launch_shard_unpack(c->n, c->xbuf, F.pos, F.hyd, F.dd, c->n_ngb, c->st));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_device_buffer(sph_ctx *c, int which, void **ptr, long long *doubles) {
  if (!c || !ptr || !doubles) return SPH_ERR_ARG;
  Fields &F = c->f[c->cur];
  switch (which) {
    case SPH_BUF_EXCHANGE:
      if (!c->xbuf) return SPH_ERR_STATE;
      *ptr = c->xbuf; *doubles = 8LL * c->n; break;
    case SPH_BUF_DOTS: *ptr = F.dots; *doubles = 4LL * c->n; break;
    case SPH_BUF_VSIG: *ptr = F.vsig; *doubles = c->n; break;
    case SPH_BUF_GRAV: *ptr = F.grav; *doubles = 4LL * c->n; break;
    default: return SPH_ERR_ARG;
  }
  return SPH_OK;
}

extern "C" int cudasph_get_stream(sph_ctx *c, void **stream) {
  if (!c || !stream) return SPH_ERR_ARG;
  *stream = (void *)c->st;
  return SPH_OK;
}

// internal accessors used by the reference-ABI layer (legacy.cu)
namespace sph {
cudaStream_t ctx_stream(sph_ctx *c) { return c->st; }
Fields &ctx_fields(sph_ctx *c) { return c->f[c->cur]; }
int *ctx_n_ngb(sph_ctx *c) { return c->n_ngb; }
int *ctx_list(sph_ctx *c, int *cap) {
  *cap = c->list_cap;
  return c->list;
}
const TreeView &ctx_tree(sph_ctx *c) { return c->tree; }
unsigned *ctx_flags(sph_ctx *c) { return c->flags; }
void ctx_mark_lists(sph_ctx *c) { c->lists_ok = true; }
void ctx_mark_positions(sph_ctx *c) {
  c->need_sort = true;
  c->tree_ok = c->lists_ok = c->density_ok = false;
}
int *ctx_slot_of(sph_ctx *c) { return c->slot_of; }
HydroArgs ctx_hydro_args(sph_ctx *c) { return hydro_args(c); }
}  // namespace sph
