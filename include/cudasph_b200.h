/*
 * cudasph_b200.h -- C ABI of the B200 (sm_100a) SPH + self-gravity step.
 *
 * Two layers:
 *
 *  1. The native ("v2") API: an opaque context that owns a device-resident,
 *     tree-ordered particle state (FP64 SoA of double4 records) and runs the
 *     per-step pipeline of the reference driver (step.cpp:13-147):
 *        sort -> predict -> [tree, solve_range, find_ngb, density, pressure,
 *        hydro] -> gravity -> diagnostics -> timestep -> kick.
 *     Every phase is also callable on its own.  All calls are ordered on the
 *     context's CUDA stream; errors are returned as sph_status codes, and
 *     device-side conditions (list overflow, walk-stack overflow, ...) are
 *     accumulated in a status word read by cudasph_device_status().
 *
 *  2. The reference's own extern "C" symbols (CUDAsph.h:22-48, defined in
 *     host_calls.cu:27-376), with the reference's signatures and float4
 *     layouts, so that the reference's C++ driver links against this library
 *     unchanged.  They are implemented on top of layer 1.
 *
 * All pointers are plain pointers; no C++ or torch types cross this boundary.
 */
#ifndef CUDASPH_B200_H_
#define CUDASPH_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* status codes (returned)                                                 */
/* ---------------------------------------------------------------------- */
typedef enum {
  SPH_OK = 0,
  SPH_ERR_CUDA = 1,      /* a CUDA runtime call failed (message: cudasph_last_error) */
  SPH_ERR_ARG = 2,       /* invalid argument */
  SPH_ERR_ALLOC = 3,     /* device allocation failed */
  SPH_ERR_DEVICE = 4,    /* a device-side condition was raised (see the flags below) */
  SPH_ERR_STATE = 5      /* a phase was called before its inputs exist */
} sph_status;

/* device-side condition flags (cudasph_device_status) */
#define SPH_FLAG_NGB_OVERFLOW 0x1u      /* a neighbour list longer than ngb_cap was truncated */
#define SPH_FLAG_STACK_OVERFLOW 0x2u    /* a tree walk ran out of stack (results incomplete) */
#define SPH_FLAG_NONFINITE 0x4u         /* a non-finite EOS root or timestep was produced */
#define SPH_FLAG_H_NOT_CONVERGED 0x8u   /* the h solve stopped at max_iter (reference behaviour) */

/* ---------------------------------------------------------------------- */
/* parameters                                                              */
/* ---------------------------------------------------------------------- */
typedef enum { SPH_EOS_IDEAL = 0, SPH_EOS_GAS_RADIATION = 1 } sph_eos_mode;
typedef enum { SPH_SOFT_SPLINE = 0, SPH_SOFT_PLUMMER = 1 } sph_soft_mode;
typedef enum { SPH_PREC_FP64 = 0, SPH_PREC_MIXED = 1 } sph_precision;
typedef enum { SPH_GRAV_DIRECT = 0, SPH_GRAV_TREE = 1 } sph_grav_mode;
typedef enum { SPH_KEY_MORTON = 0, SPH_KEY_PEANO = 1 } sph_key_mode;

typedef struct {
  double n_target;   /* smoothed neighbour number; DESIRED_NGB, dev_solve_range.cu:14 */
  double rel_err;    /* h-solve tolerance; CUDA_calls.cpp:4 */
  int max_iter;      /* MAX_ITER, dev_solve_range.cu:15 */
  double f_scale;    /* Newton step clamp in the bracket phase, dev_solve_range.cu:92 */
  double av_alpha;   /* CUDA_calls.cpp:13 */
  double av_beta;    /* CUDA_calls.cpp:14 */
  double gamma;      /* adiabatic index (sound speed and ideal EOS), dev_art_visc.cu:15 */
  int eos_mode;      /* sph_eos_mode; the reference has gas + radiation only */
  int soft_mode;     /* sph_soft_mode; the reference softens with the spline at range */
  double eps;        /* Plummer softening length */
  int use_psi;       /* Psi (softening grad-h) term of dev_hydro_dots.cu:69-70; -1 = auto */
  double cn1, cn2;   /* Courant factors, compute_timestep.cpp:4-5 */
  double G;          /* gravitational constant (1 in the reference's solar units) */
  int precision;     /* sph_precision */
  int ngb_cap;       /* neighbour-list capacity per particle (0 = 4 * n_target + 32) */
  int sort_every;    /* Morton re-sort period in steps (reference: 100, step.cpp:26) */
  int mixed_sph;     /* mixed form only: bit 0 = density pair terms in FP32, bit 1 = hydro
                        pair terms in FP32; a cleared bit keeps that loop in FP64.  Default 0:
                        the SPH loops are gather-bound, so FP64 pair terms cost ~0.5 % of a
                        1M-particle step, while FP32 ones raise the RMS total-force error of a
                        star near hydrostatic equilibrium (hydro and gravity nearly cancel)
                        from 4.9e-7 to 2.2e-5 */
  int grav_mode;     /* sph_grav_mode: direct N^2 sum (the reference's sph_grav_kernel.cu, default)
                        or the Barnes-Hut tree with quadrupoles (no counterpart in the reference;
                        Plummer softening only; force error set by theta) */
  double theta;      /* tree opening angle: a node of radius b is accepted when b < theta * its
                        distance to the target group's box (default 0.5) */
  int key_mode;      /* sph_key_mode of the spatial sort: Morton keys, 21 bits per dimension in
                        the double bounding cube (default), or the reference's Peano-Hilbert keys
                        (sort_bodies.cpp:66-160: positions rounded to float, 18 bits per
                        dimension), which reproduce its particle order */
} sph_params;

/* particle fields, addressed in the caller's ORIGINAL particle order */
typedef enum {
  SPH_X = 0, SPH_Y, SPH_Z, SPH_RANGE,        /* bodies_pos {x,y,z,range = 2h} */
  SPH_VX, SPH_VY, SPH_VZ, SPH_M,             /* bodies_vel {vx,vy,vz,mass} */
  SPH_RHO, SPH_P, SPH_U, SPH_MU,             /* hydro_data {rho,P,u,mean_mu} */
  SPH_DIVV, SPH_CURLV, SPH_OMEGA, SPH_PSI,   /* dots_data {divv,curlv,omega,psi} */
  SPH_AX, SPH_AY, SPH_AZ, SPH_DU,            /* bodies_dots {ax,ay,az,du/dt} (total) */
  SPH_GX, SPH_GY, SPH_GZ, SPH_PHI,           /* grav_data {gx,gy,gz,phi} */
  SPH_VSIG,                                  /* hydro_data2.x (max signal speed) */
  SPH_NFIELDS
} sph_field;

/* diagnostics vector of cudasph_statistics (system_statistics.cpp:4-84,
 * step.cpp:99-117, compute_timestep.cpp:3-25) */
enum {
  SPH_ST_W = 0, SPH_ST_T, SPH_ST_U, SPH_ST_E,
  SPH_ST_JX, SPH_ST_JY, SPH_ST_JZ,
  SPH_ST_RCMX, SPH_ST_RCMY, SPH_ST_RCMZ,
  SPH_ST_VCMX, SPH_ST_VCMY, SPH_ST_VCMZ,
  SPH_ST_MTOT,
  SPH_ST_FX, SPH_ST_FY, SPH_ST_FZ,           /* total force  sum m a */
  SPH_ST_TX, SPH_ST_TY, SPH_ST_TZ,           /* total torque sum m x cross a */
  SPH_ST_NGB_MEAN, SPH_ST_NGB_SIGMA, SPH_ST_NGB_MIN, SPH_ST_NGB_MAX,
  SPH_ST_DT_VEL, SPH_ST_DT_ETH, SPH_ST_DT,   /* compute_timestep minima */
  SPH_ST_TIME, SPH_ST_DT_OLD,
  SPH_NSTATS
};

typedef struct sph_ctx sph_ctx;

/* defaults = the reference's constants (N 24, rel_err 1e-3, MAX_ITER 20,
 * f_scale 0.1, alpha 1, beta 2, gamma 5/3, gas+radiation EOS, spline
 * softening, Courant 0.3/0.2, G 1), FP64, sort every step. */
sph_params cudasph_default_params(void);

/* lifecycle */
int cudasph_create(const sph_params *params, int n, int device, sph_ctx **out);
int cudasph_destroy(sph_ctx *ctx);
const char *cudasph_last_error(void);
int cudasph_set_params(sph_ctx *ctx, const sph_params *params);
int cudasph_get_params(const sph_ctx *ctx, sph_params *out);
int cudasph_num_particles(const sph_ctx *ctx);

/* state exchange; `on_device` = 1 when src/dst is a device pointer.
 * Arrays are n doubles in the caller's original order. */
int cudasph_set_field(sph_ctx *ctx, int field, const double *src, int on_device);
int cudasph_get_field(sph_ctx *ctx, int field, double *dst, int on_device);
/* whole-state exchange in one call: fields[k] for k < SPH_NFIELDS (NULL = skip) */
int cudasph_set_state(sph_ctx *ctx, const double *const *fields, int on_device);
int cudasph_get_state(sph_ctx *ctx, double *const *fields, int on_device);
int cudasph_get_n_ngb(sph_ctx *ctx, int *dst, int on_device);
/* the tree (sorted) slot of each original particle: slot_of[orig] */
int cudasph_get_order(sph_ctx *ctx, int *sorted_ids_host);
int cudasph_set_time(sph_ctx *ctx, double time, double dt);
int cudasph_get_time(sph_ctx *ctx, double *time, double *dt);

/* neighbour lists in original ids: counts[n]; offsets[n+1] (int64) and
 * list[offsets[n]] ascending by tree slot.  Pass list = NULL to get the
 * counts and offsets only. */
int cudasph_get_neighbours(sph_ctx *ctx, int *counts, int64_t *offsets, int *list);

/* pipeline phases (stream ordered; see step.cpp:13-147 for the order) */
int cudasph_sort(sph_ctx *ctx);              /* Morton keys + radix sort + permute (sort_bodies.cpp:119) */
int cudasph_predict(sph_ctx *ctx);           /* step.cpp:38-61 */
int cudasph_build_tree(sph_ctx *ctx);        /* kd_tree.cpp:97-128 replacement */
int cudasph_solve_range(sph_ctx *ctx);       /* dev_solve_range.cu:174 */
int cudasph_find_ngb(sph_ctx *ctx);          /* dev_find_ngb.cu:75 */
int cudasph_density(sph_ctx *ctx);           /* dev_density_loop.cu:88 */
int cudasph_pressure(sph_ctx *ctx);          /* dev_compute_pressure.cu:99 */
int cudasph_hydro(sph_ctx *ctx);             /* dev_hydro_dots.cu:86 + sph_accelerations.cpp:106-114 */
int cudasph_sph_accelerations(sph_ctx *ctx); /* tree .. hydro, sph_accelerations.cpp:3-121 */
int cudasph_gravity(sph_ctx *ctx);           /* sph_grav_kernel.cu:179 */
int cudasph_finish(sph_ctx *ctx);            /* a += g, diagnostics, timestep (step.cpp:96-127) */
int cudasph_kick(sph_ctx *ctx);              /* step.cpp:128-134 */
int cudasph_step(sph_ctx *ctx);              /* the whole step */
/* the step's opening when it is driven phase by phase: count the step and
 * re-sort when due (every sort_every steps, or after positions were set) */
int cudasph_begin_step(sph_ctx *ctx);
/* Replay steady steps (sorted every step, profiling and keep off) from a
 * captured CUDA graph: one graph launch per step instead of ~45 launches.
 * Changing parameters drops the captured graphs. */
int cudasph_set_graph(sph_ctx *ctx, int on);
int cudasph_steps(sph_ctx *ctx, int k);      /* k whole steps */

/* End-to-end step through host buffers, the way the reference driver owns
 * its state: copy the fields in (host, pinned or not), run one step, copy
 * the fields out.  fields_in/fields_out as in cudasph_set_state. */
int cudasph_step_host(sph_ctx *ctx, const double *const *fields_in, double *const *fields_out);

int cudasph_synchronize(sph_ctx *ctx);
int cudasph_statistics(sph_ctx *ctx, double *stats /* SPH_NSTATS */);
/* read and clear the device condition flags (synchronizes) */
int cudasph_device_status(sph_ctx *ctx, unsigned *flags);
/* number of h-solve evaluations per particle of the last solve (original order) */
int cudasph_get_solve_evals(sph_ctx *ctx, int *dst);

/* instrumentation: CUDA-event time of each phase, summed since the last reset */
enum {
  SPH_PH_SORT = 0, SPH_PH_PREDICT, SPH_PH_TREE, SPH_PH_SOLVE, SPH_PH_FIND, SPH_PH_DENSITY,
  SPH_PH_PRESSURE, SPH_PH_HYDRO, SPH_PH_GRAVITY, SPH_PH_FINISH, SPH_PH_KICK, SPH_PH_ADJOINT, SPH_NPHASES
};
int cudasph_set_profiling(sph_ctx *ctx, int on);
int cudasph_phase_times(sph_ctx *ctx, double *ms /* SPH_NPHASES */, int *launches /* SPH_NPHASES */);
int cudasph_reset_counters(sph_ctx *ctx);
/* kernels launched by this context since the last reset */
long long cudasph_kernel_launches(const sph_ctx *ctx);

/* ---------------------------------------------------------------------- */
/* sharding over several GPUs (no counterpart in the reference, which runs */
/* one GPU).  Every rank holds a whole replica of the state; a context     */
/* given shard `rank` of `world` runs the leaf-parallel SPH loops (h solve */
/* + lists, density, hydro) over its contiguous range of tree leaves and   */
/* its contiguous share of the gravity blocks and work items.  The caller  */
/* steps it phase by phase (cudasph_step refuses a sharded context) and    */
/* sums three buffers over the ranks (e.g. an NCCL all-reduce on the       */
/* context's stream, cudasph_get_stream):                                  */
/*   sort, predict, build_tree, solve_range, density, shard_pack,          */
/*   SUM(SPH_BUF_EXCHANGE), shard_unpack, pressure, hydro,                 */
/*   SUM(SPH_BUF_DOTS), SUM(SPH_BUF_VSIG), gravity, SUM(SPH_BUF_GRAV),     */
/*   finish, kick.                                                         */
/* Each summed buffer holds a rank's own contributions and zeros elsewhere,*/
/* so the sums are exact and every rank continues with identical state.    */
/* The adjoint and CUDA-graph replay run on unsharded contexts only.       */
/* ---------------------------------------------------------------------- */
enum { SPH_BUF_EXCHANGE = 0, SPH_BUF_DOTS = 1, SPH_BUF_VSIG = 2, SPH_BUF_GRAV = 3 };
/* [lo, hi) of [0, count) owned by shard rank of world (host only) */
int cudasph_shard_range(long long count, int rank, int world, long long *lo, long long *hi);
int cudasph_set_shard(sph_ctx *ctx, int rank, int world);
/* rank, world and the context's leaves [leaf0, leaf1) (any pointer may be NULL) */
int cudasph_get_shard(sph_ctx *ctx, int *rank, int *world, int *leaf0, int *leaf1);
/* own h, rho, div, curl, omega, psi, n_ngb into the exchange buffer (zeros elsewhere) */
int cudasph_shard_pack(sph_ctx *ctx);
/* the summed exchange buffer back into the state of every particle */
int cudasph_shard_unpack(sph_ctx *ctx);
/* device address and length (doubles) of a buffer of the current state */
int cudasph_device_buffer(sph_ctx *ctx, int which, void **ptr, long long *doubles);
/* the context's CUDA stream (cudaStream_t) */
int cudasph_get_stream(sph_ctx *ctx, void **stream);

/* ---------------------------------------------------------------------- */
/* discrete adjoint of one step (no counterpart in the reference; the      */
/* differentiation form of the step).  With keep on, each step saves what  */
/* its reverse sweep needs; cudasph_adjoint then maps the adjoints of the  */
/* post-step state (x, v, u, a, du, dt) plus an optional adjoint of the    */
/* step's density (SPH_ADJ_RHO, consumed by the call) to the adjoints of   */
/* the pre-step state, in place.  The h solve is differentiated through    */
/* its implicit derivative; the forward neighbour lists are reused.        */
/* Plummer softening only.                                                 */
/* ---------------------------------------------------------------------- */
enum {
  SPH_ADJ_X = 0, SPH_ADJ_Y, SPH_ADJ_Z,
  SPH_ADJ_VX, SPH_ADJ_VY, SPH_ADJ_VZ, SPH_ADJ_U,
  SPH_ADJ_AX, SPH_ADJ_AY, SPH_ADJ_AZ, SPH_ADJ_DU,
  SPH_ADJ_RHO,
  SPH_NADJ
};
int cudasph_set_keep(sph_ctx *ctx, int on);
int cudasph_adjoint_set_field(sph_ctx *ctx, int field, const double *src, int on_device);
int cudasph_adjoint_get_field(sph_ctx *ctx, int field, double *dst, int on_device);
int cudasph_adjoint_set_dt(sph_ctx *ctx, double dtbar);
int cudasph_adjoint_get_dt(sph_ctx *ctx, double *dtbar);
int cudasph_adjoint(sph_ctx *ctx);

/* ---------------------------------------------------------------------- */
/* stand-alone operators on caller-owned device buffers                    */
/* ---------------------------------------------------------------------- */
/* Morton keys (21 bits per dimension in the bounding cube) and a stable
 * LSD radix sort of (key, value) pairs; `scratch` must hold
 * cudasph_sort_scratch_bytes(n) bytes.  Results land in keys/vals. */
size_t cudasph_sort_scratch_bytes(int n);
int cudasph_morton_keys(int n, const double *x, const double *y, const double *z, uint64_t *keys,
                        double *box4 /* device, 4 doubles: lo xyz, scale */, void *stream);
int cudasph_radix_sort_u64(int n, uint64_t *keys, uint32_t *vals, void *scratch, void *stream);

/* Peano-Hilbert keys of the reference's curve.  cudasph_peano_hilbert_keys is
 * peano_hilbert_key(x, y, z, bits) of sort_bodies.cpp:66-105 over n integer
 * triplets (device arrays; bits in [1, 21]; coordinate bits above bits-1 are
 * ignored).  cudasph_peano_keys keys positions the way CUDAsph::sort_bodies
 * does (sort_bodies.cpp:121-160): coordinates rounded to float, offset by the
 * float bounding box's low corner, scaled by domain_fac = float(2^18 / largest
 * extent) in float and truncated, 18 bits per dimension (a coordinate at the
 * box's far side becomes 2^18 and keeps its low 18 bits, as there); box4
 * receives {lo.x, lo.y, lo.z, domain_fac}.  A degenerate box (one point) gives
 * domain_fac = 0 and all keys 0. */
int cudasph_peano_hilbert_keys(int n, const int *x, const int *y, const int *z, int bits, uint64_t *keys,
                               void *stream);
int cudasph_peano_keys(int n, const double *x, const double *y, const double *z, uint64_t *keys,
                       double *box4 /* device, 4 doubles */, void *stream);

/* Allocation-free variant of cudasph_radix_sort_u64; it has no counterpart
 * in the reference.  It is for callers that cannot allocate device memory on
 * their own: a host application whose memory manager owns the whole GPU and
 * hands out no extra buffers, a loop that must not call cudaMalloc/cudaFree
 * because those calls can synchronise the device, or a run whose device
 * footprint is fixed at start-up.  The caller passes only the keys and values
 * (device pointers, results in place, same stable order as
 * cudasph_radix_sort_u64); the scratch is a fixed array compiled into this
 * library, sized for at most CUDASPH_SORT_NOALLOC_MAX_KEYS keys (about 3.1 MB,
 * held on every GPU that loads the library until the process exits).  Larger
 * n returns SPH_ERR_ARG with a message.  No cudaMalloc, cudaFree or other
 * allocating routine is called.  The first call on a device looks up the
 * array's device address on that device (cudaGetSymbolAddress), so make that
 * first call outside any stream capture; the first call after a
 * cudaDeviceReset of that device looks it up again (the array moves with the
 * reloaded library module), so make that one outside capture too.  Null
 * keys or vals with n > 1 return SPH_ERR_ARG with a message.  All calls share the one array and
 * nothing in it needs to start at zero, but calls whose GPU work overlaps
 * (two streams, or two host threads) race on it: serialise them. */
#define CUDASPH_SORT_NOALLOC_MAX_KEYS 262144
int cudasph_radix_sort_u64_noalloc(int n, uint64_t *keys, uint32_t *vals, void *stream);

/* The direct-N gravity work of shard `rank` of `world` for n particles at
 * `precision` / `soft_mode` (host only, no device): out8[0] = particles per
 * symmetric tile (0: the one-sided blocks cover every pair), [1] = particles
 * per one-sided block, [2..3] = the shard's one-sided blocks [lo, hi) (each
 * block's particles against the sources of their own tile, or against all
 * sources when the tile is 0), [4..5] = its symmetric work items [lo, hi),
 * [6] = tiles, [7] = tiles per item.  No counterpart in the reference (one
 * GPU, CUDA_gravity.cpp:3-71). */
int cudasph_gravity_plan(int n, int precision, int soft_mode, int rank, int world, long long *out8);
/* symmetric work item -> i-tile `row` and j-tiles [t_lo, t_hi) above it;
 * every pair of distinct tiles belongs to exactly one item (host only) */
int cudasph_gravity_item(int n, long long item, int *row, int *t_lo, int *t_hi);

/* direct-N gravity of n sources on themselves: pos4 = {x,y,z,m}, range =
 * smoothing ranges (spline mode), out4 = {gx,gy,gz,phi}; double buffers. */
int cudasph_gravity_direct(int n, const double *pos4, const double *range, double *out4, int soft_mode,
                           double eps, double G, int precision, void *stream);

/* FMA-pipe throughput probe (FLOP/s, 2 per FMA) on `stream`: precision 1 =
 * FP32, 0 = FP64.  The roofline denominator of the direct-N gravity loop. */
double cudasph_fma_peak(int precision, int iters, void *stream);

/* L2 read-bandwidth probe (bytes/s): a 48 MB buffer, resident in L2 after a
 * first pass, read `iters` times by every SM with 32-byte L2-only loads, on
 * `stream`.  The denominator of the neighbour loops' gather rates. */
double cudasph_l2_peak(int iters, void *stream);

/* ---------------------------------------------------------------------- */
/* the reference's extern "C" boundary (CUDAsph.h:22-48)                   */
/* ---------------------------------------------------------------------- */
#ifndef CUDASPH_B200_NO_LEGACY
#include "cudasph_b200_legacy.h"
#endif

#ifdef __cplusplus
}
#endif

#endif /* CUDASPH_B200_H_ */
