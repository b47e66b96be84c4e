// common.cuh -- shared device types and helpers of the sm_100a SPH step.
//
// Data layout in HBM (all arrays in tree order = Morton order after sorting):
//   pos   double4 {x, y, z, range}     range = 2h (the reference's bodies_pos)
//   vel   double4 {vx, vy, vz, m}      (bodies_vel)
//   hyd   double4 {rho, P, u, mu}      (hydro_data)
//   dd    double4 {divv, curlv, omega, psi}  (dots_data)
//   dots  double4 {ax, ay, az, du}     (bodies_dots, total after gravity)
//   grav  double4 {gx, gy, gz, phi}    (grav_data)
//   vsig  double                       (hydro_data2.x)
//   id    int     original particle index of each slot
// A gather of one neighbour reads whole 32-byte records (two 16-byte loads).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cudasph_b200.h"

namespace sph {

constexpr int kLeaf = 32;        // particles per tree leaf = one warp
constexpr int kFan = 32;         // children per internal node = one warp
constexpr int kMaxLevels = 8;    // supports up to 32^8 leaves
constexpr int kStack = 256;      // per-warp traversal stack (entries)

// Device-side view of the tree over Morton-ordered leaves.  Level 0 holds
// the leaves, level top the single root.  Each box is stored as two float4
// (lo.xyz, hi.xyz) rounded outward from the FP64 extrema, so that box tests
// are conservative and the exact FP64 predicate decides membership.
struct TreeView {
  int n;                       // particles
  int levels;                  // number of levels (top = levels - 1)
  int count[kMaxLevels];       // nodes per level
  long long base[kMaxLevels];  // offset of each level in lo/hi
  const float4 *lo;
  const float4 *hi;
};

// All per-particle state arrays (one buffer set).
struct Fields {
  double4 *pos, *vel, *hyd, *dd, *dots, *grav;
  double *vsig;
  int *id;
};

// arguments of the density / hydro kernels (both precision forms)
struct HydroArgs {
  int n, nleaf, cap;
  int leaf0, leaf1;  // leaves [leaf0, leaf1) processed by this launch (a shard's range, or all)
  const double4 *pos, *vel;
  double4 *hyd, *dd, *dots;
  double *vsig;
  const int *n_ngb, *list;
  double *ngb_acc;  // optional, list layout: m_i * acc per pair
  double4 *aux;     // per particle {c, P / rho^2, Balsara factor, 0}, written by launch_hydro
  double4 *dsum;    // optional (kept for the adjoint): the density loop's raw sums {S, Cx, Cy, Cz}
  double alpha, beta, gamma;
  int use_psi;
  int jside;  // 1: add the j-side pair force with atomics; 0: leave it to the caller
};

// arguments of the adjoint kernels (adjoint.cu)
struct AdjArgs {
  int n, nleaf, cap;
  // forward state of the step (slot order)
  const double4 *pos;     // x1, w
  const double4 *vel;     // (v1), m
  const double4 *hyd;     // rho, P, (u1), mu
  const double4 *dd;      // div, curl, omega, psi
  const double4 *dots;    // a1, du1
  const double *vsig;
  const double4 *old;     // v0, u0
  const double4 *pre_acc; // a0, du0
  const double4 *x0;      // x0 (pre-predict positions)
  double4 *vpup;          // vp, up (recomputed)
  const int *n_ngb, *list;
  const double *sc;       // forward scalars: [0] dt0  [1] dt1
  // adjoints
  double4 *xb;  // xbar (xyz), wbar (w)
  double4 *vb;  // vbar (xyz), ubar (w)
  double4 *ab;  // abar (xyz), dubar (w)
  double4 *vpb; // vpbar (xyz), upbar (w)
  double *rhob, *Pb, *omb, *psib, *divb, *curlb, *cb, *bb, *prb;
  double4 *aux;  // per particle {c, P / rho^2, Balsara factor, 0}, written before the hydro VJP
  const double4 *dsum;  // the forward density loop's raw sums {S, Cx, Cy, Cz}, or null (recomputed)
  const double *rho_ext;
  double *asc;  // [0] dtbar1 in  [1] dtbar0 out  [2] vsigbar  [3] istar  [4] fbar
  double *part;
  double alpha, beta, gamma, cn1, cn2;
  int eos_mode, use_psi;
};

struct StepScalars {
  // [0] dt_old  [1] dt_new  [2] time  [3..] statistics (SPH_NSTATS)
  double v[4 + SPH_NSTATS];
};

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ double4 ld4(const double4 *p) {
  // one 32-byte read-only load (sm_100's 256-bit vector load) of one
  // 32-byte-aligned record; against two 16-byte loads it halves the load
  // instructions of the list-driven gathers (N = 1M: hydro 1.89 -> 1.75 ms)
  double4 r;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
  return r;
}

// Exact neighbour predicate, evaluated without contraction so the tree walk
// reproduces (dx*dx + dy*dy) + dz*dz < range*range bit for bit
// (dev_find_ngb.cu:66-67 in FP64).
__device__ __forceinline__ double ds2_exact(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ void raise_flag(unsigned *flags, unsigned f) { atomicOr(flags, f); }

// Work items of the symmetric (each pair once) direct-N kernels: the Morton
// order is cut into nt tiles; tile row b owns the nt - 1 - b tiles above the
// diagonal, split into items of up to `chunk` tiles, rows in order.
// S(M) = sum_{m=1..M} ceil(m / chunk): items of the rows with 1..M tiles.
// The chunk is one of 8, 4, 2, 1, dispatched to constants so that every
// division is a shift (64-bit division by a runtime value is a long software
// routine, and the item map runs it in a binary search at every block start:
// 10 % of the 1M gravity kernel when it did).
template <int C>
__host__ __device__ __forceinline__ long long sym_S_c(long long M) {
  const long long q = M / C, r = M % C;
  return C * q * (q + 1) / 2 + (q + 1) * r;
}
__host__ __device__ __forceinline__ long long sym_S(long long M, int chunk) {
  switch (chunk) {
    case 8: return sym_S_c<8>(M);
    case 4: return sym_S_c<4>(M);
    case 2: return sym_S_c<2>(M);
    default: return sym_S_c<1>(M);
  }
}

// The chunk for nt tiles: the largest of 8, 4, 2, 1 that still gives every
// SM of the GPU four items (592 on 148 SMs), so small N fills the GPU and
// large N keeps long items.  A pure function of nt: every kernel, launch and
// shard computes the same one.
constexpr long long kSymMinItems = 4 * 148;
__host__ __device__ __forceinline__ int sym_chunk(int nt) {
  int c = 8;
  while (c > 1 && sym_S(nt - 1, c) < kSymMinItems) c >>= 1;
  return c;
}

// item -> (row b, j-tiles [t_lo, t_hi)), by binary search over the rows
template <int C>
__host__ __device__ __forceinline__ void sym_item_c(long long item, int nt, int &b, int &t_lo, int &t_hi) {
  const long long top = sym_S_c<C>(nt - 1);
  int lo = 0, hi = nt - 2;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (top - sym_S_c<C>(nt - 1 - mid) <= item) lo = mid; else hi = mid - 1;
  }
  b = lo;
  t_lo = b + 1 + (int)(item - (top - sym_S_c<C>(nt - 1 - b))) * C;
  t_hi = min(t_lo + C, nt);
}
__host__ __device__ __forceinline__ void sym_item(long long item, int nt, int &b, int &t_lo, int &t_hi) {
  switch (sym_chunk(nt)) {
    case 8: sym_item_c<8>(item, nt, b, t_lo, t_hi); break;
    case 4: sym_item_c<4>(item, nt, b, t_lo, t_hi); break;
    case 2: sym_item_c<2>(item, nt, b, t_lo, t_hi); break;
    default: sym_item_c<1>(item, nt, b, t_lo, t_hi); break;
  }
}

// number of work items for nt tiles
__host__ __device__ __forceinline__ long long sym_items(int nt) { return nt >= 2 ? sym_S(nt - 1, sym_chunk(nt)) : 0; }

// Contiguous balanced split of [0, count) over `world` shards: shard `rank`
// owns [count * rank / world, count * (rank + 1) / world).
__host__ __device__ __forceinline__ void shard_range(long long count, int rank, int world, long long &lo,
                                                     long long &hi) {
  lo = count * rank / world;
  hi = count * (rank + 1) / world;
}

}  // namespace sph

#define SPH_CUDA_TRY(expr)                                       \
  do {                                                           \
    cudaError_t err__ = (expr);                                  \
    if (err__ != cudaSuccess) return sph_internal_cuda_fail(err__, #expr, __FILE__, __LINE__); \
  } while (0)

int sph_internal_cuda_fail(cudaError_t err, const char *what, const char *file, int line);
void sph_internal_set_error(const char *msg);
