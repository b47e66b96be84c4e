/*
 * ref_cpu_harness.cpp -- builds the REFERENCE's own device code for the host CPU.
 *
 * TEST INFRASTRUCTURE.  This translation unit #includes the reference's
 * dev_*.cu / sph_grav_kernel.cu files from the reference tree (the include
 * path is given by oracle/Makefile) behind a small shim that turns CUDA
 * qualifiers into nothing and texture fetches into array reads.  The result,
 * oracle/_ref/libref_cpu.so, runs the reference's FP32 per-particle functions
 * (compute_ngb / solve_range / get_ngb / compute_density / get_pressure /
 * compute_dots / bodyBodyInteraction) unchanged on the CPU.  It is used
 *   (1) to pin the FP64 restatement in sph_oracle.c (tests/golden fixtures are
 *       generated from it by tests/golden/make_golden.py), and
 *   (2) as the timed "reference" CPU baseline of bench.py.
 * Nothing here is linked into the product library.
 *
 * The per-particle loops below only replace the CUDA launch grid
 * (blockIdx*blockDim+threadIdx) by an OpenMP loop over particles; the bodies
 * that run are the reference's.  The host-side j-scatter of
 * sph_accelerations.cpp:106-114 and the CSR offset scan of
 * sph_accelerations.cpp:58-72 live in member functions that cannot be linked
 * alone, so they are restated here (marked).
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <builtin_types.h>
#include <vector_functions.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- shim: CUDA qualifiers and texture references on the host ---- */
#undef __device__
#undef __global__
#undef __shared__
#undef __constant__
#define __device__
#define __global__
#define __shared__
#define __constant__

template <class T, int dim, enum cudaTextureReadMode mode>
struct texture {
  const T *ptr;
};
template <class T>
static inline T tex1Dfetch(const texture<T, 1, cudaReadModeElementType> &t, int i) {
  return t.ptr[i];
}
static inline int __float_as_int(float f) {
  int i;
  memcpy(&i, &f, sizeof(i));
  return i;
}
static inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
static inline float max(float a, float b) { return a > b ? a : b; }
static inline void __syncthreads() {}
static uint3 threadIdx, blockIdx;
static dim3 blockDim;
float4 shared_mem[1];

/* ---- the reference device code, in host_calls.cu:2-9 order ---- */
#include "radixsort/radixsort.cuh"
#include "dev_solve_range.cu"
#include "dev_find_ngb.cu"
#include "dev_density_loop.cu"
#include "dev_compute_pressure.cu"
#include "dev_hydro_dots.cu"
#include "sph_grav_kernel.cu"

/* reference host code linked from kd_tree.cpp / sort_bodies.cpp */
#include "kd_tree.h"
typedef long long peanokey;
peanokey peano_hilbert_key(int x, int y, int z, int bits);

extern "C" {

int ref_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* dev_sph_kernels.cu:7-99 */
void ref_kernel_eval(int which, int n, const float *u, float *out) {
  for (int i = 0; i < n; i++) {
    float v = u[i], r = 0;
    switch (which) {
      case 0: r = w(v); break;
      case 1: r = dw(v); break;
      case 2: r = dwdh(v); break;
      case 3: r = dphidh(v); break;
      case 4: r = iw(v); break;
      case 5: r = ig(v); break;
      case 6: r = dig(v); break;
      case 7: r = digdh(v); break;
      case 8: r = diw(v); break;
    }
    out[i] = r;
  }
}

/* dev_compute_pressure kernel body, dev_compute_pressure.cu:99-111 */
void ref_pressure(int n, const float *rho, const float *u, const float *mu, float *P) {
  for (int i = 0; i < n; i++) {
    float density = rho[i] * DENSITY_UNIT;
    float energy = u[i] * ENERGY_UNIT;
    float mean_mu = mu[i] * AMU;
    P[i] = get_pressure(density, energy, mean_mu);
  }
}

float ref_find_root(float q, float r) { return dev_find_root(q, r); }

/* peano_hilbert_key, sort_bodies.cpp:66-105 */
long long ref_peano_key(int x, int y, int z, int bits) { return peano_hilbert_key(x, y, z, bits); }

/* build_left_balanced_tree + packing of sph_accelerations.cpp:14-33.
 * nodes has n+1 float4 entries (index 0 unused); map gets build_kd_hash. */
void ref_build_kdtree(int n, const float4 *pos, float4 *nodes, int *map) {
  kd_node *kd = (kd_node *)malloc((n + 1) * sizeof(kd_node));
  build_left_balanced_tree(n, kd, (float4 *)pos);
  if (map) build_kd_hash(n, kd, map);
  for (int i = 1; i <= n; i++) {
    nodes[i].x = kd[i].pos[0];
    nodes[i].y = kd[i].pos[1];
    nodes[i].z = kd[i].pos[2];
    int data = (kd[i].body_id | (kd[i].split << (24)));
    memcpy(&nodes[i].w, &data, sizeof(int));
  }
  nodes[0] = make_float4(0, 0, 0, 0);
  free(kd);
}

/* dev_solve_range kernel (dev_solve_range.cu:174-189) over all particles;
 * CUDA_solve_range constants from CUDA_calls.cpp:3-10. */
void ref_solve_range(int n, float4 *pos, int *n_ngb, const float4 *nodes, float host_rel_err) {
  kd_tree_tex.ptr = nodes;
  n_nodes = n;
  rel_err = host_rel_err;
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; i++) {
    float4 bp = pos[i];
    float2 range = {0, 0};
    if (bp.w > 0) range = solve_range(bp);
    bp.w = range.x;
    pos[i] = bp;
    n_ngb[i] = (int)range.y;
  }
}

/* Restated: CSR offsets with lists padded to multiples of 4
 * (sph_accelerations.cpp:58-65).  offsets has n+1 entries; returns ngb_tot. */
int ref_ngb_offsets(int n, const int *n_ngb, int *offsets) {
  offsets[0] = 0;
  for (int i = 0; i < n; i++) {
    int k = n_ngb[i];
    int padded = ((k - 1) / 4) * 4 + 4;
    if (padded == 0) padded = 4;
    offsets[i + 1] = offsets[i] + padded;
  }
  return offsets[n];
}

/* get_ngb (dev_find_ngb.cu:13-73) for every particle; walk[i] = n_walk. */
void ref_find_ngb(int n, const float4 *pos, const float4 *nodes, const int *offsets, int *list, int *walk) {
  kd_tree_tex.ptr = nodes;
  n_nodes = n;
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; i++) {
    int nw = get_ngb(pos[i], &list[offsets[i]]);
    if (walk) walk[i] = nw;
  }
}

/* dev_density_loop kernel body (dev_density_loop.cu:88-111). */
void ref_density(int n, const float4 *pos, const float4 *vel, const int *n_ngb, const int *offsets,
                 const int *list, float4 *hydro, float4 *dots_data) {
  bodies_pos_tex.ptr = pos;
  bodies_vel_tex.ptr = vel;
  ngb_list_tex.ptr = list;
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; i++) {
    density_loop_data d = compute_density(n_ngb[i], offsets[i], pos[i], vel[i]);
    hydro[i].x = d.density;
    dots_data[i] = make_float4(d.div_v, d.curl_v, d.omega, d.Psi);
  }
}

/* dev_hydro_dots kernel body (dev_hydro_dots.cu:86-113) with the
 * CUDA_sph_accelerations constants alpha, beta (CUDA_calls.cpp:12-26). */
void ref_hydro(int n, const float4 *pos, const float4 *vel, const float4 *hydro, const float4 *dots_data,
               const int *n_ngb, const int *offsets, const int *list, float4 *bodies_dots, float *vsig,
               float *ngb_acc, float alpha, float beta) {
  bodies_pos_tex.ptr = pos;
  bodies_vel_tex.ptr = vel;
  hydro_data_tex.ptr = hydro;
  dots_data_tex.ptr = dots_data;
  ngb_list_tex.ptr = list;
  av_alpha = alpha;
  av_beta = beta;
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; i++) {
    dots_loop_data d = compute_dots(n_ngb[i], offsets[i], pos[i], vel[i], hydro[i], dots_data[i], ngb_acc);
    bodies_dots[i] = make_float4(d.vxdot, d.vydot, d.vzdot, d.u_dot);
    vsig[i] = d.v_sig;
  }
}

/* Restated: the host scatter of sph_accelerations.cpp:106-114. */
void ref_add_ngb_acc(int n, const float4 *pos, const int *n_ngb, const int *offsets, const int *list,
                     const float *ngb_acc, float4 *bodies_dots) {
  for (int i = 0; i < n; i++) {
    for (int k = offsets[i]; k < offsets[i] + n_ngb[i]; k++) {
      int j = list[k];
      float acc = ngb_acc[k];
      bodies_dots[j].x += acc * (pos[i].x - pos[j].x);
      bodies_dots[j].y += acc * (pos[i].y - pos[j].y);
      bodies_dots[j].z += acc * (pos[i].z - pos[j].z);
    }
  }
}

/* get_CUDA_forces (sph_grav_kernel.cu:179-195) for the targets tgt[0..nt)
 * (NULL: all n): the j loop calls bodyBodyInteraction on every source in
 * order, as the shared-memory tiles of computeBodyAccel do.  gpos = (x,y,z,m),
 * gvel = (vx,vy,vz,range^2) as packed by CUDA_gravity.cpp:41-47. */
void ref_gravity(int nt, const int *tgt, int n, const float4 *gpos, const float4 *gvel, float4 *acc_out) {
  int ntot = tgt ? nt : n;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < ntot; t++) {
    int i = tgt ? tgt[t] : t;
    acc3 acc;
    for (int c = 0; c < 4; c++) acc.v[c].v[0] = acc.v[c].v[1] = 0;
    float4 pi = gpos[i], vi = gvel[i];
    for (int j = 0; j < n; j++) acc = bodyBodyInteraction(acc, pi, vi, gpos[j], gvel[j]);
    acc_out[t] = make_float4(acc.v[0].v[0], acc.v[1].v[0], acc.v[2].v[0], acc.v[3].v[0]);
  }
}

}  // extern "C"
