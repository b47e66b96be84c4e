// legacy.cu -- the reference's extern "C" boundary (CUDAsph.h:22-48,
// host_calls.cu:27-376, radixsort/radixsort.cu:50-77) on top of the native
// context, so the reference's C++ driver runs on these kernels unchanged.
//
// The driver owns float4 AoS device arrays (bodies_pos {x,y,z,range},
// bodies_vel {vx,vy,vz,m}, hydro_data {rho,P,u,mu}, ...) and calls
// host_solve_range, then builds a CSR neighbour layout on the host from the
// returned counts, then calls host_sph_accelerations.  Both calls share one
// cached FP64 context sized to the number of real bodies (n_nodes); the
// float4 inputs are widened into it on the device and the results narrowed
// back into the driver's arrays and CSR lists.  Failures print a message and
// exit(1), the behaviour of CUDA_SAFE_CALL (host_calls.cu:14-22).
#include <cstdio>
#include <cstdlib>

#include "common.cuh"

namespace sph {
cudaStream_t ctx_stream(sph_ctx *c);
Fields &ctx_fields(sph_ctx *c);
int *ctx_n_ngb(sph_ctx *c);
int *ctx_list(sph_ctx *c, int *cap);
const TreeView &ctx_tree(sph_ctx *c);
void ctx_mark_positions(sph_ctx *c);
int *ctx_slot_of(sph_ctx *c);
HydroArgs ctx_hydro_args(sph_ctx *c);
int launch_density(const HydroArgs &a, cudaStream_t st);
int launch_hydro(const HydroArgs &a, cudaStream_t st);
int launch_invert(int n, const int *id, int *slot_of, cudaStream_t st);
int launch_gravity(int n, const double4 *src, const double *h2src, double4 *out, int soft_mode, double eps, double G,
                   int precision, const int *mass_mixed, int rank, int world, cudaStream_t st);
size_t radix_scratch_bytes(int n);
int radix_sort_u64(int n, uint64_t *keys, uint32_t *vals, void *scratch, cudaStream_t st);
}  // namespace sph

using namespace sph;

namespace {

void die(const char *what, const char *detail) {
  fprintf(stderr, "\nerror: %s failed with error %s\n", what, detail ? detail : "");
  exit(1);
}

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) die(what, cudaGetErrorName(e));
}

void check_rc(int rc, const char *what) {
  if (rc != SPH_OK) die(what, cudasph_last_error());
}

sph_ctx *g_ctx = nullptr;
int g_n = 0;
double *g_acc = nullptr;  // ngb_acc in list layout (FP64)
size_t g_acc_cap = 0;
double4 *g_grav_src = nullptr, *g_grav_out = nullptr;  // compute_CUDA_gravity's sources and results
double *g_grav_h2 = nullptr;
size_t g_grav_cap = 0;

sph_ctx *legacy_ctx(int n_real) {
  if (g_ctx && g_n == n_real) return g_ctx;
  if (g_ctx) cudasph_destroy(g_ctx);
  sph_params p = cudasph_default_params();  // the reference's constants
  p.use_psi = 1;
  int dev = 0;
  cudaGetDevice(&dev);
  check_rc(cudasph_create(&p, n_real, dev, &g_ctx), "cudasph_create");
  g_n = n_real;
  return g_ctx;
}

__global__ void k_legacy_in(int n, const float4 *__restrict__ pos, const float4 *__restrict__ vel,
                            const int *__restrict__ id, Fields F) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int i = id[s];
  const float4 p = pos[i], v = vel[i];
  F.pos[s] = make_double4(p.x, p.y, p.z, p.w);
  F.vel[s] = make_double4(v.x, v.y, v.z, v.w);
}

__global__ void k_legacy_solve_out(int n, const int *__restrict__ id, Fields F, const int *__restrict__ cnt,
                                   float4 *__restrict__ pos, int *__restrict__ n_ngb) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int i = id[s];
  pos[i].w = (float)F.pos[s].w;
  n_ngb[i] = cnt[s];
}

__global__ void k_legacy_hydro_in(int n, const float4 *__restrict__ hydro, const int *__restrict__ id, Fields F) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float4 h = hydro[id[s]];
  F.hyd[s].z = h.z;
  F.hyd[s].w = h.w;
}

__global__ void k_legacy_sph_out(int n, const int *__restrict__ id, Fields F, const int *__restrict__ cnt,
                                 const int *__restrict__ list, const double *__restrict__ acc, int cap,
                                 const int *__restrict__ offset, int *__restrict__ list_out,
                                 float *__restrict__ acc_out, float4 *__restrict__ hydro, float4 *__restrict__ dd,
                                 float4 *__restrict__ dots, float4 *__restrict__ hydro2) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int i = id[s];
  const double4 h = F.hyd[s], d = F.dd[s], a = F.dots[s];
  hydro[i].x = (float)h.x;
  hydro[i].y = (float)h.y;
  dd[i] = make_float4((float)d.x, (float)d.y, (float)d.z, (float)d.w);
  dots[i] = make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w);
  hydro2[i].x = (float)F.vsig[s];
  const int leaf = s / kLeaf, lane = s % kLeaf;
  const int m = min(cnt[s], cap);
  const int o = offset[i];
  for (int k = 0; k < m; k++) {
    const size_t e = ((size_t)leaf * cap + k) * kLeaf + lane;
    list_out[o + k] = id[list[e]];
    acc_out[o + k] = (float)acc[e];
  }
}

__global__ void k_legacy_hash_key(int n_pad, int n, sph_legacy_kv *__restrict__ hash, const int *__restrict__ slot_of,
                                  const int *__restrict__ cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_pad) return;
  const unsigned i = hash[t].value;
  hash[t].key = (i < (unsigned)n) ? (unsigned)cnt[slot_of[i]] : 0u;
}

__global__ void k_grav_in(int n, const float4 *__restrict__ pos, const float4 *__restrict__ vel, double4 *src,
                          double *h2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = pos[i], v = vel[i];
  src[i] = make_double4(p.x, p.y, p.z, p.w);
  h2[i] = v.w;
}

__global__ void k_grav_out(int n, const double4 *__restrict__ g, float4 *__restrict__ acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 a = g[i];
  acc[i] = make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w);
}

__global__ void k_kv_split(int n, const sph_legacy_kv *__restrict__ d, uint64_t *keys, uint32_t *vals,
                           unsigned mask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = d[i].key & mask;
  vals[i] = (uint32_t)i;
}

__global__ void k_kv_gather(int n, const sph_legacy_kv *__restrict__ src, const uint32_t *__restrict__ order,
                            sph_legacy_kv *__restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[order[i]];
}

double now_seconds() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

}  // namespace

extern "C" {

void initCUDA(void) {}

int cuda_get_device(void) {
  int d = 0;
  check(cudaGetDevice(&d), "cudaGetDevice(&device)");
  return d;
}

void cuda_set_device0(int device_id) {
  if (device_id > 0) check(cudaSetDevice(device_id - 1), "cudaSetDevice(device_id - 1)");
}

void cuda_set_device(int) {}

int get_device_count(void) {
  int n = 0;
  check(cudaGetDeviceCount(&n), "cudaGetDeviceCount(&s_gpuCount)");
  return n;
}

void allocateCUDAarray(void **pos, int n, int) { check(cudaMalloc(pos, (size_t)n), "cudaMalloc((void**)pos, n)"); }
void deleteCUDAarray(void *pos, int) { check(cudaFree(pos), "cudaFree((void*)pos)"); }
void copyArrayToDevice(void *device, const void *host, int n, int) {
  check(cudaMemcpy(device, host, (size_t)n, cudaMemcpyHostToDevice), "cudaMemcpy(device, host, n)");
}
void copyArrayFromDevice(void *host, const void *device, int n, int) {
  check(cudaMemcpy(host, device, (size_t)n, cudaMemcpyDeviceToHost), "cudaMemcpy(host, device, n)");
}

void allocateNBodyArrays(float **pos, int numBodies, int) {
  check(cudaMalloc((void **)pos, sizeof(float) * 4 * (size_t)numBodies), "cudaMalloc((void**)pos, memSize)");
}
void deleteNBodyArrays(float *pos, int) { check(cudaFree(pos), "cudaFree((void*)pos)"); }
void zallocateNBodyArrays(float **pos, int numBodies, int d) { allocateNBodyArrays(pos, numBodies, d); }
void zdeleteNBodyArrays(float *pos, int d) { deleteNBodyArrays(pos, d); }
void zcopyArrayFromDevice(float *host, const float *device, unsigned int numBodies, int) {
  check(cudaMemcpy(host, device, (size_t)numBodies * 4 * sizeof(float), cudaMemcpyDeviceToHost),
        "cudaMemcpy(host, device, numBodies*4*sizeof(float))");
}
void zcopyArrayToDevice(float *device, const float *host, int numBodies, int) {
  check(cudaMemcpy(device, host, (size_t)numBodies * 4 * sizeof(float), cudaMemcpyHostToDevice),
        "cudaMemcpy(device, host, numBodies*4*sizeof(float))");
}

void compute_CUDA_gravity(int numBodies, sph_legacy_float4 *accel, float *pos, float *vel, int, int, int) {
  if (numBodies <= 0) return;
  // FP64 sources and results live in buffers kept across calls (grown when a
  // call has more bodies), so a driver step allocates nothing here
  if ((size_t)numBodies > g_grav_cap) {
    cudaFree(g_grav_src);
    cudaFree(g_grav_out);
    cudaFree(g_grav_h2);
    g_grav_src = g_grav_out = nullptr;
    g_grav_h2 = nullptr;
    check(cudaMalloc((void **)&g_grav_src, sizeof(double4) * numBodies), "cudaMalloc");
    check(cudaMalloc((void **)&g_grav_out, sizeof(double4) * numBodies), "cudaMalloc");
    check(cudaMalloc((void **)&g_grav_h2, sizeof(double) * numBodies), "cudaMalloc");
    g_grav_cap = (size_t)numBodies;
  }
  const int nb = (numBodies + 255) / 256;
  k_grav_in<<<nb, 256>>>(numBodies, (const float4 *)pos, (const float4 *)vel, g_grav_src, g_grav_h2);
  launch_gravity(numBodies, g_grav_src, g_grav_h2, g_grav_out, SPH_SOFT_SPLINE, 0.0, 1.0, SPH_PREC_FP64, nullptr, 0,
                 1, 0);
  k_grav_out<<<nb, 256>>>(numBodies, g_grav_out, (float4 *)accel);
  check(cudaDeviceSynchronize(), "get_CUDA_forces");
}

float host_solve_range(int n_bodies, int n_nodes, float rel_err, sph_legacy_kv *bodies_hash, int *bodies_map,
                       sph_legacy_float4 *bodies_pos, sph_legacy_float4 *bodies_vel, sph_legacy_float4 *kd_tree,
                       int *n_ngb, int device_id) {
  (void)bodies_hash; (void)bodies_map; (void)kd_tree; (void)device_id;
  const double t0 = now_seconds();
  const int n = n_nodes;
  if (n <= 0) return 0.f;
  sph_ctx *c = legacy_ctx(n);
  sph_params p;
  cudasph_get_params(c, &p);
  p.rel_err = rel_err;
  check_rc(cudasph_set_params(c, &p), "cudasph_set_params");
  cudaStream_t st = ctx_stream(c);
  Fields &F = ctx_fields(c);
  k_legacy_in<<<(n + 255) / 256, 256, 0, st>>>(n, (const float4 *)bodies_pos, (const float4 *)bodies_vel, F.id, F);
  ctx_mark_positions(c);
  check_rc(cudasph_solve_range(c), "dev_solve_range");
  check_rc(cudasph_find_ngb(c), "dev_find_ngb");
  Fields &G = ctx_fields(c);
  k_legacy_solve_out<<<(n + 255) / 256, 256, 0, st>>>(n, G.id, G, ctx_n_ngb(c), (float4 *)bodies_pos, n_ngb);
  // pads (n_nodes .. n_bodies) keep range 0 and get no neighbours
  if (n_bodies > n) {
    check(cudaMemsetAsync(n_ngb + n, 0, sizeof(int) * (size_t)(n_bodies - n), st), "cudaMemset(n_ngb)");
  }
  check(cudaStreamSynchronize(st), "host_solve_range");
  return (float)(now_seconds() - t0);
}

float host_sph_accelerations(int n_bodies, int ngb_tot, float av_alpha, float av_beta, sph_legacy_kv *bodies_hash,
                             sph_legacy_kv *bodies_hash_extra, int *bodies_map, int *ngb_list, int *ngb_offset,
                             sph_legacy_float4 *hydro_data, sph_legacy_float4 *dots_data,
                             sph_legacy_float4 *bodies_dots, sph_legacy_float4 *hydro_data2, float *ngb_acc,
                             int device_id) {
  (void)ngb_tot; (void)bodies_hash_extra; (void)bodies_map; (void)device_id;
  const double t0 = now_seconds();
  if (!g_ctx) die("host_sph_accelerations", "host_solve_range was not called first");
  sph_ctx *c = g_ctx;
  const int n = g_n;
  sph_params p;
  cudasph_get_params(c, &p);
  p.av_alpha = av_alpha;
  p.av_beta = av_beta;
  check_rc(cudasph_set_params(c, &p), "cudasph_set_params");
  cudaStream_t st = ctx_stream(c);
  Fields &F = ctx_fields(c);
  k_legacy_hydro_in<<<(n + 255) / 256, 256, 0, st>>>(n, (const float4 *)hydro_data, F.id, F);
  int cap = 0;
  int *list = ctx_list(c, &cap);
  const size_t entries = (size_t)ctx_tree(c).count[0] * kLeaf * cap;
  if (entries > g_acc_cap) {
    if (g_acc) cudaFree(g_acc);
    check(cudaMalloc((void **)&g_acc, sizeof(double) * entries), "cudaMalloc(ngb_acc)");
    g_acc_cap = entries;
  }
  check_rc(cudasph_density(c), "dev_density_loop");
  check_rc(cudasph_pressure(c), "dev_compute_pressure");
  check(cudaMemsetAsync(F.dots, 0, sizeof(double4) * n, st), "cudaMemset(bodies_dots)");
  HydroArgs a = ctx_hydro_args(c);
  a.ngb_acc = g_acc;
  a.jside = 0;  // the driver scatters the j-side itself (sph_accelerations.cpp:106-114)
  launch_hydro(a, st);
  k_legacy_sph_out<<<(n + 255) / 256, 256, 0, st>>>(n, F.id, F, ctx_n_ngb(c), list, g_acc, cap, ngb_offset, ngb_list,
                                                    ngb_acc, (float4 *)hydro_data, (float4 *)dots_data,
                                                    (float4 *)bodies_dots, (float4 *)hydro_data2);
  launch_invert(n, F.id, ctx_slot_of(c), st);
  k_legacy_hash_key<<<(n_bodies + 255) / 256, 256, 0, st>>>(n_bodies, n, bodies_hash, ctx_slot_of(c), ctx_n_ngb(c));
  check(cudaStreamSynchronize(st), "host_sph_accelerations");
  return (float)(now_seconds() - t0);
}

void RadixSort(sph_legacy_kv *pData0, sph_legacy_kv *pData1, unsigned int elements, unsigned int bits) {
  if (elements <= 1) return;
  const int n = (int)elements;
  const unsigned mask = bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
  uint64_t *keys = nullptr;
  uint32_t *vals = nullptr;
  void *scratch = nullptr;
  check(cudaMalloc((void **)&keys, sizeof(uint64_t) * n), "cudaMalloc");
  check(cudaMalloc((void **)&vals, sizeof(uint32_t) * n), "cudaMalloc");
  check(cudaMalloc(&scratch, radix_scratch_bytes(n)), "cudaMalloc");
  k_kv_split<<<(n + 255) / 256, 256>>>(n, pData0, keys, vals, mask);
  radix_sort_u64(n, keys, vals, scratch, 0);
  k_kv_gather<<<(n + 255) / 256, 256>>>(n, pData0, vals, pData1);
  check(cudaMemcpy(pData0, pData1, sizeof(sph_legacy_kv) * n, cudaMemcpyDeviceToDevice), "RadixSort");
  cudaFree(keys);
  cudaFree(vals);
  cudaFree(scratch);
}

}  // extern "C"
