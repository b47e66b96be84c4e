// integrate.cu -- the device-resident host loops of the reference step:
// predictor (step.cpp:38-61), gravity add + total force / torque
// (step.cpp:96-117), system_statistics (system_statistics.cpp:4-84),
// compute_timestep (compute_timestep.cpp:3-25), the kick (step.cpp:128-134)
// and the permutation that applies the Morton sort to the state.
//
// Reductions are deterministic: a fixed shuffle tree inside each block,
// block partials written to memory, and one block that folds the partials
// in block order.  dt, time and the statistics stay on the device
// (StepScalars), so a step needs no host round trip.
#include "common.cuh"

namespace sph {

// scalars: v[0] = dt of the drift just taken, v[1] = current dt, v[2] = time
constexpr int kS_DTOLD = 0, kS_DT = 1, kS_TIME = 2, kS_STATS = 4;

__global__ void k_predict(int n, double4 *__restrict__ pos, double4 *__restrict__ vel, double4 *__restrict__ hyd,
                          const double4 *__restrict__ dots, double4 *__restrict__ old,
                          const double *__restrict__ sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double dt = sc[kS_DT], dth = 0.5 * dt;
  double4 p = pos[i], v = vel[i], h = hyd[i];
  const double4 d = dots[i];
  p.x += v.x * dt;
  p.y += v.y * dt;
  p.z += v.z * dt;
  old[i] = make_double4(v.x, v.y, v.z, h.z);
  v.x += d.x * dth;
  v.y += d.y * dth;
  v.z += d.z * dth;
  h.z += d.w * dth;
  pos[i] = p;
  vel[i] = v;
  hyd[i] = h;
}

// statistics accumulated per block (sums) and extrema
enum {
  kQ_M = 0, kQ_CX, kQ_CY, kQ_CZ, kQ_VX, kQ_VY, kQ_VZ, kQ_JX, kQ_JY, kQ_JZ, kQ_U, kQ_W, kQ_T,
  kQ_FX, kQ_FY, kQ_FZ, kQ_TX, kQ_TY, kQ_TZ, kQ_NGB, kQ_NGB2,
  kQ_NSUM,
  kQ_NGBMIN = kQ_NSUM, kQ_NGBMAX, kQ_DTV, kQ_DTE, kQ_DT,
  kQ_N
};
constexpr int kFinThreads = 256;

__global__ void __launch_bounds__(kFinThreads) k_finish_partial(int n, const double4 *__restrict__ pos,
                                                                const double4 *__restrict__ vel,
                                                                const double4 *__restrict__ hyd,
                                                                double4 *__restrict__ dots,
                                                                const double4 *__restrict__ grav,
                                                                const double *__restrict__ vsig,
                                                                const int *__restrict__ n_ngb, int add_gravity,
                                                                double cn1, double cn2, double *__restrict__ part) {
  double q[kQ_N];
#pragma unroll
  for (int k = 0; k < kQ_NSUM; k++) q[k] = 0;
  q[kQ_NGBMIN] = 1e300;
  q[kQ_NGBMAX] = -1e300;
  q[kQ_DTV] = q[kQ_DTE] = q[kQ_DT] = 1.0e30;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double4 p = pos[i], v = vel[i], h = hyd[i];
    double4 a = dots[i];
    const double4 g = grav[i];
    if (add_gravity) {
      a.x += g.x;
      a.y += g.y;
      a.z += g.z;
      dots[i] = a;
    }
    const double m = v.w;
    q[kQ_M] += m;
    q[kQ_CX] += m * p.x; q[kQ_CY] += m * p.y; q[kQ_CZ] += m * p.z;
    q[kQ_VX] += m * v.x; q[kQ_VY] += m * v.y; q[kQ_VZ] += m * v.z;
    q[kQ_JX] += m * (p.y * v.z - p.z * v.y);
    q[kQ_JY] += m * (p.z * v.x - p.x * v.z);
    q[kQ_JZ] += m * (p.x * v.y - p.y * v.x);
    q[kQ_U] += m * h.z;
    q[kQ_W] += 0.5 * m * g.w;
    q[kQ_T] += 0.5 * m * (v.x * v.x + v.y * v.y + v.z * v.z);
    q[kQ_FX] += m * a.x; q[kQ_FY] += m * a.y; q[kQ_FZ] += m * a.z;
    q[kQ_TX] += m * (p.y * a.z - p.z * a.y);
    q[kQ_TY] += m * (p.z * a.x - p.x * a.z);
    q[kQ_TZ] += m * (p.x * a.y - p.y * a.x);
    const double nn = n_ngb ? (double)n_ngb[i] : 0.0;
    q[kQ_NGB] += nn;
    q[kQ_NGB2] += nn * nn;
    q[kQ_NGBMIN] = fmin(q[kQ_NGBMIN], nn);
    q[kQ_NGBMAX] = fmax(q[kQ_NGBMAX], nn);
    // compute_timestep.cpp:10-16
    const double dtv = cn1 * fabs(p.w / vsig[i]);
    const double dte = cn2 * fabs(h.z / a.w);
    q[kQ_DTV] = fmin(q[kQ_DTV], dtv);
    q[kQ_DTE] = fmin(q[kQ_DTE], dte);
    q[kQ_DT] = fmin(q[kQ_DT], 1.0 / (1.0 / dtv + 1.0 / dte));
  }
  // fixed-order block reduction
#pragma unroll
  for (int k = 0; k < kQ_N; k++) {
    double x = q[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, x, o);
      if (k < kQ_NSUM) x += y;
      else if (k == kQ_NGBMAX) x = fmax(x, y);
      else x = fmin(x, y);
    }
    q[k] = x;
  }
  __shared__ double s[kFinThreads / 32][kQ_N];
  const int w = threadIdx.x >> 5;
  if (lane_id() == 0)
#pragma unroll
    for (int k = 0; k < kQ_N; k++) s[w][k] = q[k];
  __syncthreads();
  if (threadIdx.x < kQ_N) {
    const int k = threadIdx.x;
    double x = s[0][k];
    for (int ww = 1; ww < kFinThreads / 32; ww++) {
      const double y = s[ww][k];
      if (k < kQ_NSUM) x += y;
      else if (k == kQ_NGBMAX) x = fmax(x, y);
      else x = fmin(x, y);
    }
    part[blockIdx.x * kQ_N + k] = x;
  }
}

__global__ void k_finish_final(int n, int nb, const double *__restrict__ part, double *__restrict__ sc,
                               unsigned *flags) {
  __shared__ double q[kQ_N];
  const int k = threadIdx.x;
  if (k < kQ_N) {
    double x = part[k];
    for (int b = 1; b < nb; b++) {
      const double y = part[b * kQ_N + k];
      if (k < kQ_NSUM) x += y;
      else if (k == kQ_NGBMAX) x = fmax(x, y);
      else x = fmin(x, y);
    }
    q[k] = x;
  }
  __syncthreads();
  if (k != 0) return;
  double *st = sc + kS_STATS;
  const double M = q[kQ_M];
  const double dt_old = sc[kS_DT];
  const double time = sc[kS_TIME] + dt_old;  // global_time += dt (step.cpp:121)
  st[SPH_ST_W] = q[kQ_W];
  st[SPH_ST_T] = q[kQ_T];
  st[SPH_ST_U] = q[kQ_U];
  st[SPH_ST_E] = q[kQ_T] + q[kQ_U] + q[kQ_W];
  st[SPH_ST_JX] = q[kQ_JX]; st[SPH_ST_JY] = q[kQ_JY]; st[SPH_ST_JZ] = q[kQ_JZ];
  st[SPH_ST_RCMX] = M > 0 ? q[kQ_CX] / M : 0; st[SPH_ST_RCMY] = M > 0 ? q[kQ_CY] / M : 0;
  st[SPH_ST_RCMZ] = M > 0 ? q[kQ_CZ] / M : 0;
  st[SPH_ST_VCMX] = M > 0 ? q[kQ_VX] / M : 0; st[SPH_ST_VCMY] = M > 0 ? q[kQ_VY] / M : 0;
  st[SPH_ST_VCMZ] = M > 0 ? q[kQ_VZ] / M : 0;
  st[SPH_ST_MTOT] = M;
  st[SPH_ST_FX] = q[kQ_FX]; st[SPH_ST_FY] = q[kQ_FY]; st[SPH_ST_FZ] = q[kQ_FZ];
  st[SPH_ST_TX] = q[kQ_TX]; st[SPH_ST_TY] = q[kQ_TY]; st[SPH_ST_TZ] = q[kQ_TZ];
  const double mean = n > 0 ? q[kQ_NGB] / n : 0;
  const double var = n > 0 ? q[kQ_NGB2] / n - mean * mean : 0;
  st[SPH_ST_NGB_MEAN] = mean;
  st[SPH_ST_NGB_SIGMA] = sqrt(fmax(var, 0.0));
  st[SPH_ST_NGB_MIN] = q[kQ_NGBMIN];
  st[SPH_ST_NGB_MAX] = q[kQ_NGBMAX];
  st[SPH_ST_DT_VEL] = q[kQ_DTV];
  st[SPH_ST_DT_ETH] = q[kQ_DTE];
  st[SPH_ST_DT] = q[kQ_DT];
  st[SPH_ST_TIME] = time;
  st[SPH_ST_DT_OLD] = dt_old;
  if (!isfinite(q[kQ_DT])) raise_flag(flags, SPH_FLAG_NONFINITE);
  sc[kS_DTOLD] = dt_old;
  sc[kS_DT] = q[kQ_DT];
  sc[kS_TIME] = time;
}

// step.cpp:128-134: v = v_old + a (dt_new/2 + dt_old/2), u likewise
__global__ void k_kick(int n, double4 *__restrict__ vel, double4 *__restrict__ hyd, const double4 *__restrict__ dots,
                       const double4 *__restrict__ old, const double *__restrict__ sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double f = 0.5 * sc[kS_DT] + 0.5 * sc[kS_DTOLD];
  const double4 a = dots[i], o = old[i];
  double4 v = vel[i];
  v.x = o.x + a.x * f;
  v.y = o.y + a.y * f;
  v.z = o.z + a.z * f;
  vel[i] = v;
  hyd[i].z = o.w + a.w * f;
}

// apply a permutation: dst[s] = src[order[s]] for every state array
__global__ void k_permute(int n, const uint32_t *__restrict__ order, Fields src, Fields dst) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = (int)order[s];
  dst.pos[s] = src.pos[o];
  dst.vel[s] = src.vel[o];
  dst.hyd[s] = src.hyd[o];
  dst.dd[s] = src.dd[o];
  dst.dots[s] = src.dots[o];
  dst.grav[s] = src.grav[o];
  dst.vsig[s] = src.vsig[o];
  dst.id[s] = src.id[o];
}

// slot_of[id[s]] = s
__global__ void k_invert(int n, const int *__restrict__ id, int *__restrict__ slot_of) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) slot_of[id[s]] = s;
}

int launch_predict(int n, double4 *pos, double4 *vel, double4 *hyd, const double4 *dots, double4 *old,
                   const double *sc, cudaStream_t st) {
  k_predict<<<(n + 255) / 256, 256, 0, st>>>(n, pos, vel, hyd, dots, old, sc);
  return 1;
}

int finish_partial_blocks(int n) {
  int nb = (n + kFinThreads - 1) / kFinThreads;
  if (nb > 148 * 4) nb = 148 * 4;
  if (nb < 1) nb = 1;
  return nb;
}
int finish_partial_doubles(int n) { return finish_partial_blocks(n) * kQ_N; }

int launch_finish(int n, const double4 *pos, const double4 *vel, const double4 *hyd, double4 *dots,
                  const double4 *grav, const double *vsig, const int *n_ngb, int add_gravity, double cn1, double cn2,
                  double *part, double *sc, unsigned *flags, cudaStream_t st) {
  const int nb = finish_partial_blocks(n);
  k_finish_partial<<<nb, kFinThreads, 0, st>>>(n, pos, vel, hyd, dots, grav, vsig, n_ngb, add_gravity, cn1, cn2, part);
  k_finish_final<<<1, 32, 0, st>>>(n, nb, part, sc, flags);
  return 2;
}

int launch_kick(int n, double4 *vel, double4 *hyd, const double4 *dots, const double4 *old, const double *sc,
                cudaStream_t st) {
  k_kick<<<(n + 255) / 256, 256, 0, st>>>(n, vel, hyd, dots, old, sc);
  return 1;
}

// Exchange of the SPH results between shards.  Every particle has two
// double4 records in xbuf: {range, rho, div, curl} and {omega, psi, n_ngb, 0}.
// pack: the shard's own slots [s0, s1) are copied in, every other slot is
// zeroed, so the element-wise sum of the shards' buffers holds every
// particle's values exactly once; unpack writes the summed buffer back.
__global__ void k_shard_pack(int n, int s0, int s1, const double4 *__restrict__ pos, const double4 *__restrict__ hyd,
                             const double4 *__restrict__ dd, const int *__restrict__ n_ngb,
                             double4 *__restrict__ xbuf) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  double4 a = make_double4(0, 0, 0, 0), b = make_double4(0, 0, 0, 0);
  if (s >= s0 && s < s1) {
    const double4 d = dd[s];
    a = make_double4(pos[s].w, hyd[s].x, d.x, d.y);
    b = make_double4(d.z, d.w, (double)n_ngb[s], 0.0);
  }
  xbuf[2 * s] = a;
  xbuf[2 * s + 1] = b;
}

__global__ void k_shard_unpack(int n, const double4 *__restrict__ xbuf, double4 *__restrict__ pos,
                               double4 *__restrict__ hyd, double4 *__restrict__ dd, int *__restrict__ n_ngb) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const double4 a = xbuf[2 * s], b = xbuf[2 * s + 1];
  pos[s].w = a.x;
  hyd[s].x = a.y;
  dd[s] = make_double4(a.z, a.w, b.x, b.y);
  n_ngb[s] = (int)b.z;
}

int launch_shard_pack(int n, int s0, int s1, const double4 *pos, const double4 *hyd, const double4 *dd,
                      const int *n_ngb, double4 *xbuf, cudaStream_t st) {
  k_shard_pack<<<(n + 255) / 256, 256, 0, st>>>(n, s0, s1, pos, hyd, dd, n_ngb, xbuf);
  return 1;
}

int launch_shard_unpack(int n, const double4 *xbuf, double4 *pos, double4 *hyd, double4 *dd, int *n_ngb,
                        cudaStream_t st) {
  k_shard_unpack<<<(n + 255) / 256, 256, 0, st>>>(n, xbuf, pos, hyd, dd, n_ngb);
  return 1;
}

int launch_permute(int n, const uint32_t *order, const Fields &src, const Fields &dst, cudaStream_t st) {
  k_permute<<<(n + 255) / 256, 256, 0, st>>>(n, order, src, dst);
  return 1;
}

int launch_invert(int n, const int *id, int *slot_of, cudaStream_t st) {
  k_invert<<<(n + 255) / 256, 256, 0, st>>>(n, id, slot_of);
  return 1;
}

// field exchange between the caller's original order and tree order:
// to_state: arr[s*stride + comp] = flat[id[s]]; else flat[id[s]] = arr[...].
// stride < 0 selects an int array copied out as ints.
__global__ void k_field_io(int n, double *__restrict__ arr, int stride, int comp, const int *__restrict__ id,
                           double *__restrict__ flat, int to_state) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = id[s];
  if (stride < 0) {
    reinterpret_cast<int *>(flat)[o] = reinterpret_cast<const int *>(arr)[s];
    return;
  }
  if (to_state) arr[(size_t)s * stride + comp] = flat[o];
  else flat[o] = arr[(size_t)s * stride + comp];
}

__global__ void k_iota(int n, int *__restrict__ id) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) id[s] = s;
}

int launch_field_io(int n, double *arr, int stride, int comp, const int *id, double *flat, int to_state,
                    cudaStream_t st) {
  k_field_io<<<(n + 255) / 256, 256, 0, st>>>(n, arr, stride, comp, id, flat, to_state);
  return 1;
}

int launch_iota(int n, int *id, cudaStream_t st) {
  k_iota<<<(n + 255) / 256, 256, 0, st>>>(n, id);
  return 1;
}

}  // namespace sph
