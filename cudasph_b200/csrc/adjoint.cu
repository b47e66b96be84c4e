// adjoint.cu -- hand-written discrete adjoint of one step.
//
// Forward step (step.cpp:13-147, as run by capi.cu):
//   x1 = x0 + v0 dt0;  vp = v0 + a0 dt0/2;  up = u0 + du0 dt0/2
//   w  = root of F_i(w) = sum_j ig(2 r_ij / w_i) - N      (h solve)
//   rho, div, curl, omega, psi = DENSITY(x1, vp, w)
//   P  = EOS(rho, up)
//   ah, du1, vsig = HYDRO(x1, vp, w, rho, P, div, curl, omega, psi)
//   a1 = ah + GRAVITY(x1)                                  (Plummer)
//   dt1 = min_i tau_i(w, vsig, up, du1)                    (compute_timestep)
//   v1 = v0 + a1 (dt1/2 + dt0/2);  u1 = u0 + du1 (dt1/2 + dt0/2)
//
// Given adjoints of (x1, v1, u1, a1, du1, dt1) and of the step's density,
// the kernels below run the reverse sweep and leave the adjoints of
// (x0, v0, u0, a0, du0, dt0).  The forward neighbour lists are reused; the h
// solve enters through its implicit derivative dw_i/dx = -(dF_i/dx)/(dF_i/dw_i);
// min (timestep) and max (signal speed) pass their adjoint to the arg-min /
// arg-max.  The pair reverse sweeps are written out by hand with the analytic
// derivatives of the M4 kernel family.  The SPH part is FP64; the gravity VJP
// has an FP64 and a mixed (FP32 pair terms on anchors) form.
#include <cstdio>

#include "common.cuh"
#include "pairmath.cuh"
#include "sph_math.cuh"

namespace sph {

// ---------------------------------------------------------------------------
// derivatives of the kernel functions, d/du
// ---------------------------------------------------------------------------
__device__ __forceinline__ double kd_dw(double u) {
  const double ipi = 0.318309886183791;
  if (u < 1) return 2.25 * ipi;
  if (u < 2) return 0.75 * ipi * (4 - u * u) / (u * u);
  return 0;
}
__device__ __forceinline__ double kd_dig(double u) {
  const double c = 256.0 * 3.141592653589793;
  if (u <= 0) return 0;
  if (u < 1) return c * (k_w<double>(4 * u) + 16 * u * u * k_dw<double>(4 * u));
  if (u < 2) {
    const double s = 2 - u;
    return c * (2 * s * k_w<double>(4 * s) / u + 16 * s * s * s * k_dw<double>(4 * s) / u +
                s * s * k_w<double>(4 * s) / (u * u));
  }
  return 0;
}
__device__ __forceinline__ double kd_dwdh(double u) {
  const double ipi = 0.318309886183791;
  if (u < 1) return ipi * (15 * u - 13.5 * u * u);
  if (u < 2) return ipi * (12 - 15 * u + 4.5 * u * u);
  return 0;
}
__device__ __forceinline__ double kd_dphidh(double u) {
  if (u < 1) return -4 * u + 6 * u * u * u - 3 * u * u * u * u;
  if (u < 2) return -8 * u + 12 * u * u - 6 * u * u * u + u * u * u * u;
  return 0;
}
__device__ __forceinline__ double kd_digdh(double u) { return 2 * u * k_dig<double>(u) + u * u * kd_dig(u); }

// AdjArgs: see common.cuh


constexpr int kAT = 256;  // threads of the per-particle kernels

__device__ __forceinline__ int warp_max_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ void atomic_add3(double4 *p, double x, double y, double z) {
  atomicAdd(&p->x, x);
  atomicAdd(&p->y, y);
  atomicAdd(&p->z, z);
}

// -- 1. vp, up of the forward predictor; clear the internal adjoints ---------
__global__ void k_adj_init(AdjArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double dth = 0.5 * a.sc[0];
  const double4 o = a.old[i], ac = a.pre_acc[i];
  a.vpup[i] = make_double4(o.x + ac.x * dth, o.y + ac.y * dth, o.z + ac.z * dth, o.w + ac.w * dth);
  a.vpb[i] = make_double4(0, 0, 0, 0);
  a.rhob[i] = a.rho_ext ? a.rho_ext[i] : 0.0;
  a.Pb[i] = 0; a.omb[i] = 0; a.psib[i] = 0; a.divb[i] = 0; a.curlb[i] = 0;
  a.cb[i] = 0; a.bb[i] = 0; a.prb[i] = 0;
  a.xb[i].w = 0;  // wbar of this step starts at zero
}

// -- 2. kick adjoint + the reduction sum(vbar.a1 + ubar du1) -----------------
__global__ void __launch_bounds__(kAT) k_adj_kick(AdjArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0;
  if (i < a.n) {
    const double f = 0.5 * a.sc[1] + 0.5 * a.sc[0];
    const double4 vb = a.vb[i], d = a.dots[i];
    double4 ab = a.ab[i];
    ab.x += vb.x * f; ab.y += vb.y * f; ab.z += vb.z * f; ab.w += vb.w * f;
    a.ab[i] = ab;
    s = vb.x * d.x + vb.y * d.y + vb.z * d.z + vb.w * d.w;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double ws[kAT / 32];
  if (lane_id() == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < kAT / 32; k++) t += ws[k];
    a.part[blockIdx.x] = t;
  }
}

// tau_i of compute_timestep.cpp:10-16
__device__ __forceinline__ double tau_of(double w, double vs, double up, double du, double cn1, double cn2) {
  const double dtv = cn1 * fabs(w / vs);
  const double dte = cn2 * fabs(up / du);
  return 1.0 / (1.0 / dtv + 1.0 / dte);
}

// -- 3. arg-min of tau over particles (block partials) -----------------------
__global__ void __launch_bounds__(kAT) k_adj_argmin(AdjArgs a) {
  double t = 1e300;
  int idx = 0x7fffffff;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const double ti = tau_of(a.pos[i].w, a.vsig[i], a.vpup[i].w, a.dots[i].w, a.cn1, a.cn2);
    if (ti < t || (ti == t && i < idx)) { t = ti; idx = i; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double t2 = __shfl_xor_sync(0xffffffffu, t, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
    if (t2 < t || (t2 == t && i2 < idx)) { t = t2; idx = i2; }
  }
  __shared__ double st[kAT / 32];
  __shared__ int si[kAT / 32];
  if (lane_id() == 0) { st[threadIdx.x >> 5] = t; si[threadIdx.x >> 5] = idx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kAT / 32; k++)
      if (st[k] < t || (st[k] == t && si[k] < idx)) { t = st[k]; idx = si[k]; }
    a.part[2 * blockIdx.x] = t;
    a.part[2 * blockIdx.x + 1] = (double)idx;
  }
}

// -- 4. fold: dtbar, the arg-min particle, the timestep adjoint --------------
__global__ void k_adj_timestep(AdjArgs a, int nb_kick, int nb_min) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double f = 0;
  for (int b = 0; b < nb_kick; b++) f += a.part[b];
  double t = 1e300;
  int idx = 0;
  for (int b = 0; b < nb_min; b++) {
    const double tb = a.part[nb_kick + 2 * b];
    const int ib = (int)a.part[nb_kick + 2 * b + 1];
    if (tb < t || (tb == t && ib < idx)) { t = tb; idx = ib; }
  }
  const double dtb1 = a.asc[0] + 0.5 * f;
  a.asc[1] = 0.5 * f;  // dtbar0 so far (predictor terms follow)
  a.asc[3] = (double)idx;
  a.asc[2] = 0;
  if (dtb1 == 0 || idx >= a.n) return;
  // tau = 1/(1/dtv + 1/dte); dtv = cn1 |w/vs|; dte = cn2 |up/du|
  const double w = a.pos[idx].w, vs = a.vsig[idx], up = a.vpup[idx].w, du = a.dots[idx].w;
  const double dtv = a.cn1 * fabs(w / vs), dte = a.cn2 * fabs(up / du);
  const double tau = 1.0 / (1.0 / dtv + 1.0 / dte);
  const double gv = isfinite(dtv) ? dtb1 * tau * tau / (dtv * dtv) : 0.0;  // dL/d dtv
  const double ge = isfinite(dte) ? dtb1 * tau * tau / (dte * dte) : 0.0;  // dL/d dte
  const double sw = (w / vs) >= 0 ? 1.0 : -1.0, se = (up / du) >= 0 ? 1.0 : -1.0;
  // a limit that is not active (du = 0 gives dte = inf) passes no adjoint; its
  // terms would be 0 * inf
  if (gv != 0) {
    a.xb[idx].w += gv * a.cn1 * sw / vs;
    a.asc[2] = -gv * a.cn1 * sw * w / (vs * vs);
  }
  if (ge != 0) {
    a.vpb[idx].w += ge * a.cn2 * se / du;
    a.ab[idx].w += -ge * a.cn2 * se * up / (du * du);
  }
}

// -- 5. gravity VJP: xbar_i += sum_j T_ij (m_i gbar_j - m_j gbar_i) ----------
// T_ij = I / s^3 - 3 d d^T / s^5, d = x_j - x_i, s^2 = |d|^2 + eps^2 (Plummer).
// The pair term v = T_ij w_ij is antisymmetric (d -> -d leaves T, w_ji =
// -w_ij), so xbar_j receives -v: the symmetric kernels compute each pair
// once with the tiles, work items and travelling sources of the forward
// symmetric kernels (gravity.cu), and the one-sided kernels cover the
// diagonal tiles (tile > 0) or all pairs of a small system (tile = 0).
constexpr int kGA = 128;

__global__ void __launch_bounds__(kGA) k_adj_grav_f64(int n, const double4 *__restrict__ src,
                                                      const double4 *__restrict__ ab, double4 *__restrict__ xb,
                                                      double eps2, double G, int tile) {
  __shared__ double4 sp[kGA];
  __shared__ double4 sg[kGA];
  const int t = threadIdx.x;
  const int i = blockIdx.x * kGA + t;
  const int ii = min(i, n - 1);
  const int i0 = blockIdx.x * kGA;
  const int jlo = tile > 0 ? (i0 / tile) * tile : 0;
  const int jhi = tile > 0 ? min(jlo + tile, n) : n;
  const double4 pi = src[ii];
  const double4 gi4 = ab[ii];
  const double mi = pi.w, gix = gi4.x, giy = gi4.y, giz = gi4.z;
  double rx = 0, ry = 0, rz = 0;
  for (int j0 = jlo; j0 < jhi; j0 += kGA) {
    const int j = j0 + t;
    __syncthreads();
    if (j < jhi) {
      sp[t] = src[j];
      const double4 g = ab[j];
      sg[t] = make_double4(g.x, g.y, g.z, 0);
    } else {
      sp[t] = make_double4(pi.x, pi.y, pi.z, 0);
      sg[t] = make_double4(0, 0, 0, 0);
    }
    __syncthreads();
    const int m = min(kGA, jhi - j0);
    for (int k = 0; k < m; k++) {
      const double4 q = sp[k];
      const double4 gj = sg[k];
      const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
      const double s2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
      const double inv = rsqrt_f64(s2);
      const double inv2 = inv * inv, inv3 = inv2 * inv;
      const double wx = mi * gj.x - q.w * gix, wy = mi * gj.y - q.w * giy, wz = mi * gj.z - q.w * giz;
      const double dw = dx * wx + dy * wy + dz * wz;
      const double c = 3.0 * inv2 * dw;
      rx = fma(inv3, wx - c * dx, rx);
      ry = fma(inv3, wy - c * dy, ry);
      rz = fma(inv3, wz - c * dz, rz);
    }
  }
  if (i < n) {
    double4 x = xb[i];
    x.x += G * rx; x.y += G * ry; x.z += G * rz;
    xb[i] = x;
  }
}

// mixed form of the gravity VJP: FP32 pair terms relative to the block's FP64
// anchor, FP64 per-tile accumulation
__global__ void __launch_bounds__(kGA) k_adj_grav_f32(int n, const double4 *__restrict__ src,
                                                      const double4 *__restrict__ ab, double4 *__restrict__ xb,
                                                      float eps2, double G, int tile) {
  __shared__ float4 sp[kGA];
  __shared__ float4 sg[kGA];
  const int t = threadIdx.x;
  const int i = blockIdx.x * kGA + t;
  const int ii = min(i, n - 1);
  const int i0 = blockIdx.x * kGA;
  const int jlo = tile > 0 ? (i0 / tile) * tile : 0;
  const int jhi = tile > 0 ? min(jlo + tile, n) : n;
  const double4 anc = src[min(i0, n - 1)];
  const double4 pi = src[ii];
  const double4 gi4 = ab[ii];
  const float xi = (float)(pi.x - anc.x), yi = (float)(pi.y - anc.y), zi = (float)(pi.z - anc.z);
  const float mi = (float)pi.w, gix = (float)gi4.x, giy = (float)gi4.y, giz = (float)gi4.z;
  double rx = 0, ry = 0, rz = 0;
  for (int j0 = jlo; j0 < jhi; j0 += kGA) {
    const int j = j0 + t;
    __syncthreads();
    if (j < jhi) {
      const double4 q = src[j];
      const double4 g = ab[j];
      sp[t] = make_float4((float)(q.x - anc.x), (float)(q.y - anc.y), (float)(q.z - anc.z), (float)q.w);
      sg[t] = make_float4((float)g.x, (float)g.y, (float)g.z, 0.f);
    } else {
      sp[t] = make_float4(xi, yi, zi, 0.f);
      sg[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    float px = 0.f, py = 0.f, pz = 0.f;
    const int m = min(kGA, jhi - j0);
    for (int k = 0; k < m; k++) {
      const float4 q = sp[k];
      const float4 gj = sg[k];
      const float dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
      const float s2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
      const float inv = rsqrt_f32(s2);
      const float inv2 = inv * inv, inv3 = inv2 * inv;
      const float wx = mi * gj.x - q.w * gix, wy = mi * gj.y - q.w * giy, wz = mi * gj.z - q.w * giz;
      const float c = 3.f * inv2 * (dx * wx + dy * wy + dz * wz);
      px = fmaf(inv3, wx - c * dx, px);
      py = fmaf(inv3, wy - c * dy, py);
      pz = fmaf(inv3, wz - c * dz, pz);
    }
    rx += px; ry += py; rz += pz;
  }
  if (i < n) {
    double4 x = xb[i];
    x.x += G * rx; x.y += G * ry; x.z += G * rz;
    xb[i] = x;
  }
}

// Symmetric mixed form: packed f32x2 i-pairs, FP32 positions relative to the
// i-tile's FP64 anchor, sources {x, m, gbar} travelling through the lanes
// with their FP32 j-side sums; per two pairs 31 packed FP32 instructions and
// 2 MUFU.rsq (3 sub, 3 FMA for s^2, 3 mul for s^-2, s^-3 and -3 s^-2, 6 for
// w, 3 for d.w, 1 for the scale, 3 FMA for w - c d, 3 mul by s^-3, 3 + 3 adds
// into the i- and j-side sums).  Equal masses (the forward step's device
// flag): w = m (gbar_j - gbar_i), 3 sub instead of 6, the mass applied to the
// FP64 partial sums; padding sources sit 1e18 away so that s^-3 underflows
// to 0 (the same form as the forward symmetric kernels).  Measured at
// N = 1M (reverse sweep of the bench workload, 487 ms): the source loop
// unrolled by two took 513 ms, 2 warps x 8 i-pairs per lane 519 ms; two
// half-tile blocks per FP64 item left the FP64 sweep at 1.11 s.
constexpr int kAdjWarps = 4;
constexpr int kAdjRP = 4;
constexpr int kAdjTile = kAdjWarps * 64 * kAdjRP;  // 1024

template <bool UNI>
__device__ __forceinline__ void adj_sym_f32_item(long long item, int n, int nt, const double4 *__restrict__ src,
                                                 const double4 *__restrict__ ab, double4 *__restrict__ xb,
                                                 float eps2, double G, float (&red)[2][kAdjWarps][3][32],
                                                 double (&iacc)[2 * kAdjRP * 3][kAdjWarps * 32]) {
  int b, t_lo, t_hi;
  sym_item(item, nt, b, t_lo, t_hi);
  const int j_lo = t_lo * kAdjTile, j_hi = min(t_hi * kAdjTile, n);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nxt = (l + 1) & 31;
  const int i0 = b * kAdjTile;
  const double4 anc = src[i0];
  const int ib = i0 + w * 64 * kAdjRP + l;
  f32x2 xi[kAdjRP], yi[kAdjRP], zi[kAdjRP], mi[kAdjRP], gx[kAdjRP], gy[kAdjRP], gz[kAdjRP];
#pragma unroll
  for (int p = 0; p < kAdjRP; p++) {
    float x[2] = {0.f, 0.f}, y[2] = {0.f, 0.f}, z[2] = {0.f, 0.f}, m[2] = {0.f, 0.f};
    float u[2] = {0.f, 0.f}, v[2] = {0.f, 0.f}, q[2] = {0.f, 0.f};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int i = ib + (2 * p + h) * 32;
      if (i < n) {  // padding i-slots: massless, no gbar, at the anchor
        const double4 s = src[i], g = ab[i];
        x[h] = (float)(s.x - anc.x); y[h] = (float)(s.y - anc.y); z[h] = (float)(s.z - anc.z); m[h] = (float)s.w;
        u[h] = (float)g.x; v[h] = (float)g.y; q[h] = (float)g.z;
      }
#pragma unroll
      for (int c = 0; c < 3; c++) iacc[(2 * p + h) * 3 + c][threadIdx.x] = 0.0;
    }
    xi[p] = pk2(x[0], x[1]); yi[p] = pk2(y[0], y[1]); zi[p] = pk2(z[0], z[1]); mi[p] = pk2(m[0], m[1]);
    gx[p] = pk2(u[0], u[1]); gy[p] = pk2(v[0], v[1]); gz[p] = pk2(q[0], q[1]);
  }
  const f32x2 e2 = pk2(eps2, eps2), m3 = pk2(-3.f, -3.f);
  const double gm = UNI ? G * src[0].w : G;  // UNI: the common mass joins G
  int k = 0;
  for (int jb = j_lo; jb < j_hi; jb += 32, k ^= 1) {
    float xj = UNI ? 1e18f : 0.f, yj = xj, zj = xj, mj = 0.f, gjx = 0.f, gjy = 0.f, gjz = 0.f;
    if (jb + l < j_hi) {  // padding sources: massless, no gbar, at the anchor (UNI: far away)
      const double4 s = src[jb + l], g = ab[jb + l];
      xj = (float)(s.x - anc.x); yj = (float)(s.y - anc.y); zj = (float)(s.z - anc.z); mj = (float)s.w;
      gjx = (float)g.x; gjy = (float)g.y; gjz = (float)g.z;
    }
    float ajx = 0.f, ajy = 0.f, ajz = 0.f;
    f32x2 px[kAdjRP], py[kAdjRP], pz[kAdjRP];
#pragma unroll
    for (int p = 0; p < kAdjRP; p++) px[p] = py[p] = pz[p] = 0ull;
#pragma unroll 1
    for (int s = 0; s < 32; s++) {
      const f32x2 XJ = pk2(xj, xj), YJ = pk2(yj, yj), ZJ = pk2(zj, zj), NMJ = pk2(-mj, -mj);
      const f32x2 GX = pk2(gjx, gjx), GY = pk2(gjy, gjy), GZ = pk2(gjz, gjz);
      f32x2 AX = pk2(ajx, 0.f), AY = pk2(ajy, 0.f), AZ = pk2(ajz, 0.f);
#pragma unroll
      for (int p = 0; p < kAdjRP; p++) {
        const f32x2 dx = sub2(XJ, xi[p]), dy = sub2(YJ, yi[p]), dz = sub2(ZJ, zi[p]);
        f32x2 r2 = fma2(dx, dx, e2);
        r2 = fma2(dy, dy, r2);
        r2 = fma2(dz, dz, r2);
        float r2a, r2b;
        upk2(r2, r2a, r2b);
        const f32x2 inv = pk2(rsqrt_f32(r2a), rsqrt_f32(r2b));
        const f32x2 inv2 = mul2(inv, inv);
        const f32x2 inv3 = mul2(inv2, inv), nc3 = mul2(inv2, m3);
        // w = m_i gbar_j - m_j gbar_i (UNI: gbar_j - gbar_i, the mass applied later)
        const f32x2 wx = UNI ? sub2(GX, gx[p]) : fma2(mi[p], GX, mul2(NMJ, gx[p]));
        const f32x2 wy = UNI ? sub2(GY, gy[p]) : fma2(mi[p], GY, mul2(NMJ, gy[p]));
        const f32x2 wz = UNI ? sub2(GZ, gz[p]) : fma2(mi[p], GZ, mul2(NMJ, gz[p]));
        const f32x2 nc = mul2(nc3, fma2(dz, wz, fma2(dy, wy, mul2(dx, wx))));  // -3 (d.w) / s^2
        const f32x2 vx = mul2(inv3, fma2(nc, dx, wx));
        const f32x2 vy = mul2(inv3, fma2(nc, dy, wy));
        const f32x2 vz = mul2(inv3, fma2(nc, dz, wz));
        px[p] = add2(px[p], vx);
        py[p] = add2(py[p], vy);
        pz[p] = add2(pz[p], vz);
        AX = sub2(AX, vx);
        AY = sub2(AY, vy);
        AZ = sub2(AZ, vz);
      }
      float a0, a1;
      upk2(AX, a0, a1); ajx = a0 + a1;
      upk2(AY, a0, a1); ajy = a0 + a1;
      upk2(AZ, a0, a1); ajz = a0 + a1;
      xj = __shfl_sync(0xffffffffu, xj, nxt);
      yj = __shfl_sync(0xffffffffu, yj, nxt);
      zj = __shfl_sync(0xffffffffu, zj, nxt);
      mj = __shfl_sync(0xffffffffu, mj, nxt);
      gjx = __shfl_sync(0xffffffffu, gjx, nxt);
      gjy = __shfl_sync(0xffffffffu, gjy, nxt);
      gjz = __shfl_sync(0xffffffffu, gjz, nxt);
      ajx = __shfl_sync(0xffffffffu, ajx, nxt);
      ajy = __shfl_sync(0xffffffffu, ajy, nxt);
      ajz = __shfl_sync(0xffffffffu, ajz, nxt);
    }
#pragma unroll
    for (int p = 0; p < kAdjRP; p++) {
      const f32x2 part[3] = {px[p], py[p], pz[p]};
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float a0, a1;
        upk2(part[c], a0, a1);
        iacc[(2 * p) * 3 + c][threadIdx.x] += a0;
        iacc[(2 * p + 1) * 3 + c][threadIdx.x] += a1;
      }
    }
    red[k][w][0][l] = ajx;
    red[k][w][1][l] = ajy;
    red[k][w][2][l] = ajz;
    __syncthreads();  // also orders this batch's reads of red[k] before batch + 2 writes it
    for (int qq = threadIdx.x; qq < 96; qq += kAdjWarps * 32) {
      const int c = qq >> 5, ll = qq & 31;
      double sum = 0.0;
#pragma unroll
      for (int v = 0; v < kAdjWarps; v++) sum += (double)red[k][v][c][ll];
      if (jb + ll < j_hi) atomicAdd(&reinterpret_cast<double *>(xb + jb + ll)[c], gm * sum);
    }
  }
#pragma unroll
  for (int r = 0; r < 2 * kAdjRP; r++) {
    const int i = ib + r * 32;
    if (i < n) {
      double *o = reinterpret_cast<double *>(xb + i);
#pragma unroll
      for (int c = 0; c < 3; c++) atomicAdd(o + c, gm * iacc[r * 3 + c][threadIdx.x]);
    }
  }
}

// mass_mixed: the forward step's device word, 0 when all masses are equal
__global__ void __launch_bounds__(kAdjWarps * 32) k_adj_grav_sym_f32(int n, int nt, const double4 *__restrict__ src,
                                                                    const double4 *__restrict__ ab,
                                                                    double4 *__restrict__ xb, float eps2, double G,
                                                                    const int *__restrict__ mass_mixed) {
  __shared__ float red[2][kAdjWarps][3][32];
  __shared__ double iacc[2 * kAdjRP * 3][kAdjWarps * 32];  // [i-slot * 3 + component][thread]
  if (mass_mixed != nullptr && __ldg(mass_mixed) == 0)
    adj_sym_f32_item<true>(blockIdx.x, n, nt, src, ab, xb, eps2, G, red, iacc);
  else
    adj_sym_f32_item<false>(blockIdx.x, n, nt, src, ab, xb, eps2, G, red, iacc);
}

// Symmetric FP64 form: absolute coordinates, kAdj64R i-particles per lane
// with their sums in registers; equal masses as in the mixed form (padding
// sources 1e150 away).
constexpr int kAdj64Warps = 4;
constexpr int kAdj64R = 8;
static_assert(kAdj64Warps * 32 * kAdj64R == kAdjTile, "the FP64 form shares the tile layout");

template <bool UNI>
__device__ __forceinline__ void adj_sym_f64_item(long long item, int n, int nt, const double4 *__restrict__ src,
                                                 const double4 *__restrict__ ab, double4 *__restrict__ xb,
                                                 double eps2, double G, double (&red)[2][kAdj64Warps][3][32]) {
  int b, t_lo, t_hi;
  sym_item(item, nt, b, t_lo, t_hi);
  const int j_lo = t_lo * kAdjTile, j_hi = min(t_hi * kAdjTile, n);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nxt = (l + 1) & 31;
  const int ib = b * kAdjTile + w * 32 * kAdj64R + l;
  const double4 far = src[b * kAdjTile];  // position given to padding slots
  double xi[kAdj64R], yi[kAdj64R], zi[kAdj64R], mi[kAdj64R], gx[kAdj64R], gy[kAdj64R], gz[kAdj64R];
  double rx[kAdj64R], ry[kAdj64R], rz[kAdj64R];
#pragma unroll
  for (int r = 0; r < kAdj64R; r++) {
    const int i = ib + r * 32;
    const bool in = i < n;
    const double4 s = in ? src[i] : make_double4(far.x, far.y, far.z, 0.0);
    const double4 g = in ? ab[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    xi[r] = s.x; yi[r] = s.y; zi[r] = s.z; mi[r] = s.w;
    gx[r] = g.x; gy[r] = g.y; gz[r] = g.z;
    rx[r] = ry[r] = rz[r] = 0.0;
  }
  const double gm = UNI ? G * src[0].w : G;  // UNI: the common mass joins G
  int k = 0;
  for (int jb = j_lo; jb < j_hi; jb += 32, k ^= 1) {
    const bool in = jb + l < j_hi;
    const double4 s = in ? src[jb + l] : (UNI ? make_double4(1e150, 1e150, 1e150, 0.0)
                                              : make_double4(far.x, far.y, far.z, 0.0));
    const double4 g = in ? ab[jb + l] : make_double4(0.0, 0.0, 0.0, 0.0);
    double xj = s.x, yj = s.y, zj = s.z, mj = s.w, gjx = g.x, gjy = g.y, gjz = g.z;
    double ajx = 0.0, ajy = 0.0, ajz = 0.0;
#pragma unroll 1
    for (int st = 0; st < 32; st++) {
#pragma unroll
      for (int r = 0; r < kAdj64R; r++) {
        const double dx = xj - xi[r], dy = yj - yi[r], dz = zj - zi[r];
        const double s2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
        const double inv = rsqrt_f64(s2);
        const double inv2 = inv * inv, inv3 = inv2 * inv;
        const double wx = UNI ? gjx - gx[r] : mi[r] * gjx - mj * gx[r];
        const double wy = UNI ? gjy - gy[r] : mi[r] * gjy - mj * gy[r];
        const double wz = UNI ? gjz - gz[r] : mi[r] * gjz - mj * gz[r];
        const double c = 3.0 * inv2 * (dx * wx + dy * wy + dz * wz);
        const double vx = inv3 * (wx - c * dx), vy = inv3 * (wy - c * dy), vz = inv3 * (wz - c * dz);
        rx[r] += vx; ry[r] += vy; rz[r] += vz;
        ajx -= vx; ajy -= vy; ajz -= vz;
      }
      xj = __shfl_sync(0xffffffffu, xj, nxt);
      yj = __shfl_sync(0xffffffffu, yj, nxt);
      zj = __shfl_sync(0xffffffffu, zj, nxt);
      mj = __shfl_sync(0xffffffffu, mj, nxt);
      gjx = __shfl_sync(0xffffffffu, gjx, nxt);
      gjy = __shfl_sync(0xffffffffu, gjy, nxt);
      gjz = __shfl_sync(0xffffffffu, gjz, nxt);
      ajx = __shfl_sync(0xffffffffu, ajx, nxt);
      ajy = __shfl_sync(0xffffffffu, ajy, nxt);
      ajz = __shfl_sync(0xffffffffu, ajz, nxt);
    }
    red[k][w][0][l] = ajx;
    red[k][w][1][l] = ajy;
    red[k][w][2][l] = ajz;
    __syncthreads();  // also orders this batch's reads of red[k] before batch + 2 writes it
    for (int qq = threadIdx.x; qq < 96; qq += kAdj64Warps * 32) {
      const int c = qq >> 5, ll = qq & 31;
      double sum = 0.0;
#pragma unroll
      for (int v = 0; v < kAdj64Warps; v++) sum += red[k][v][c][ll];
      if (jb + ll < j_hi) atomicAdd(&reinterpret_cast<double *>(xb + jb + ll)[c], gm * sum);
    }
  }
#pragma unroll
  for (int r = 0; r < kAdj64R; r++) {
    const int i = ib + r * 32;
    if (i < n) {
      double *o = reinterpret_cast<double *>(xb + i);
      atomicAdd(o + 0, gm * rx[r]);
      atomicAdd(o + 1, gm * ry[r]);
      atomicAdd(o + 2, gm * rz[r]);
    }
  }
}

__global__ void __launch_bounds__(kAdj64Warps * 32) k_adj_grav_sym_f64(int n, int nt, const double4 *__restrict__ src,
                                                                      const double4 *__restrict__ ab,
                                                                      double4 *__restrict__ xb, double eps2, double G,
                                                                      const int *__restrict__ mass_mixed) {
  __shared__ double red[2][kAdj64Warps][3][32];
  if (mass_mixed != nullptr && __ldg(mass_mixed) == 0)
    adj_sym_f64_item<true>(blockIdx.x, n, nt, src, ab, xb, eps2, G, red);
  else
    adj_sym_f64_item<false>(blockIdx.x, n, nt, src, ab, xb, eps2, G, red);
}

// -- 6. hydro VJP (warp per leaf, lane per particle, lists of find_ngb) ------
// Per pair the forward computes (dev_hydro_dots.cu:25-84 with the j-side):
//   a_i -= m_j acc d,  a_j += m_i acc d,  du_i += ud * drdv
// with d = x_i - x_j, ds = |d|, u = ds / h_i, h_i = w_i / 2,
//   visc = (pr_i + pr_j)(-alpha mu + beta mu^2), mu = drdv (b_i + b_j) / ((c_i + c_j) ds)   [drdv < 0]
//   acc = (pr_i + visc/2) dw(u) / h^5 - (pr_i om_i + psi_i/2) / m_j dig(u) / h^2
//   ud  = m_j (pr_i + visc/2) dw(u) / h^5 - pr_i om_i dig(u) / h^2
// where pr = P / rho^2, c = sqrt(gamma P / rho), b = Balsara factor.  The
// reverse sweep leaves xbar, vpbar, wbar_i and the adjoints of the
// per-particle pr, c, b, om, psi (folded into rho, P, div, curl, w later).
__global__ void __launch_bounds__(128) k_adj_hydro(AdjArgs a) {
  const int leaf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (leaf >= a.nleaf) return;
  const int lane = (int)lane_id();
  const int s = leaf * kLeaf + lane;
  const bool valid = s < a.n;
  double4 pi = make_double4(0, 0, 0, 1), vi = make_double4(0, 0, 0, 0), hi4 = make_double4(1, 0, 0, 0),
          di = make_double4(0, 0, 0, 0), abi = make_double4(0, 0, 0, 0);
  double mi = 1;
  int cnt = 0;
  if (valid) {
    pi = a.pos[s];
    vi = a.vpup[s];
    hi4 = a.hyd[s];
    di = a.dd[s];
    abi = a.ab[s];
    mi = a.vel[s].w;
    cnt = min(a.n_ngb[s], a.cap);
  }
  const int kmax = warp_max_i(cnt);
  const int *lst = a.list + (size_t)leaf * a.cap * kLeaf + lane;
  const double gam = a.gamma, alpha = a.alpha, beta = a.beta;
  const double wi = pi.w, hh = 0.5 * wi;
  const double ih = hh > 0 ? 1.0 / hh : 0.0, ih2 = ih * ih, ih5 = ih2 * ih2 * ih;
  const double pr_i = hi4.x > 0 ? hi4.y / (hi4.x * hi4.x) : 0.0;
  const double c_i = hi4.x > 0 ? sqrt(gam * hi4.y / hi4.x) : 0.0;
  const double ad_i = fabs(di.x);
  const double b_i = ad_i / (ad_i + di.y + 0.0001 * c_i / (0.5 * wi));
  const double om_i = di.z, psi_i = a.use_psi ? di.w : 0.0;
  // i-side accumulators
  double xbx = 0, xby = 0, xbz = 0, vbx = 0, vby = 0, vbz = 0, ihb = 0;
  double prb_i = 0, cb_i = 0, bb_i = 0, omb_i = 0, psib_i = 0;
  for (int k = 0; k < kmax; k++) {
    if (k >= cnt) continue;
    const int j = __ldg(lst + (size_t)k * kLeaf);
    if (j == s) continue;
    const double4 pj = ld4(a.pos + j), vj = ld4(a.vpup + j), fj = ld4(a.aux + j);
    const double4 abj = ld4(a.ab + j);
    const double mj = __ldg(&a.vel[j].w);
    const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
    const double ds = sqrt(dx * dx + dy * dy + dz * dz);
    const double ids = ds > 0 ? 1.0 / ds : 0.0, imj = 1.0 / mj;
    const double drdv = dx * dvx + dy * dvy + dz * dvz;
    const double u = ds * ih;
    const double pr_j = fj.y, c_j = fj.x, b_j = fj.z;  // the neighbour's factors (k_hydro_prep)
    // forward
    const bool neg = drdv < 0;
    const double S = c_i + c_j, B = b_i + b_j, Q = pr_i + pr_j;
    double mu0 = 0, mu = 0, visc = 0;
    if (neg) {
      mu0 = drdv * ids / S;
      mu = mu0 * B;
      visc = Q * (-alpha * mu + beta * mu * mu);
    }
    const double dwu = k_dw<double>(u), digu = k_dig<double>(u);
    const double A1 = pr_i + 0.5 * visc;
    const double K2 = pr_i * om_i + 0.5 * psi_i;
    const double acc = A1 * dwu * ih5 - K2 * imj * digu * ih2;
    const double ud = mj * A1 * dwu * ih5 - pr_i * om_i * digu * ih2;
    // output adjoints of the pair: force vector acc*d (i: -m_j, j: +m_i), and ud*drdv
    const double gx = -mj * abi.x + mi * abj.x, gy = -mj * abi.y + mi * abj.y, gz = -mj * abi.z + mi * abj.z;
    const double accb = gx * dx + gy * dy + gz * dz;
    const double udb = abi.w * drdv;
    double dxb = acc * gx, dyb = acc * gy, dzb = acc * gz;
    double drdvb = abi.w * ud;
    // acc, ud -> A1, dwu, digu, ih5, ih2, pr_i, om_i, psi_i
    const double A1b = accb * dwu * ih5 + udb * mj * dwu * ih5;
    const double dwub = accb * A1 * ih5 + udb * mj * A1 * ih5;
    const double digub = -accb * K2 * imj * ih2 - udb * pr_i * om_i * ih2;
    const double ih5b = accb * A1 * dwu + udb * mj * A1 * dwu;
    const double ih2b = -accb * K2 * imj * digu - udb * pr_i * om_i * digu;
    const double K2b = -accb * imj * digu * ih2;
    prb_i += K2b * om_i - udb * om_i * digu * ih2 + A1b;
    omb_i += K2b * pr_i - udb * pr_i * digu * ih2;
    psib_i += 0.5 * K2b;
    ihb += ih5b * 5.0 * ih2 * ih2 + ih2b * 2.0 * ih;
    // visc
    if (neg) {
      const double viscb = 0.5 * A1b;
      const double Qb = viscb * (-alpha * mu + beta * mu * mu);
      const double mub = viscb * Q * (-alpha + 2.0 * beta * mu);
      prb_i += Qb;
      const double prjb = Qb;
      const double mu0b = mub * B;
      const double Bb = mub * mu0;
      bb_i += Bb;
      const double Sb = -mu0b * mu0 / S;
      cb_i += Sb;
      drdvb += mu0b * ids / S;
      const double dsb_v = -mu0b * mu0 * ids;
      atomicAdd(&a.prb[j], prjb);
      atomicAdd(&a.bb[j], Bb);
      atomicAdd(&a.cb[j], Sb);
      dxb += dsb_v * dx * ids; dyb += dsb_v * dy * ids; dzb += dsb_v * dz * ids;
    }
    // u = ds * ih
    const double ub = dwub * kd_dw(u) + digub * kd_dig(u);
    ihb += ub * ds;
    const double dsb = ub * ih;
    dxb += dsb * dx * ids; dyb += dsb * dy * ids; dzb += dsb * dz * ids;  // ids = 0 where ds = 0
    // drdv = d . dv
    dxb += drdvb * dvx; dyb += drdvb * dvy; dzb += drdvb * dvz;
    const double dvxb = drdvb * dx, dvyb = drdvb * dy, dvzb = drdvb * dz;
    xbx += dxb; xby += dyb; xbz += dzb;
    vbx += dvxb; vby += dvyb; vbz += dvzb;
    atomic_add3(&a.xb[j], -dxb, -dyb, -dzb);
    atomic_add3(&a.vpb[j], -dvxb, -dvyb, -dvzb);
  }
  if (!valid) return;
  atomic_add3(&a.xb[s], xbx, xby, xbz);
  atomic_add3(&a.vpb[s], vbx, vby, vbz);
  // ih = 2 / w  ->  wbar += ihb * (-2 / w^2) = -ihb ih^2 / 2
  atomicAdd(&a.xb[s].w, -0.5 * ihb * ih * ih);
  atomicAdd(&a.prb[s], prb_i);
  atomicAdd(&a.cb[s], cb_i);
  atomicAdd(&a.bb[s], bb_i);
  atomicAdd(&a.omb[s], omb_i);
  atomicAdd(&a.psib[s], a.use_psi ? psib_i : 0.0);
}

// -- 7. signal-speed adjoint at the arg-min particle of the timestep ---------
// vsig_i = max_j vs_ij, vs = c_i + c_j - beta drdv / ds (drdv < 0) else c_i + c_j;
// the adjoint goes to the first pair (list order) that attains the maximum,
// recomputed here in FP64 (the mixed form's forward value is FP32).
__device__ __forceinline__ double pair_vs(const AdjArgs &a, int s, int j, double c_i, double4 pi, double4 vi) {
  const double4 pj = a.pos[j], vj = a.vpup[j], hj = a.hyd[j];
  const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
  const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
  const double ds = sqrt(dx * dx + dy * dy + dz * dz);
  const double drdv = dx * dvx + dy * dvy + dz * dvz;
  double vs = c_i + sqrt(a.gamma * hj.y / hj.x);
  if (drdv < 0) vs -= a.beta * drdv / ds;
  return vs;
}

__global__ void k_adj_vsig(AdjArgs a) {
  if (threadIdx.x != 0) return;
  const double vsb = a.asc[2];
  const int s = (int)a.asc[3];
  if (vsb == 0 || s < 0 || s >= a.n) return;
  const int leaf = s / kLeaf, lane = s % kLeaf;
  const int cnt = min(a.n_ngb[s], a.cap);
  const double4 pi = a.pos[s], vi = a.vpup[s], hi4 = a.hyd[s];
  const double gam = a.gamma, beta = a.beta;
  const double c_i = sqrt(gam * hi4.y / hi4.x);
  int kbest = -1;
  double best = -1e300;
  for (int k = 0; k < cnt; k++) {
    const int j = a.list[((size_t)leaf * a.cap + k) * kLeaf + lane];
    const double vs = pair_vs(a, s, j, c_i, pi, vi);
    if (vs > best) { best = vs; kbest = k; }
  }
  if (kbest < 0) return;
  {
    const int j = a.list[((size_t)leaf * a.cap + kbest) * kLeaf + lane];
    const double4 pj = a.pos[j], vj = a.vpup[j];
    const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
    const double ds = sqrt(dx * dx + dy * dy + dz * dz);
    const double drdv = dx * dvx + dy * dvy + dz * dvz;
    a.cb[s] += vsb;
    a.cb[j] += vsb;
    if (drdv < 0 && ds > 0) {
      const double drdvb = -beta * vsb / ds;
      const double dsb = beta * vsb * drdv / (ds * ds);
      const double gx = dsb * dx / ds + drdvb * dvx, gy = dsb * dy / ds + drdvb * dvy, gz = dsb * dz / ds + drdvb * dvz;
      a.xb[s].x += gx; a.xb[s].y += gy; a.xb[s].z += gz;
      a.xb[j].x -= gx; a.xb[j].y -= gy; a.xb[j].z -= gz;
      a.vpb[s].x += drdvb * dx; a.vpb[s].y += drdvb * dy; a.vpb[s].z += drdvb * dz;
      a.vpb[j].x -= drdvb * dx; a.vpb[j].y -= drdvb * dy; a.vpb[j].z -= drdvb * dz;
    }
  }
}

// -- 8. per particle: pr, c, b -> rho, P, div, curl, w; then the EOS ---------
__global__ void k_adj_particle(AdjArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double4 h = a.hyd[i], d = a.dd[i], p = a.pos[i];
  const double rho = h.x, P = h.y, w = p.w, gam = a.gamma;
  double rhob = a.rhob[i], Pb = a.Pb[i];
  if (!(rho > 0)) return;
  // pr = P / rho^2
  const double prb = a.prb[i];
  Pb += prb / (rho * rho);
  rhob += -2.0 * prb * P / (rho * rho * rho);
  // c = sqrt(gamma P / rho)
  const double c = sqrt(gam * P / rho);
  double cb = a.cb[i];
  // b = |D| / (|D| + C + 1e-4 c / (w/2))
  const double bb = a.bb[i];
  double divb = a.divb[i], curlb = a.curlb[i], wb = 0;
  if (bb != 0) {
    const double ad = fabs(d.x);
    const double kk = 0.0001 / (0.5 * w);
    const double den = ad + d.y + kk * c;
    const double q = bb / (den * den);
    const double adb = q * (den - ad);
    curlb += -q * ad;
    cb += -q * ad * kk;
    wb += q * ad * kk * c / w;  // d(kk)/dw = -kk / w
    divb += d.x >= 0 ? adb : -adb;
  }
  if (c > 0) {
    Pb += cb * gam / (2.0 * c * rho);
    rhob += -cb * c / (2.0 * rho);
  }
  // EOS: P(rho, up)
  double upb = 0;
  const double up = a.vpup[i].w;
  if (a.eos_mode == SPH_EOS_IDEAL) {
    rhob += Pb * (gam - 1) * up;
    upb += Pb * (gam - 1) * rho;
  } else if (Pb != 0) {
    const double DU = 5.89994031541978, EU = 1.90698842928778e+15, PU = 1.1251117914994e+16;
    const double AMU = 1.66054e-24, KB = 1.380658e-16, AR = 7.56591414984829e-15, tb = 1.0e6;
    const double mu = h.w * AMU;
    const double dens = rho * DU, en = up * EU;
    const double r = -dens * (en / (tb * tb)) / (AR * tb * tb);
    const double qq = (KB / AR) / (gam - 1) * dens / (((mu * tb) * tb) * tb);
    // the positive root of x^4 + q x + r = 0 (T = tb x), recovered from P:
    // (dens KB T / mu + AR T^4 / 3) / PU = P is solved by Newton from the bound
    double x = fmin(-r / qq, pow(-r, 0.25));
    for (int it = 0; it < 60; it++) {
      const double x3 = x * x * x;
      const double xn = x - (x3 * x + qq * x + r) / (4 * x3 + qq);
      if (xn == x) break;
      x = xn;
    }
    const double T = tb * x;
    const double dPdT = (dens * KB / mu + 4.0 * AR * T * T * T / 3.0) / PU;
    const double den4 = 4 * x * x * x + qq;
    const double dxdrho = x * x * x * x / (rho * den4);    // dq/drho = q/rho, dr/drho = r/rho
    const double dxdu = -(r / up) / den4;                   // dr/du = r/u
    rhob += Pb * (KB * T / mu * DU / PU + dPdT * tb * dxdrho);
    upb += Pb * dPdT * tb * dxdu;
  }
  a.rhob[i] = rhob;
  a.divb[i] = divb;
  a.curlb[i] = curlb;
  a.vpb[i].w += upb;
  a.xb[i].w += wb;
}

// -- 9. density VJP (warp per leaf): epilogue reverse, then pairs ------------
// Forward (dev_density_loop.cu:29-86, with m_j in the divergence weight):
//   R = sum m_j W(u), O = sum m_j dwdh(u), Q = sum m_j dphidh(u), S = -sum digdh(u),
//   Dv = sum m_j dw(u) (d.dv), Cv = sum m_j dw(u) (d x dv),  u = 2 ds / w
//   rho = R/h^3, om = O/(h^3 S), psi = Q/(h S), div = Dv/(rho h^5), curl = |Cv|/(rho h^5)
__global__ void __launch_bounds__(128) k_adj_density(AdjArgs a) {
  const int leaf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (leaf >= a.nleaf) return;
  const int lane = (int)lane_id();
  const int s = leaf * kLeaf + lane;
  const bool valid = s < a.n;
  double4 pi = make_double4(0, 0, 0, 1), vi = make_double4(0, 0, 0, 0);
  int cnt = 0;
  if (valid) {
    pi = a.pos[s];
    vi = a.vpup[s];
    cnt = min(a.n_ngb[s], a.cap);
  }
  const int kmax = warp_max_i(cnt);
  const int *lst = a.list + (size_t)leaf * a.cap * kLeaf + lane;
  const double w = pi.w;
  const double i2w = w > 0 ? 2.0 / w : 0.0;
  // forward sums: from the kept step when it recorded them, else summed again
  double R = 0, O = 0, Qs = 0, S = 0, Dv = 0, Cx = 0, Cy = 0, Cz = 0;
  for (int k = 0; k < (a.dsum ? 0 : kmax); k++) {
    if (k >= cnt) continue;
    const int j = __ldg(lst + (size_t)k * kLeaf);
    const double4 pj = ld4(a.pos + j), vj = ld4(a.vpup + j);
    const double mj = __ldg(&a.vel[j].w);
    const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
    const double u = sqrt(dx * dx + dy * dy + dz * dz) * i2w;
    R += mj * k_w<double>(u);
    O += mj * k_dwdh<double>(u);
    Qs += mj * k_dphidh<double>(u);
    S -= k_digdh<double>(u);
    const double wt = mj * k_dw<double>(u);
    Dv += wt * (dx * dvx + dy * dvy + dz * dvz);
    Cx += wt * (dy * dvz - dz * dvy);
    Cy += wt * (dz * dvx - dx * dvz);
    Cz += wt * (dx * dvy - dy * dvx);
  }
  // epilogue reverse
  double Rb = 0, Ob = 0, Qb = 0, Sb = 0, Dvb = 0, Cxb = 0, Cyb = 0, Czb = 0, wb = 0;
  if (valid && w > 0 && cnt > 0) {
    const double h = 0.5 * w, h3 = h * h * h, h5 = h3 * h * h;
    double rho, div, om_k = 0, ps_k = 0;
    if (a.dsum) {  // the forward outputs and the sums they do not determine (S and the curl vector)
      const double4 sm4 = a.dsum[s], d4 = a.dd[s];
      S = sm4.x; Cx = sm4.y; Cy = sm4.z; Cz = sm4.w;
      rho = a.hyd[s].x;
      div = d4.x;
      om_k = d4.z;
      ps_k = d4.w;
    } else {
      rho = R / h3;
      div = Dv / (rho * h5);
    }
    const double cm = sqrt(Cx * Cx + Cy * Cy + Cz * Cz);
    const double curl = cm / (rho * h5);
    double rhob = a.rhob[s], hb = 0;
    const double divb = a.divb[s], curlb = a.curlb[s];
    Dvb = divb / (rho * h5);
    rhob -= divb * div / rho;
    hb -= 5.0 * divb * div / h;
    if (cm > 0) {
      const double f = curlb / (cm * rho * h5);
      Cxb = f * Cx; Cyb = f * Cy; Czb = f * Cz;
    }
    rhob -= curlb * curl / rho;
    hb -= 5.0 * curlb * curl / h;
    if (S != 0) {
      const double om = a.dsum ? om_k : O / (h3 * S), ps = a.dsum ? ps_k : Qs / (h * S);
      const double omb = a.omb[s], psb = a.psib[s];
      Ob = omb / (h3 * S);
      Sb -= omb * om / S;
      hb -= 3.0 * omb * om / h;
      Qb = psb / (h * S);
      Sb -= psb * ps / S;
      hb -= psb * ps / h;
    }
    Rb = rhob / h3;
    hb -= 3.0 * rhob * rho / h;
    wb = 0.5 * hb;
  }
  // pairs
  double xbx = 0, xby = 0, xbz = 0, vbx = 0, vby = 0, vbz = 0;
  for (int k = 0; k < kmax; k++) {
    if (k >= cnt) continue;
    const int j = __ldg(lst + (size_t)k * kLeaf);
    if (j == s) continue;
    const double4 pj = ld4(a.pos + j), vj = ld4(a.vpup + j);
    const double mj = __ldg(&a.vel[j].w);
    const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
    const double ds = sqrt(dx * dx + dy * dy + dz * dz);
    const double u = ds * i2w;
    const double dwu = k_dw<double>(u);
    const double drdv = dx * dvx + dy * dvy + dz * dvz;
    const double crx = dy * dvz - dz * dvy, cry = dz * dvx - dx * dvz, crz = dx * dvy - dy * dvx;
    const double cdot = Cxb * crx + Cyb * cry + Czb * crz;
    const double ub = mj * (Rb * u * dwu + Ob * kd_dwdh(u) + Qb * kd_dphidh(u)) - Sb * kd_digdh(u) +
                      mj * kd_dw(u) * (Dvb * drdv + cdot);
    const double wt = mj * dwu;
    // d/d(d) of Dvb (d.dv) + Cb.(d x dv) = Dvb dv + dv x Cb ; d/d(dv) = Dvb d + Cb x d
    double dxb = wt * (Dvb * dvx + (dvy * Czb - dvz * Cyb));
    double dyb = wt * (Dvb * dvy + (dvz * Cxb - dvx * Czb));
    double dzb = wt * (Dvb * dvz + (dvx * Cyb - dvy * Cxb));
    const double dvxb = wt * (Dvb * dx + (Cyb * dz - Czb * dy));
    const double dvyb = wt * (Dvb * dy + (Czb * dx - Cxb * dz));
    const double dvzb = wt * (Dvb * dz + (Cxb * dy - Cyb * dx));
    if (ds > 0) {
      const double g = ub * i2w / ds;
      dxb += g * dx; dyb += g * dy; dzb += g * dz;
    }
    wb -= ub * u / w;
    xbx += dxb; xby += dyb; xbz += dzb;
    vbx += dvxb; vby += dvyb; vbz += dvzb;
    atomic_add3(&a.xb[j], -dxb, -dyb, -dzb);
    atomic_add3(&a.vpb[j], -dvxb, -dvyb, -dvzb);
  }
  if (!valid) return;
  atomic_add3(&a.xb[s], xbx, xby, xbz);
  atomic_add3(&a.vpb[s], vbx, vby, vbz);
  atomicAdd(&a.xb[s].w, wb);
}

// -- 10. h-solve implicit derivative: xbar -= lambda_i dF_i/dx, lambda_i = wbar_i / F_w,i
// F_i = sum_j ig(2 ds/w_i) - N;  F_w = -(1/w) sum digdh(u);  dF_i/dx_i = sum_j 4 dig(u)/w^2 d_ij
__global__ void __launch_bounds__(128) k_adj_hsolve(AdjArgs a) {
  const int leaf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (leaf >= a.nleaf) return;
  const int lane = (int)lane_id();
  const int s = leaf * kLeaf + lane;
  const bool valid = s < a.n;
  double4 pi = make_double4(0, 0, 0, 1);
  int cnt = 0;
  double wbar = 0;
  if (valid) {
    pi = a.pos[s];
    cnt = min(a.n_ngb[s], a.cap);
    wbar = a.xb[s].w;
  }
  const int kmax = warp_max_i(cnt);
  const int *lst = a.list + (size_t)leaf * a.cap * kLeaf + lane;
  const double w = pi.w;
  const double i2w = w > 0 ? 2.0 / w : 0.0;
  double Fw = 0;
  for (int k = 0; k < kmax; k++) {
    if (k >= cnt) continue;
    const int j = __ldg(lst + (size_t)k * kLeaf);
    const double4 pj = ld4(a.pos + j);
    const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    Fw -= k_digdh<double>(sqrt(dx * dx + dy * dy + dz * dz) * i2w);
  }
  Fw = w > 0 ? Fw / w : 0.0;
  const double lam = (valid && Fw != 0 && wbar != 0) ? wbar / Fw : 0.0;
  double xbx = 0, xby = 0, xbz = 0;
  if (__any_sync(0xffffffffu, lam != 0)) {
    for (int k = 0; k < kmax; k++) {
      if (k >= cnt || lam == 0) continue;
      const int j = __ldg(lst + (size_t)k * kLeaf);
      if (j == s) continue;
      const double4 pj = ld4(a.pos + j);
      const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
      const double u = sqrt(dx * dx + dy * dy + dz * dz) * i2w;
      const double c = -lam * 4.0 * k_dig<double>(u) / (w * w);
      xbx += c * dx; xby += c * dy; xbz += c * dz;
      atomic_add3(&a.xb[j], -c * dx, -c * dy, -c * dz);
    }
  }
  if (!valid) return;
  atomic_add3(&a.xb[s], xbx, xby, xbz);
}

// -- 11. predictor reverse + dtbar0 partials ---------------------------------
__global__ void __launch_bounds__(kAT) k_adj_predict(AdjArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0;
  if (i < a.n) {
    const double dt0 = a.sc[0], dth = 0.5 * dt0;
    const double4 xb = a.xb[i], vpb = a.vpb[i], o = a.old[i], ac = a.pre_acc[i];
    double4 vb = a.vb[i];
    vb.x += xb.x * dt0 + vpb.x;
    vb.y += xb.y * dt0 + vpb.y;
    vb.z += xb.z * dt0 + vpb.z;
    vb.w += vpb.w;
    a.vb[i] = vb;
    a.ab[i] = make_double4(vpb.x * dth, vpb.y * dth, vpb.z * dth, vpb.w * dth);
    a.xb[i].w = 0;
    s = xb.x * o.x + xb.y * o.y + xb.z * o.z + 0.5 * (vpb.x * ac.x + vpb.y * ac.y + vpb.z * ac.z + vpb.w * ac.w);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double ws[kAT / 32];
  if (lane_id() == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < kAT / 32; k++) t += ws[k];
    a.part[blockIdx.x] = t;
  }
}

__global__ void k_adj_predict_final(AdjArgs a, int nb) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t = 0;
  for (int b = 0; b < nb; b++) t += a.part[b];
  a.asc[1] += t;
}

// block partials: nb (kick sum) + 2 nb (arg-min value, index), reused by the predictor sum
int adjoint_part_doubles(int n) { return 3 * ((n + kAT - 1) / kAT) + 8; }

// The whole reverse sweep; src = packed gravity sources {x1, m} of the step.
int launch_hydro_prep(int n, const double4 *pos, const double4 *vel, const double4 *hyd, const double4 *dd,
                      double gamma, double4 *aux, cudaStream_t st);

int launch_adjoint(AdjArgs a, const double4 *src, const int *mass_mixed, double eps, double G, int precision,
                   cudaStream_t st) {
  const int n = a.n;
  const int nb = (n + kAT - 1) / kAT;
  const int warps_blocks = (a.nleaf * 32 + 127) / 128;
  int launches = 0;
  k_adj_init<<<nb, kAT, 0, st>>>(a); launches++;
  k_adj_kick<<<nb, kAT, 0, st>>>(a); launches++;
  AdjArgs b = a;
  b.part = a.part + nb;
  k_adj_argmin<<<nb, kAT, 0, st>>>(b); launches++;
  k_adj_timestep<<<1, 32, 0, st>>>(a, nb, nb); launches++;
  {
    // diagonal tiles one-sided (plain read-modify-write of xbar), then the
    // pairs above them once each (atomics on top)
    static_assert(kAdjTile % kGA == 0, "diagonal tiles must hold whole blocks");
    const int nt = (n + kAdjTile - 1) / kAdjTile;
    const int tile = nt < 2 ? 0 : kAdjTile;
    if (precision == SPH_PREC_FP64)
      k_adj_grav_f64<<<(n + kGA - 1) / kGA, kGA, 0, st>>>(n, src, a.ab, a.xb, eps * eps, G, tile);
    else
      k_adj_grav_f32<<<(n + kGA - 1) / kGA, kGA, 0, st>>>(n, src, a.ab, a.xb, (float)(eps * eps), G, tile);
    launches++;
    if (nt >= 2) {
      if (precision == SPH_PREC_FP64)
        k_adj_grav_sym_f64<<<(unsigned)sym_items(nt), kAdj64Warps * 32, 0, st>>>(n, nt, src, a.ab, a.xb, eps * eps, G,
                                                                                  mass_mixed);
      else
        k_adj_grav_sym_f32<<<(unsigned)sym_items(nt), kAdjWarps * 32, 0, st>>>(n, nt, src, a.ab, a.xb,
                                                                            (float)(eps * eps), G, mass_mixed);
      launches++;
    }
  }
  launches += launch_hydro_prep(a.n, a.pos, a.vel, a.hyd, a.dd, a.gamma, a.aux, st);  // the neighbours' factors
  k_adj_hydro<<<warps_blocks, 128, 0, st>>>(a); launches++;
  k_adj_vsig<<<1, 32, 0, st>>>(a); launches++;
  k_adj_particle<<<nb, kAT, 0, st>>>(a); launches++;
  k_adj_density<<<warps_blocks, 128, 0, st>>>(a); launches++;
  k_adj_hsolve<<<warps_blocks, 128, 0, st>>>(a); launches++;
  k_adj_predict<<<nb, kAT, 0, st>>>(a); launches++;
  k_adj_predict_final<<<1, 32, 0, st>>>(a, nb); launches++;
  return launches;
}

}  // namespace sph
