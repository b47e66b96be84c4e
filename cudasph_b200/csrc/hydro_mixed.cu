// hydro_mixed.cu -- the mixed-precision form of the density and hydro loops.
//
// Neighbour records are gathered as in the FP64 form; the pair separation
// and velocity difference are formed in FP64 (exact differences of the FP64
// coordinates, rounded once) and everything per pair after that -- the kernel
// functions, the artificial viscosity and the force terms -- runs in FP32.
// Each per-particle sum is a compensated (Kahan-Babuska) float pair.  The
// per-particle normalisation, the j-side atomics and all outputs stay FP64.
#include "common.cuh"
#include "sph_math.cuh"

namespace sph {


struct KSum {
  float hi = 0.f, lo = 0.f;
  __device__ __forceinline__ void add(float v) {
    const float s = hi + v;
    const float bp = s - hi;
    lo += (hi - (s - bp)) + (v - bp);
    hi = s;
  }
  __device__ __forceinline__ double get() const { return (double)hi + (double)lo; }
};

__device__ __forceinline__ int leaf_max_count_m(int cnt) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt = max(cnt, __shfl_xor_sync(0xffffffffu, cnt, o));
  return cnt;
}

__global__ void __launch_bounds__(128) k_density_mixed(HydroArgs a) {
  const int leaf = a.leaf0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (leaf >= a.leaf1) return;
  const int lane = (int)lane_id();
  const int s = leaf * kLeaf + lane;
  const bool valid = s < a.n;
  double4 pi = make_double4(0, 0, 0, 0), vi = make_double4(0, 0, 0, 0);
  int cnt = 0;
  if (valid) {
    pi = a.pos[s];
    vi = a.vel[s];
    cnt = min(a.n_ngb[s], a.cap);
  }
  const int kmax = leaf_max_count_m(cnt);
  const int *lst = a.list + (size_t)leaf * a.cap * kLeaf + lane;
  const double w = pi.w;
  const float iw2 = w > 0 ? (float)(2.0 / w) : 0.f;
  KSum dens, om, ps, sdig, div, cx, cy, cz;
  for (int k = 0; k < kmax; k++) {
    if (k < cnt) {
      const int j = __ldg(lst + (size_t)k * kLeaf);
      const double4 pj = ld4(a.pos + j), vj = ld4(a.vel + j);
      const float dx = (float)(pi.x - pj.x), dy = (float)(pi.y - pj.y), dz = (float)(pi.z - pj.z);
      const float u = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx))) * iw2;
      const float mj = (float)vj.w;
      dens.add(mj * k_w<float>(u));
      om.add(mj * k_dwdh<float>(u));
      ps.add(mj * k_dphidh<float>(u));
      sdig.add(-k_digdh<float>(u));
      const float dvx = (float)(vi.x - vj.x), dvy = (float)(vi.y - vj.y), dvz = (float)(vi.z - vj.z);
      const float wt = mj * k_dw<float>(u);
      div.add(wt * (dx * dvx + dy * dvy + dz * dvz));
      cx.add(wt * (dy * dvz - dz * dvy));
      cy.add(wt * (dz * dvx - dx * dvz));
      cz.add(wt * (dx * dvy - dy * dvx));
    }
  }
  if (!valid) return;
  double4 d = make_double4(0, 0, 0, 0);
  double rho = 0;
  if (w > 0 && cnt > 0) {
    const double h = 0.5 * w;
    const double h3 = h * h * h, h5 = h3 * h * h;
    double o = om.get(), p = ps.get(), sd = sdig.get(), de = dens.get();
    if (sd != 0) {
      o *= 1.0 / h3 / sd;
      p *= 1.0 / h / sd;
    } else {
      o = p = 0;
    }
    de *= 1.0 / h3;
    const double dv = div.get() / de / h5;
    const double X = cx.get(), Y = cy.get(), Z = cz.get();
    const double c = sqrt(X * X + Y * Y + Z * Z) / de / h5;
    rho = de;
    d = make_double4(dv, c, o, p);
  }
  a.hyd[s].x = rho;
  a.dd[s] = d;
}

__global__ void __launch_bounds__(128) k_hydro_mixed(HydroArgs a) {
  const int leaf = a.leaf0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (leaf >= a.leaf1) return;
  const int lane = (int)lane_id();
  const int s = leaf * kLeaf + lane;
  const bool valid = s < a.n;
  double4 pi = make_double4(0, 0, 0, 0), vi = make_double4(0, 0, 0, 1), hi4 = make_double4(0, 0, 0, 0),
          di = make_double4(0, 0, 0, 0);
  int cnt = 0;
  if (valid) {
    pi = a.pos[s];
    vi = a.vel[s];
    hi4 = a.hyd[s];
    di = a.dd[s];
    cnt = min(a.n_ngb[s], a.cap);
  }
  const int kmax = leaf_max_count_m(cnt);
  const int *lst = a.list + (size_t)leaf * a.cap * kLeaf + lane;
  const float hh = (float)(0.5 * pi.w);
  const float ihh = pi.w > 0 ? (float)(2.0 / pi.w) : 0.f;
  const float prho2 = (hi4.x > 0) ? (float)(hi4.y / (hi4.x * hi4.x)) : 0.f;
  const float ih2 = ihh * ihh, ih5 = ih2 * ih2 * ihh;
  const float om_i = (float)di.z;
  const float psi_i = a.use_psi ? (float)di.w : 0.f;
  const float gam = (float)a.gamma, alpha = (float)a.alpha, beta = (float)a.beta;
  const float ci = hi4.x > 0 ? sqrtf(gam * (float)hi4.y / (float)hi4.x) : 0.f;
  const float absdiv_i = fabsf((float)di.x);
  const float bal_i = absdiv_i / (absdiv_i + (float)di.y + 0.0001f * ci / hh);
  const float mi = (float)vi.w;
  KSum ax, ay, az, ud;
  float vmax = 0.f;
  for (int k = 0; k < kmax; k++) {
    if (k < cnt) {
      const int j = __ldg(lst + (size_t)k * kLeaf);
      const double4 pj = ld4(a.pos + j), vj = ld4(a.vel + j), hj = ld4(a.hyd + j), dj = ld4(a.dd + j);
      const float dx = (float)(pi.x - pj.x), dy = (float)(pi.y - pj.y), dz = (float)(pi.z - pj.z);
      const float dvx = (float)(vi.x - vj.x), dvy = (float)(vi.y - vj.y), dvz = (float)(vi.z - vj.z);
      const float ds = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
      const float u = ds * ihh;
      const float drdv = fmaf(dz, dvz, fmaf(dy, dvy, dx * dvx));
      // artificial viscosity, dev_art_visc.cu:8-32
      const float rhoj = (float)hj.x, Pj = (float)hj.y;
      const float cj = sqrtf(gam * Pj / rhoj);
      float visc = 0.f, vs = ci + cj;
      if (drdv < 0.f) {
        vs -= beta * drdv / ds;
        float mu = drdv / ((ci + cj) * ds);
        const float absdiv_j = fabsf((float)dj.x);
        const float bal_j = absdiv_j / (absdiv_j + (float)dj.y + 0.0001f * cj / (0.5f * (float)pj.w));
        mu *= (bal_i + bal_j);
        visc = (prho2 + Pj / (rhoj * rhoj)) * (-alpha * mu + beta * mu * mu);
      }
      vmax = fmaxf(vmax, vs);
      const float dwu = k_dw<float>(u), digu = k_dig<float>(u);
      const float mj = (float)vj.w;
      float acc = (prho2 + 0.5f * visc) * dwu * ih5;
      acc -= (prho2 * om_i + 0.5f * psi_i) / mj * digu * ih2;
      ax.add(-mj * acc * dx);
      ay.add(-mj * acc * dy);
      az.add(-mj * acc * dz);
      const float nacc = mi * acc;
      if (a.jside && j != s) {
        atomicAdd(&a.dots[j].x, (double)(nacc * dx));
        atomicAdd(&a.dots[j].y, (double)(nacc * dy));
        atomicAdd(&a.dots[j].z, (double)(nacc * dz));
      }
      float u1 = mj * (prho2 + 0.5f * visc) * dwu * ih5;
      u1 -= prho2 * om_i * digu * ih2;
      ud.add(u1 * drdv);
    }
  }
  if (!valid) return;
  atomicAdd(&a.dots[s].x, ax.get());
  atomicAdd(&a.dots[s].y, ay.get());
  atomicAdd(&a.dots[s].z, az.get());
  a.dots[s].w = ud.get();
  a.vsig[s] = (double)vmax;
}

int launch_density_mixed(const HydroArgs &a, cudaStream_t st) {
  if (a.leaf1 <= a.leaf0) return 0;
  k_density_mixed<<<((a.leaf1 - a.leaf0) * 32 + 127) / 128, 128, 0, st>>>(a);
  return 1;
}
int launch_hydro_mixed(const HydroArgs &a, cudaStream_t st) {
  if (a.leaf1 <= a.leaf0) return 0;
  k_hydro_mixed<<<((a.leaf1 - a.leaf0) * 32 + 127) / 128, 128, 0, st>>>(a);
  return 1;
}

}  // namespace sph
