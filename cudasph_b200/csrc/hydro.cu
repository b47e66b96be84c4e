// hydro.cu -- FP64 density loop (dev_density_loop.cu:29-111), EOS
// (dev_compute_pressure.cu:3-111), hydro derivatives with Monaghan artificial
// viscosity (dev_hydro_dots.cu:25-113, dev_art_visc.cu:8-32) and the j-side
// pair force (add_ngb_acc, sph_accelerations.cpp:106-114).
//
// One warp per leaf, one lane per particle.  The neighbour list of lane l is
// read from the leaf-sliced layout, so entry k of all 32 lanes is one
// coalesced 128-byte load; neighbour records (double4 pos / vel / hydro /
// dots_data) are gathered with 16-byte loads and mostly hit L1/L2 because
// neighbours are Morton-close.  The j-side force of each pair is added to
// the neighbour with an FP64 atomic (red.global.add.f64), which keeps the
// pair force antisymmetric (momentum conserving) without a transposed list.
//
// The pair loops run with FMA contraction and one reciprocal square root per
// pair (distance, 1/distance and 1/u from it) instead of a square root and
// three or four divisions; the kernel polynomials of a pair are evaluated in
// one branch on u.  They differ from an FP64 CPU evaluation of the
// reference's formulas by rounding only (parity bounds: density 1e-12,
// hydro 1e-10 relative).  The h solve (neighbours.cu), whose ranges must
// match such an evaluation bit for bit, keeps the reference's operation order.
#include "common.cuh"
#include "sph_math.cuh"

namespace sph {

// the distance r and 1 / r of a pair from its squared distance; the self
// pair (d2 = 0) gets r = 1 / r = 0 (its terms multiply a zero vector or
// take the u = 0 branch)
__device__ __forceinline__ void dist_and_inverse(double d2, double &r, double &ir) {
  ir = d2 > 0 ? rsqrt(d2) : 0.0;
  r = d2 * ir;
}

// M4 kernel values of the density loop at u = 2 r / range (dev_sph_kernels.cu:
// 7-99): w, dW/dh term, dphi/dh term and dw = (1/u) dW/du in one branch; iu = 1/u
struct DensityKernels {
  double w, dwdh, dphidh, dw;
};

__device__ __forceinline__ DensityKernels density_kernels(double u, double iu) {
  constexpr double ipi = KC<double>::ipi;
  DensityKernels k;
  const double u2 = u * u, u3 = u2 * u;
  if (u < 1) {
    k.w = ipi * (1.0 - 1.5 * u2 + 0.75 * u3);
    k.dwdh = ipi * (-3.0 + 7.5 * u2 - 4.5 * u3);
    k.dphidh = 1.4 - 2.0 * u2 + 1.5 * u2 * u2 - 0.6 * u2 * u3;
    k.dw = ipi * (-3.0 + 2.25 * u);
  } else if (u < 2) {
    const double t = 2.0 - u;
    k.w = ipi * 0.25 * t * t * t;
    k.dwdh = ipi * (-6.0 + 12.0 * u - 7.5 * u2 + 1.5 * u3);
    k.dphidh = 1.6 - 4.0 * u2 + 4.0 * u3 - 1.5 * u2 * u2 + 0.2 * u2 * u3;
    k.dw = -ipi * 0.75 * t * t * iu;
  } else {
    k.w = k.dwdh = k.dphidh = k.dw = 0.0;
  }
  return k;
}

// u d(ig)/du (k_digdh) and (1/u) d(ig)/du (k_dig) share 4 pi x^2 w(x) at
// x = 4u (u < 1) or x = 4 (2 - u) (1 <= u < 2); w(x) vanishes for x >= 2
__device__ __forceinline__ double ig_slope_core(double u, double &sign) {
  constexpr double ipi = KC<double>::ipi, pi4 = 4.0 * KC<double>::pi;
  double x;
  if (u < 1) {
    x = 4.0 * u;
    sign = 4.0;
  } else {
    x = 4.0 * (2.0 - u);
    sign = -4.0;
  }
  double wx;
  if (x < 1) wx = ipi * (1.0 - 1.5 * x * x + 0.75 * x * x * x);
  else if (x < 2) wx = ipi * 0.25 * (2.0 - x) * (2.0 - x) * (2.0 - x);
  else wx = 0.0;
  return pi4 * x * x * wx;
}

__device__ __forceinline__ double ig_digdh(double u) {
  if (!(u > 0) || !(u < 2)) return 0.0;
  double sign;
  const double d = ig_slope_core(u, sign);
  return sign * u * d;
}

__device__ __forceinline__ double ig_dig(double u, double iu) {
  if (!(u > 0) || !(u < 2)) return 0.0;
  double sign;
  const double d = ig_slope_core(u, sign);
  return sign * iu * d;
}

// (1/u) dW/du for hydro at u = r / h
__device__ __forceinline__ double kernel_dw(double u, double iu) {
  constexpr double ipi = KC<double>::ipi;
  if (u < 1) return ipi * (-3.0 + 2.25 * u);
  if (u < 2) {
    const double t = 2.0 - u;
    return -ipi * 0.75 * t * t * iu;
  }
  return 0.0;
}


__device__ __forceinline__ int leaf_max_count(int cnt) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt = max(cnt, __shfl_xor_sync(0xffffffffu, cnt, o));
  return cnt;
}

__global__ void __launch_bounds__(128) k_density(HydroArgs a) {
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
  const int kmax = leaf_max_count(cnt);
  const int *lst = a.list + (size_t)leaf * a.cap * kLeaf + lane;
  const double w = pi.w;
  const double i2w = 2.0 / w, hw = 0.5 * w;  // u = r (2 / range), 1 / u = (1 / r) (range / 2)
  double dens = 0, om = 0, ps = 0, sdig = 0, div = 0, cx = 0, cy = 0, cz = 0;
  // the neighbours' records are gathered one pair ahead of their use and
  // the list entries two ahead, so the loads overlap the pair arithmetic
  int jn = cnt > 1 ? __ldg(lst + kLeaf) : 0;
  double4 pn = make_double4(0, 0, 0, 0), vn = pn;
  if (cnt > 0) {
    const int j0 = __ldg(lst);
    pn = ld4(a.pos + j0);
    vn = ld4(a.vel + j0);
  }
  for (int k = 0; k < kmax; k++) {
    if (k < cnt) {
      const double4 pj = pn, vj = vn;
      if (k + 1 < cnt) {
        pn = ld4(a.pos + jn);
        vn = ld4(a.vel + jn);
        if (k + 2 < cnt) jn = __ldg(lst + (size_t)(k + 2) * kLeaf);
      }
      const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
      double r, ir;
      dist_and_inverse(dx * dx + dy * dy + dz * dz, r, ir);
      const double u = r * i2w;
      const DensityKernels kv = density_kernels(u, ir * hw);
      const double mj = vj.w;
      dens += mj * kv.w;
      om += mj * kv.dwdh;
      ps += mj * kv.dphidh;
      sdig -= ig_digdh(u);
      const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
      const double wt = mj * kv.dw;
      div += wt * (dx * dvx + dy * dvy + dz * dvz);
      cx += wt * (dy * dvz - dz * dvy);
      cy += wt * (dz * dvx - dx * dvz);
      cz += wt * (dx * dvy - dy * dvx);
    }
  }
  if (!valid) return;
  if (a.dsum) a.dsum[s] = make_double4(sdig, cx, cy, cz);
  double4 d = make_double4(0, 0, 0, 0);
  double rho = 0;
  if (w > 0 && cnt > 0) {
    const double h = 0.5 * w;
    const double h3 = h * h * h, h5 = h3 * h * h;
    if (sdig != 0) {
      om *= 1.0 / h3 / sdig;
      ps *= 1.0 / h / sdig;
    } else {
      om = ps = 0;
    }
    dens *= 1.0 / h3;
    div *= 1.0 / dens / h5;
    const double c = sqrt(cx * cx + cy * cy + cz * cz) / dens / h5;
    rho = dens;
    d = make_double4(div, c, om, ps);
  }
  a.hyd[s].x = rho;
  a.dd[s] = d;
}

// ---------------------------------------------------------------------------
// EOS.  The temperature solves u = u_gas(T) + u_rad(T), i.e. the quartic
// x^4 + q x + r = 0 in x = T / 1e6 with q > 0, r < 0 (the units and constants
// of dev_compute_pressure.cu:55-96).  On x > 0, f(x) = x^4 + q x + r is
// increasing and convex with one root, and both -r/q and (-r)^(1/4) lie at
// or above it (f is non-negative there), so Newton's method started from the
// smaller of the two decreases monotonically onto the root: it stops when a
// step no longer decreases x.  Over the density and energy range of the
// workloads (rho 1e-6 .. 1e4, u 1e-8 .. 1e3 in code units) it takes at most
// six steps and agrees with the closed form of the reference polished by
// Newton to 1.5 ulp.
// ---------------------------------------------------------------------------
constexpr double kDensityUnit = 5.89994031541978;     // dev_compute_pressure.cu:57-58
constexpr double kEnergyUnit = 1.90698842928778e+15;  // :61-62
constexpr double kPressureUnit = 1.1251117914994e+16; // :65-66
constexpr double kAmu = 1.66054e-24;                   // :69-70
constexpr double kBoltzmann = 1.380658e-16;            // :73-74
constexpr double kRadConst = 7.56591414984829e-15;     // :77-78

__device__ double quartic_root(double q, double r) {
  double x = fmin(-r / q, sqrt(sqrt(-r)));
  for (int it = 0; it < 64; it++) {
    const double x3 = x * x * x;
    const double xn = x - (x3 * x + q * x + r) / (4.0 * x3 + q);
    if (!(xn < x)) break;
    x = xn;
  }
  return x;
}

__device__ __forceinline__ double pressure_of(double rho, double u, double mu, int eos_mode, double gamma) {
  if (eos_mode == SPH_EOS_IDEAL) return (gamma - 1) * rho * u;
  if (!(rho > 0) || !(mu > 0)) return 0;
  const double density = rho * kDensityUnit;
  const double energy = u * kEnergyUnit;
  const double mean_mu = mu * kAmu;
  const double tb = 1.0e6;
  const double r = -density * (energy / (tb * tb)) / (kRadConst * tb * tb);
  const double q = (kBoltzmann / kRadConst) / (gamma - 1) * density / (((mean_mu * tb) * tb) * tb);
  const double T = tb * quartic_root(q, r);
  const double pg = density * ((kBoltzmann * T) / mean_mu);
  const double pr = (((kRadConst / 3.0 * T) * T) * T) * T;
  return (pg + pr) / kPressureUnit;
}

__global__ void k_pressure(int n, double4 *__restrict__ hyd, int eos_mode, double gamma, unsigned *flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 h = hyd[i];
  const double P = pressure_of(h.x, h.z, h.w, eos_mode, gamma);
  if (!isfinite(P)) raise_flag(flags, SPH_FLAG_NONFINITE);
  hyd[i].y = P;
}

// The factors of dev_art_visc.cu:8-32 that depend on one particle only --
// sound speed c = sqrt(gamma P / rho), P / rho^2 and the Balsara factor
// |div| / (|div| + |curl| + 1e-4 c / h) -- computed once per particle with
// the same operations the pair formula applies to them, and 1 / m, so the
// pair loop gathers one record {c, P / rho^2, B, 1 / m} per neighbour instead
// of hyd and dd and computes neither square root nor division per pair.
__global__ void k_hydro_prep(int n, const double4 *__restrict__ pos, const double4 *__restrict__ vel,
                             const double4 *__restrict__ hyd, const double4 *__restrict__ dd, double gamma,
                             double4 *__restrict__ aux) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double range = pos[i].w;
  const double4 h = hyd[i], d = dd[i];
  const double c = sqrt(gamma * h.y / h.x);
  const double b = fabs(d.x) / (fabs(d.x) + d.y + 0.0001 * c / (0.5 * range));
  aux[i] = make_double4(c, h.y / (h.x * h.x), b, 1.0 / vel[i].w);
}

// dev_art_visc.cu:8-32 on the per-particle factors of k_hydro_prep
// (ids = 1 / |r_ij|)
__device__ __forceinline__ void art_visc_pre(double ids, double drdv, const double4 &fi, const double4 &fj,
                                             double alpha, double beta, double &visc, double &vsig) {
  double av = 0, vs = fi.x + fj.x;
  if (drdv < 0) {
    const double mu = drdv * ids;  // the approach speed along the pair
    vs -= beta * mu;
    av = mu / (fi.x + fj.x);
    av *= (fi.z + fj.z);
    av = (fi.y + fj.y) * (-alpha * av + beta * av * av);
  }
  visc = av;
  vsig = vs;
}

// hydro_dots (dev_hydro_dots.cu:25-113) plus the j-side of every pair.
// dots must be zero on entry (xyz accumulate); dots.w (du/dt) is stored.
// 4 blocks per SM: the one-pair-ahead gathers need the registers (N = 1M:
// 2.40 ms without them at 6 blocks per SM, 2.99 ms with them and spills at
// 6, 1.89 ms with them at 4)
__global__ void __launch_bounds__(128, 4) k_hydro(HydroArgs a) {
  const int leaf = a.leaf0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (leaf >= a.leaf1) return;
  const int lane = (int)lane_id();
  const int s = leaf * kLeaf + lane;
  const bool valid = s < a.n;
  double4 pi = make_double4(0, 0, 0, 0), vi = make_double4(0, 0, 0, 1), hi4 = make_double4(0, 0, 0, 0),
          di = make_double4(0, 0, 0, 0), fi = make_double4(0, 0, 0, 0);
  int cnt = 0;
  if (valid) {
    pi = a.pos[s];
    vi = a.vel[s];
    hi4 = a.hyd[s];
    di = a.dd[s];
    fi = a.aux[s];
    cnt = min(a.n_ngb[s], a.cap);
  }
  const int kmax = leaf_max_count(cnt);
  const int *lst = a.list + (size_t)leaf * a.cap * kLeaf + lane;
  const double hh = 0.5 * pi.w;
  const double prho2 = (hi4.x > 0) ? hi4.y / (hi4.x * hi4.x) : 0;
  const double h2 = hh * hh, h5 = h2 * h2 * hh;
  const double psi_i = a.use_psi ? di.w : 0;
  // per-particle reciprocals and factors: the pair loop divides only by the
  // neighbour's mass (and, in compression, by ds and c_i + c_j)
  const double ihh = 1.0 / hh, ih5 = 1.0 / h5;
  const double gi = (prho2 * di.z + 0.5 * psi_i) / h2;  // grad-h term of the force
  const double ei = prho2 * di.z / h2;                   // grad-h term of du/dt
  double axi = 0, ayi = 0, azi = 0, udot = 0, vmax = 0;
  // the neighbours' records are gathered one pair ahead of their use and the
  // list entries two ahead (as in the density loop)
  int jn = cnt > 1 ? __ldg(lst + kLeaf) : 0, jc = cnt > 0 ? __ldg(lst) : 0;
  double4 pn = make_double4(0, 0, 0, 0), vn = pn, fn = pn;
  if (cnt > 0) {
    pn = ld4(a.pos + jc);
    vn = ld4(a.vel + jc);
    fn = ld4(a.aux + jc);
  }
  for (int k = 0; k < kmax; k++) {
    if (k < cnt) {
      const int j = jc;
      const double4 pj = pn, vj = vn, fj = fn;
      if (k + 1 < cnt) {
        jc = jn;
        pn = ld4(a.pos + jn);
        vn = ld4(a.vel + jn);
        fn = ld4(a.aux + jn);
        if (k + 2 < cnt) jn = __ldg(lst + (size_t)(k + 2) * kLeaf);
      }
      const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
      const double dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
      double ds, ids;
      dist_and_inverse(dx * dx + dy * dy + dz * dz, ds, ids);
      const double u = ds * ihh, iu = ids * hh;
      const double drdv = dx * dvx + dy * dvy + dz * dvz;
      double visc, vs;
      art_visc_pre(ids, drdv, fi, fj, a.alpha, a.beta, visc, vs);
      if (vs > vmax) vmax = vs;
      const double dwu = kernel_dw(u, iu), digu = ig_dig(u, iu);
      const double mj = vj.w;
      const double ta = (prho2 + 0.5 * visc) * dwu * ih5;
      const double acc = ta - gi * digu * fj.w;  // fj.w = 1 / m_j
      axi -= mj * acc * dx;
      ayi -= mj * acc * dy;
      azi -= mj * acc * dz;
      const double nacc = vi.w * acc;
      if (a.ngb_acc) a.ngb_acc[(size_t)leaf * a.cap * kLeaf + (size_t)k * kLeaf + lane] = nacc;
      if (a.jside && j != s) {
        atomicAdd(&a.dots[j].x, nacc * dx);
        atomicAdd(&a.dots[j].y, nacc * dy);
        atomicAdd(&a.dots[j].z, nacc * dz);
      }
      const double ud = mj * ta - ei * digu;
      udot += ud * drdv;
    }
  }
  if (!valid) return;
  atomicAdd(&a.dots[s].x, axi);
  atomicAdd(&a.dots[s].y, ayi);
  atomicAdd(&a.dots[s].z, azi);
  a.dots[s].w = udot;
  a.vsig[s] = vmax;
}

int launch_density(const HydroArgs &a, cudaStream_t st) {
  if (a.leaf1 <= a.leaf0) return 0;
  k_density<<<((a.leaf1 - a.leaf0) * 32 + 127) / 128, 128, 0, st>>>(a);
  return 1;
}
int launch_pressure(int n, double4 *hyd, int eos_mode, double gamma, unsigned *flags, cudaStream_t st) {
  k_pressure<<<(n + 255) / 256, 256, 0, st>>>(n, hyd, eos_mode, gamma, flags);
  return 1;
}
int launch_hydro_prep(int n, const double4 *pos, const double4 *vel, const double4 *hyd, const double4 *dd,
                      double gamma, double4 *aux, cudaStream_t st) {
  if (n <= 0) return 0;
  k_hydro_prep<<<(n + 255) / 256, 256, 0, st>>>(n, pos, vel, hyd, dd, gamma, aux);
  return 1;
}

int launch_hydro(const HydroArgs &a, cudaStream_t st) {
  if (a.leaf1 <= a.leaf0) return 0;
  // every particle's factors: a shard's pairs reach outside its own leaves
  int launches = launch_hydro_prep(a.n, a.pos, a.vel, a.hyd, a.dd, a.gamma, a.aux, st);
  k_hydro<<<((a.leaf1 - a.leaf0) * 32 + 127) / 128, 128, 0, st>>>(a);
  return launches + 1;
}

}  // namespace sph
