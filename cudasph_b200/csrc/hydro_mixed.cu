// hydro_mixed.cu -- the mixed-precision form of the density and hydro loops.
//
// Neighbour records are gathered as in the FP64 form; the pair separation
// and velocity difference are formed in FP64 (exact differences of the FP64
// coordinates, rounded once), and everything that varies per pair -- the
// distance, u, the kernel functions, the artificial viscosity and the pair
// vectors -- runs in FP32 with compensated (Kahan-Babuska) float sums.  The
// factors that are constant over a particle's pairs (1/h^5, 1/h^2, P/rho^2,
// the grad-h terms, m_i) are applied in FP64 to those sums, and u = r (2 /
// range) takes the per-particle scale as a float-float pair: rounding such a
// constant to FP32 would bias every pair of that particle the same way, and
// in near-hydrostatic stars, where the pair forces largely cancel, such a
// bias (unlike the random per-pair rounding) grows into the net force.  The
// j-side pair force is assembled in FP64 from the FP32 pair vectors and the
// owner's FP64 factors; outputs and atomics stay FP64.
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

// x (hi + lo) for a float-float constant: the product to about 2^-46
__device__ __forceinline__ float mul_ff(float x, float hi, float lo) { return fmaf(x, hi, x * lo); }

__device__ __forceinline__ void split_ff(double v, float &hi, float &lo) {
  hi = (float)v;
  lo = (float)(v - (double)hi);
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
  float iw_hi = 0.f, iw_lo = 0.f;  // 2 / range as a float-float pair
  if (w > 0) split_ff(2.0 / w, iw_hi, iw_lo);
  KSum dens, om, ps, sdig, div, cx, cy, cz;
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
      const float dx = (float)(pi.x - pj.x), dy = (float)(pi.y - pj.y), dz = (float)(pi.z - pj.z);
      const float u = mul_ff(sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx))), iw_hi, iw_lo);
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
  if (a.dsum) a.dsum[s] = make_double4(sdig.get(), cx.get(), cy.get(), cz.get());
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

// Hydro (dev_hydro_dots.cu:25-113 with dev_art_visc.cu:8-32): with
// A = P_i / rho_i^2 the i-side force is
//   a_i = -[A S1 + S2 / 2] / h^5 + K [S3] / h^2,  K = A omega_i + psi_i / 2,
//   S1 = sum_j m_j dw(u) r_ij,  S2 = sum_j m_j Pi_ij dw(u) r_ij,
//   S3 = sum_j dig(u) r_ij,
// du_i/dt = [A T1 + T2 / 2] / h^5 - A omega_i T3 / h^2 with the same sums of
// r_ij . v_ij in place of r_ij; the pair's force on j, m_i acc_ij (r_i - r_j),
// is assembled in FP64 from the FP32 pair vectors dw r_ij, Pi dw r_ij, dig r_ij.
__global__ void __launch_bounds__(128) k_hydro_mixed(HydroArgs a) {
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
  const int kmax = leaf_max_count_m(cnt);
  const int *lst = a.list + (size_t)leaf * a.cap * kLeaf + lane;
  const double hh = 0.5 * pi.w;
  float ih_hi = 0.f, ih_lo = 0.f;  // 1 / h as a float-float pair
  if (hh > 0) split_ff(1.0 / hh, ih_hi, ih_lo);
  const double prho2 = (hi4.x > 0) ? hi4.y / (hi4.x * hi4.x) : 0;
  const double h2 = hh * hh, h5 = h2 * h2 * hh;
  const double ih5 = hh > 0 ? 1.0 / h5 : 0.0, ih2 = hh > 0 ? 1.0 / h2 : 0.0;
  const double psi_i = a.use_psi ? di.w : 0;
  const double K = prho2 * di.z + 0.5 * psi_i;
  // the owner's factors of the j-side force m_i acc_ij (FP64)
  const double mi = vi.w;
  const double c1 = mi * prho2 * ih5, c2 = 0.5 * mi * ih5, c3 = mi * K * ih2;
  const float alpha = (float)a.alpha, beta = (float)a.beta;
  const float ci = (float)fi.x, pr_i = (float)fi.y, bal_i = (float)fi.z;
  KSum s1x, s1y, s1z, s2x, s2y, s2z, s3x, s3y, s3z, t1, t2, t3;
  float vmax = 0.f;
  for (int k = 0; k < kmax; k++) {
    if (k < cnt) {
      const int j = __ldg(lst + (size_t)k * kLeaf);
      const double4 pj = ld4(a.pos + j), vj = ld4(a.vel + j), fj = ld4(a.aux + j);
      const float dx = (float)(pi.x - pj.x), dy = (float)(pi.y - pj.y), dz = (float)(pi.z - pj.z);
      const float dvx = (float)(vi.x - vj.x), dvy = (float)(vi.y - vj.y), dvz = (float)(vi.z - vj.z);
      const float ds = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
      const float u = mul_ff(ds, ih_hi, ih_lo);
      const float drdv = fmaf(dz, dvz, fmaf(dy, dvy, dx * dvx));
      // artificial viscosity on the per-particle factors {c, P / rho^2, B}
      const float cj = (float)fj.x;
      float visc = 0.f, vs = ci + cj;
      if (drdv < 0.f) {
        const float mu0 = drdv / ds;
        vs -= beta * mu0;
        const float mu = mu0 / (ci + cj) * (bal_i + (float)fj.z);
        visc = (pr_i + (float)fj.y) * (-alpha * mu + beta * mu * mu);
      }
      vmax = fmaxf(vmax, vs);
      const float dwu = k_dw<float>(u), digu = k_dig<float>(u);
      const float mj = (float)vj.w;
      const float mdw = mj * dwu, mpdw = visc * mdw;
      const float e1x = mdw * dx, e1y = mdw * dy, e1z = mdw * dz;     // m_j dw r_ij
      const float e2x = mpdw * dx, e2y = mpdw * dy, e2z = mpdw * dz;  // m_j Pi dw r_ij
      const float e3x = digu * dx, e3y = digu * dy, e3z = digu * dz;  // dig r_ij
      s1x.add(e1x); s1y.add(e1y); s1z.add(e1z);
      s2x.add(e2x); s2y.add(e2y); s2z.add(e2z);
      s3x.add(e3x); s3y.add(e3y); s3z.add(e3z);
      t1.add(mdw * drdv);
      t2.add(mpdw * drdv);
      t3.add(digu * drdv);
      if (a.jside && j != s) {
        // m_i acc_ij r_ij = [c1 m_j dw r + c2 m_j Pi dw r] / m_j - c3 dig r / m_j
        const double imj = fj.w;
        const double f1 = c1 * imj, f2 = c2 * imj, f3 = c3 * imj;
        atomicAdd(&a.dots[j].x, f1 * e1x + f2 * e2x - f3 * e3x);
        atomicAdd(&a.dots[j].y, f1 * e1y + f2 * e2y - f3 * e3y);
        atomicAdd(&a.dots[j].z, f1 * e1z + f2 * e2z - f3 * e3z);
      }
    }
  }
  if (!valid) return;
  atomicAdd(&a.dots[s].x, -(prho2 * s1x.get() + 0.5 * s2x.get()) * ih5 + K * ih2 * s3x.get());
  atomicAdd(&a.dots[s].y, -(prho2 * s1y.get() + 0.5 * s2y.get()) * ih5 + K * ih2 * s3y.get());
  atomicAdd(&a.dots[s].z, -(prho2 * s1z.get() + 0.5 * s2z.get()) * ih5 + K * ih2 * s3z.get());
  a.dots[s].w = (prho2 * t1.get() + 0.5 * t2.get()) * ih5 - prho2 * di.z * ih2 * t3.get();
  a.vsig[s] = (double)vmax;
}

int launch_density_mixed(const HydroArgs &a, cudaStream_t st) {
  if (a.leaf1 <= a.leaf0) return 0;
  k_density_mixed<<<((a.leaf1 - a.leaf0) * 32 + 127) / 128, 128, 0, st>>>(a);
  return 1;
}
int launch_hydro_prep(int n, const double4 *pos, const double4 *vel, const double4 *hyd, const double4 *dd,
                      double gamma, double4 *aux, cudaStream_t st);

int launch_hydro_mixed(const HydroArgs &a, cudaStream_t st) {
  if (a.leaf1 <= a.leaf0) return 0;
  // every particle's factors {c, P / rho^2, B, 1 / m}: a shard's pairs reach outside its own leaves
  int launches = launch_hydro_prep(a.n, a.pos, a.vel, a.hyd, a.dd, a.gamma, a.aux, st);
  k_hydro_mixed<<<((a.leaf1 - a.leaf0) * 32 + 127) / 128, 128, 0, st>>>(a);
  return launches + 1;
}

}  // namespace sph
