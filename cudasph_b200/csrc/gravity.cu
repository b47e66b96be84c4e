// gravity.cu -- softened direct-N self-gravity (sph_grav_kernel.cu:14-195).
//
// Each block owns an i-tile of kThreads * R consecutive (Morton-ordered)
// particles, R per thread held in registers; the sources stream through
// shared memory in j-tiles of kThreads records, each record read once per
// block and broadcast to the R i-particles of every thread.  The inner loop
// runs on the FP64 pipe (plain form) or on the FP32 FMA pipe (mixed form).
//
// Mixed form: all positions of a block are taken relative to an FP64 anchor
// (the first particle of the i-tile) and rounded to FP32 once per j per
// block, so a close pair keeps the relative accuracy of FP32 on its small
// separation.  Each thread sums a j-tile's contributions in FP32 and folds
// the tile partial into a compensated (Kahan-Babuska) float-float
// accumulator, the counterpart of the reference's float-float `dreal`
// accumulation (dreal.h:4-127).
//
// Softening: Plummer (r^2 + eps^2) or the reference's M4-spline softening at
// the smoothing ranges of i and j with half contributions
// (sph_grav_kernel.cu:32-105); the spline branch is taken only by pairs
// closer than max(range_i, range_j), so warps almost never diverge on it.
//
// Reciprocal square roots: FP32 uses rsqrt.approx.ftz.f32.  FP64 has no
// full-precision hardware rsqrt; it is seeded with rsqrt.approx.ftz.f64 and
// refined by one third-order Householder step for 1/sqrt
// (y = y0 (1 + e/2 + 3 e^2 / 8), e = 1 - r2 y0^2), checked against
// 1/sqrt(r2) to a few ulp by the test suite.
#include "common.cuh"
#include "pairmath.cuh"

namespace sph {

constexpr int kGThreads = 128;


// reference spline softening polynomials, sph_grav_kernel.cu:53-61
template <class R>
__device__ __forceinline__ void spline_poly(R u, R u2, R &gacc, R &gpot) {
  const R u3 = u2 * u;
  if (u < (R)0.5) {
    gacc = (R)10.666666666667 + u2 * ((R)32.0 * u - (R)38.4);
    gpot = (R)(-2.8) + u2 * ((R)5.333333333333 + u2 * ((R)6.4 * u - (R)9.6));
  } else {
    gacc = (R)21.333333333333 - (R)48.0 * u + (R)38.4 * u2 - (R)10.666666666667 * u3 - (R)0.066666666667 / u3;
    gpot = (R)(-3.2) + (R)0.066666666667 / u + u2 * ((R)10.666666666667 + u * ((R)(-16.0) + u * ((R)9.6 - (R)2.133333333333 * u)));
  }
}

template <class R>
__device__ __forceinline__ R rsq(R x);
template <>
__device__ __forceinline__ float rsq<float>(float x) { return rsqrt_f32(x); }
template <>
__device__ __forceinline__ double rsq<double>(double x) { return rsqrt_f64(x); }

// The near-field pair of the spline mode (r < max(range_i, range_j)),
// bodyBodyInteraction's else-branch, sph_grav_kernel.cu:40-106.
// dx = x_j - x_i; accumulates acceleration into a (a += contribution).
template <class R>
__device__ __noinline__ void spline_near(R dx, R dy, R dz, R r2, R mj, R hi2, R hj2, R &ax, R &ay, R &az, R &pot) {
  R inv = r2 > 0 ? rsq<R>(r2) : (R)0;
  R s3h = (R)0.5 * mj * inv * inv * inv;
  R g;
  if (r2 < hi2) {
    const R u2 = r2 / hi2, h = sqrt(hi2), u = sqrt(u2);
    R ga, gp;
    spline_poly<R>(u, u2, ga, gp);
    g = (R)0.5 * mj * ga / (hi2 * h);
    pot += mj * gp / h;
  } else {
    g = s3h;
    pot -= mj * inv;
  }
  if (r2 < hj2) {
    const R u2 = r2 / hj2, h = sqrt(hj2), u = sqrt(u2);
    R ga, gp;
    spline_poly<R>(u, u2, ga, gp);
    g += (R)0.5 * mj * ga / (hj2 * h);
  } else {
    g += s3h;
  }
  ax = fma(dx, g, ax);
  ay = fma(dy, g, ay);
  az = fma(dz, g, az);
}

// -------------------------------- FP64 --------------------------------------
// One-sided form: every i of the block against the sources [jlo, jhi); with
// tile > 0 the range is the tile of `tile` particles that holds the block
// (the diagonal tiles of the symmetric form), else all n.
template <int SOFT, int R>
__global__ void __launch_bounds__(kGThreads) k_grav_f64(int n, const double4 *__restrict__ src,
                                                        const double *__restrict__ h2src, double4 *__restrict__ out,
                                                        double eps2, double G, int tile, int block0) {
  __shared__ double4 sj[kGThreads];
  __shared__ double sh[SOFT == SPH_SOFT_SPLINE ? kGThreads : 1];
  const int t = threadIdx.x;
  const int i0 = (blockIdx.x + block0) * kGThreads * R;
  const int jlo = tile > 0 ? (i0 / tile) * tile : 0;
  const int jhi = tile > 0 ? min(jlo + tile, n) : n;
  double xi[R], yi[R], zi[R], hi2[R], ax[R], ay[R], az[R], pot[R];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = min(i0 + r * kGThreads + t, n - 1);
    const double4 p = src[i];
    xi[r] = p.x; yi[r] = p.y; zi[r] = p.z;
    hi2[r] = (SOFT == SPH_SOFT_SPLINE) ? h2src[i] : 0.0;
    ax[r] = ay[r] = az[r] = pot[r] = 0.0;
  }
  for (int j0 = jlo; j0 < jhi; j0 += kGThreads) {
    const int j = j0 + t;
    __syncthreads();
    if (j < jhi) {
      sj[t] = src[j];
      if (SOFT == SPH_SOFT_SPLINE) sh[t] = h2src[j];
    }
    __syncthreads();
    const int m = min(kGThreads, jhi - j0);
    if (SOFT == SPH_SOFT_PLUMMER) {
#pragma unroll 4
      for (int k = 0; k < m; k++) {
        const double4 q = sj[k];
#pragma unroll
        for (int r = 0; r < R; r++) {
          const double dx = q.x - xi[r], dy = q.y - yi[r], dz = q.z - zi[r];
          const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
          const double inv = rsqrt_f64(r2);
          const double s = q.w * inv;
          const double s3 = s * inv * inv;
          ax[r] = fma(dx, s3, ax[r]);
          ay[r] = fma(dy, s3, ay[r]);
          az[r] = fma(dz, s3, az[r]);
          pot[r] -= s;
        }
      }
    } else {
      for (int k = 0; k < m; k++) {
        const double4 q = sj[k];
        const double hj2 = sh[k];
#pragma unroll
        for (int r = 0; r < R; r++) {
          const double dx = q.x - xi[r], dy = q.y - yi[r], dz = q.z - zi[r];
          const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
          if (r2 >= hi2[r] && r2 >= hj2) {
            if (r2 > 0) {
              const double inv = rsqrt_f64(r2);
              const double s = q.w * inv;
              const double s3 = s * inv * inv;
              ax[r] = fma(dx, s3, ax[r]);
              ay[r] = fma(dy, s3, ay[r]);
              az[r] = fma(dz, s3, az[r]);
              pot[r] -= s;
            }
          } else {
            spline_near<double>(dx, dy, dz, r2, q.w, hi2[r], hj2, ax[r], ay[r], az[r], pot[r]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = i0 + r * kGThreads + t;
    if (i < n) out[i] = make_double4(G * ax[r], G * ay[r], G * az[r], G * pot[r]);
  }
}

// ----------------------------- mixed (FP32) ---------------------------------
__device__ __forceinline__ void kahan_add(float &hi, float &lo, float v) {
  // Knuth TwoSum of (hi, v); the rounding error joins lo
  const float s = hi + v;
  const float bp = s - hi;
  const float err = (hi - (s - bp)) + (v - bp);
  hi = s;
  lo += err;
}

template <int SOFT, int R>
__global__ void __launch_bounds__(kGThreads) k_grav_f32(int n, const double4 *__restrict__ src,
                                                        const double *__restrict__ h2src, double4 *__restrict__ out,
                                                        float eps2, double G, int block0) {
  __shared__ float4 sj[kGThreads];
  __shared__ float sh[SOFT == SPH_SOFT_SPLINE ? kGThreads : 1];
  const int t = threadIdx.x;
  const int i0 = (blockIdx.x + block0) * kGThreads * R;
  const double4 anc = src[min(i0, n - 1)];
  float xi[R], yi[R], zi[R], hi2[R];
  float ahi[R][4], alo[R][4];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = min(i0 + r * kGThreads + t, n - 1);
    const double4 p = src[i];
    xi[r] = (float)(p.x - anc.x);
    yi[r] = (float)(p.y - anc.y);
    zi[r] = (float)(p.z - anc.z);
    hi2[r] = (SOFT == SPH_SOFT_SPLINE) ? (float)h2src[i] : 0.f;
#pragma unroll
    for (int c = 0; c < 4; c++) ahi[r][c] = alo[r][c] = 0.f;
  }
  for (int j0 = 0; j0 < n; j0 += kGThreads) {
    const int j = j0 + t;
    __syncthreads();
    if (j < n) {
      const double4 q = src[j];
      sj[t] = make_float4((float)(q.x - anc.x), (float)(q.y - anc.y), (float)(q.z - anc.z), (float)q.w);
      if (SOFT == SPH_SOFT_SPLINE) sh[t] = (float)h2src[j];
    }
    __syncthreads();
    const int m = min(kGThreads, n - j0);
    float px[R], py[R], pz[R], pp[R];
#pragma unroll
    for (int r = 0; r < R; r++) px[r] = py[r] = pz[r] = pp[r] = 0.f;
    if (SOFT == SPH_SOFT_PLUMMER) {
      if (m == kGThreads) {
#pragma unroll 8
        for (int k = 0; k < kGThreads; k++) {
          const float4 q = sj[k];
#pragma unroll
          for (int r = 0; r < R; r++) {
            const float dx = q.x - xi[r], dy = q.y - yi[r], dz = q.z - zi[r];
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
            const float inv = rsqrt_f32(r2);
            const float s = q.w * inv;
            const float s3 = s * inv * inv;
            px[r] = fmaf(dx, s3, px[r]);
            py[r] = fmaf(dy, s3, py[r]);
            pz[r] = fmaf(dz, s3, pz[r]);
            pp[r] -= s;
          }
        }
      } else {
        for (int k = 0; k < m; k++) {
          const float4 q = sj[k];
#pragma unroll
          for (int r = 0; r < R; r++) {
            const float dx = q.x - xi[r], dy = q.y - yi[r], dz = q.z - zi[r];
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
            const float inv = rsqrt_f32(r2);
            const float s = q.w * inv;
            const float s3 = s * inv * inv;
            px[r] = fmaf(dx, s3, px[r]);
            py[r] = fmaf(dy, s3, py[r]);
            pz[r] = fmaf(dz, s3, pz[r]);
            pp[r] -= s;
          }
        }
      }
    } else {
      for (int k = 0; k < m; k++) {
        const float4 q = sj[k];
        const float hj2 = sh[k];
#pragma unroll
        for (int r = 0; r < R; r++) {
          const float dx = q.x - xi[r], dy = q.y - yi[r], dz = q.z - zi[r];
          const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
          if (r2 >= hi2[r] && r2 >= hj2) {
            if (r2 > 0) {
              const float inv = rsqrt_f32(r2);
              const float s = q.w * inv;
              const float s3 = s * inv * inv;
              px[r] = fmaf(dx, s3, px[r]);
              py[r] = fmaf(dy, s3, py[r]);
              pz[r] = fmaf(dz, s3, pz[r]);
              pp[r] -= s;
            }
          } else {
            spline_near<float>(dx, dy, dz, r2, q.w, hi2[r], hj2, px[r], py[r], pz[r], pp[r]);
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
      kahan_add(ahi[r][0], alo[r][0], px[r]);
      kahan_add(ahi[r][1], alo[r][1], py[r]);
      kahan_add(ahi[r][2], alo[r][2], pz[r]);
      kahan_add(ahi[r][3], alo[r][3], pp[r]);
    }
  }
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = i0 + r * kGThreads + t;
    if (i < n)
      out[i] = make_double4(G * ((double)ahi[r][0] + (double)alo[r][0]), G * ((double)ahi[r][1] + (double)alo[r][1]),
                            G * ((double)ahi[r][2] + (double)alo[r][2]), G * ((double)ahi[r][3] + (double)alo[r][3]));
  }
}

// --------------------- mixed (FP32), packed f32x2 form ----------------------
// Plummer-softened mixed kernel on Blackwell's packed FP32 instructions
// (add/mul/fma.rn.f32x2): each instruction advances two i-particles against
// the same source, which halves the FP32 instruction count per interaction
// (13 packed + 2 MUFU per two interactions) and moves the loop from the
// warp-issue limit to the FMA-pipe limit.  Sources are stored in shared
// memory pre-duplicated ({x,x}, {y,y}, {z,z}, {m,m}) so a source costs two
// 16-byte shared loads per thread and no repacking.  Padding sources beyond n
// have m = 0 at the anchor; eps > 0 keeps their r^2 > 0, so every tile is a
// full tile.

// One-sided form: every i of the block against the sources [jlo, jhi); with
// tile > 0 the range is the tile of `tile` particles that holds the block
// (the diagonal tiles of the symmetric form), else all n.
template <int RP>  // i-particle pairs per thread
__global__ void __launch_bounds__(kGThreads) k_grav_f32x2_plummer(int n, const double4 *__restrict__ src,
                                                                  double4 *__restrict__ out, float eps2, double G,
                                                                  int tile, int block0) {
  __shared__ ulonglong2 sj[kGThreads][2];
  const int t = threadIdx.x;
  const int i0 = (blockIdx.x + block0) * kGThreads * 2 * RP;
  const int jlo = tile > 0 ? (i0 / tile) * tile : 0;
  const int jhi = tile > 0 ? min(jlo + tile, n) : n;
  const double4 anc = src[min(i0, n - 1)];
  f32x2 xi[RP], yi[RP], zi[RP];
  float ahi[2 * RP][4], alo[2 * RP][4];
#pragma unroll
  for (int p = 0; p < RP; p++) {
    const double4 a = src[min(i0 + (2 * p) * kGThreads + t, n - 1)];
    const double4 b = src[min(i0 + (2 * p + 1) * kGThreads + t, n - 1)];
    xi[p] = pk2((float)(a.x - anc.x), (float)(b.x - anc.x));
    yi[p] = pk2((float)(a.y - anc.y), (float)(b.y - anc.y));
    zi[p] = pk2((float)(a.z - anc.z), (float)(b.z - anc.z));
  }
#pragma unroll
  for (int r = 0; r < 2 * RP; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) ahi[r][c] = alo[r][c] = 0.f;
  const f32x2 e2 = pk2(eps2, eps2);
  for (int j0 = jlo; j0 < jhi; j0 += kGThreads) {
    const int j = j0 + t;
    __syncthreads();
    if (j < jhi) {
      const double4 q = src[j];
      const float x = (float)(q.x - anc.x), y = (float)(q.y - anc.y), z = (float)(q.z - anc.z), m = (float)q.w;
      sj[t][0] = make_ulonglong2(pk2(x, x), pk2(y, y));
      sj[t][1] = make_ulonglong2(pk2(z, z), pk2(m, m));
    } else {
      sj[t][0] = make_ulonglong2(0ull, 0ull);
      sj[t][1] = make_ulonglong2(0ull, 0ull);
    }
    __syncthreads();
    f32x2 px[RP], py[RP], pz[RP], pp[RP];
#pragma unroll
    for (int p = 0; p < RP; p++) px[p] = py[p] = pz[p] = pp[p] = 0ull;
#pragma unroll 4
    for (int k = 0; k < kGThreads; k++) {
      const ulonglong2 a = sj[k][0], b = sj[k][1];
#pragma unroll
      for (int p = 0; p < RP; p++) {
        const f32x2 dx = sub2(a.x, xi[p]), dy = sub2(a.y, yi[p]), dz = sub2(b.x, zi[p]);
        f32x2 r2 = fma2(dx, dx, e2);
        r2 = fma2(dy, dy, r2);
        r2 = fma2(dz, dz, r2);
        float r2a, r2b;
        upk2(r2, r2a, r2b);
        const f32x2 inv = pk2(rsqrt_f32(r2a), rsqrt_f32(r2b));
        const f32x2 inv2 = mul2(inv, inv);
        const f32x2 s = mul2(b.y, inv);
        const f32x2 s3 = mul2(s, inv2);
        px[p] = fma2(dx, s3, px[p]);
        py[p] = fma2(dy, s3, py[p]);
        pz[p] = fma2(dz, s3, pz[p]);
        pp[p] = sub2(pp[p], s);
      }
    }
#pragma unroll
    for (int p = 0; p < RP; p++) {
      float a0, a1;
      upk2(px[p], a0, a1);
      kahan_add(ahi[2 * p][0], alo[2 * p][0], a0);
      kahan_add(ahi[2 * p + 1][0], alo[2 * p + 1][0], a1);
      upk2(py[p], a0, a1);
      kahan_add(ahi[2 * p][1], alo[2 * p][1], a0);
      kahan_add(ahi[2 * p + 1][1], alo[2 * p + 1][1], a1);
      upk2(pz[p], a0, a1);
      kahan_add(ahi[2 * p][2], alo[2 * p][2], a0);
      kahan_add(ahi[2 * p + 1][2], alo[2 * p + 1][2], a1);
      upk2(pp[p], a0, a1);
      kahan_add(ahi[2 * p][3], alo[2 * p][3], a0);
      kahan_add(ahi[2 * p + 1][3], alo[2 * p + 1][3], a1);
    }
  }
#pragma unroll
  for (int r = 0; r < 2 * RP; r++) {
    const int i = i0 + r * kGThreads + t;
    if (i < n)
      out[i] = make_double4(G * ((double)ahi[r][0] + (double)alo[r][0]), G * ((double)ahi[r][1] + (double)alo[r][1]),
                            G * ((double)ahi[r][2] + (double)alo[r][2]), G * ((double)ahi[r][3] + (double)alo[r][3]));
  }
}

// ------------------ mixed (FP32), symmetric pair form -----------------------
// Plummer gravity computing each pair once (Newton's third law): the force
// of a pair is applied to i and, with the opposite sign and i's mass, to j.
// Per two pairs (one packed i-pair against one j) the loop issues 18 packed
// FP32 instructions (3 sub, 3 FMA for s^2, 2 mul for s^-3, 2 mul for the
// mass-weighted s^-3 of each side, 2 x 4 FMA into the i- and j-side sums)
// and 2 MUFU.rsq, against 26 and 4 when both directions are computed
// separately.
//
// Work split: the Morton order is cut into tiles of kSymTile particles; a
// block owns one i-tile (kSymWarps warps, kSymRP packed i-pairs per lane) and
// one work item = up to sym_chunk(nt) j-tiles strictly above its own, so the
// upper triangle of tile pairs is covered once; the diagonal tiles run
// through the one-sided kernel.  Inside a warp the j's travel: a batch of 32
// sources, one per lane, rotates through the lanes by shuffles, each lane
// meeting every source of the batch once; a source carries its own
// accumulator with it, so after 32 steps lane l holds the batch-partial of
// source l.  The partials of the block's warps are summed in shared memory
// (FP64) and added to the output with FP64 atomics; the i-side partials fold
// after every batch into FP64 accumulators kept in shared memory (registers
// go to the eight i-pairs a lane carries: many independent pairs per lane
// hide the MUFU and shuffle latencies better than more resident warps, as a
// sweep of warps x i-pairs per lane at N = 1M showed: 2 x 8 took 357 ms,
// 4 x 5 360 ms, 4 x 4 371 ms, 8 x 2 with FP64 registers 412 ms; later, with
// the equal-mass form, 2 x 8 at 248 registers took 315 ms and 2 x 6 at 168
// registers, six blocks per SM, 327 ms) and are added to the output at the
// end of the item.  The FMA pipe is the limiter; moving work to the MUFU
// pipe does not pay: s^-2 from a MUFU reciprocal instead of a multiply for
// 2, 4 or 8 of the 8 i-pairs measured 308, 312 and 330 ms against 303.
// The output therefore holds the diagonal-tile sums first (stored by the
// one-sided kernel) and receives the off-diagonal sums by atomics, so the
// order of the FP64 additions, not their values, varies between runs.
//
// Equal masses (UNI): when every particle has the same mass m (a flag the
// source-packing kernel computes on the device every step), the mass factors
// out of both sums -- a_i = m sum_j d / s^3, a_j = -m sum_i d / s^3,
// phi = -m sum 1/s -- and is applied once per batch partial (FP64) instead
// of per pair: 16 packed instructions per two pairs instead of 18, the same
// interactions.  Padding sources of a ragged last j-tile sit 1e18 away: their
// d / s^3 underflows to 0 and their 1/s of about 1e-18 vanishes in the FP32
// potential sums (every real term of a batch exceeds it by far more than
// 2^24), so no potential weight travels with the sources -- seven shuffles
// per source step instead of eight (N = 1M: 315 -> 303 ms, the same sums).
constexpr int kSymWarps = 2;
constexpr int kSymRP = 8;
constexpr int kSymTile = kSymWarps * 64 * kSymRP;  // 1024 i-particles per block

template <bool UNI>
__device__ __forceinline__ void sym_plummer_item(long long item, int n, int nt, const double4 *__restrict__ src,
                                                 double4 *__restrict__ out, float eps2, double G,
                                                 float (&red)[2][kSymWarps][4][32],
                                                 double (&iacc)[2 * kSymRP * 4][kSymWarps * 32]) {
  int b, t_lo, t_hi;
  sym_item(item, nt, b, t_lo, t_hi);
  const int j_lo = t_lo * kSymTile, j_hi = min(t_hi * kSymTile, n);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nxt = (l + 1) & 31;
  const int i0 = b * kSymTile;
  const double4 anc = src[i0];
  const int ib = i0 + w * 64 * kSymRP + l;
  // UNI: the common mass, applied to the i-side (+m) and j-side (-m) partials
  const double mi_scale = UNI ? src[0].w : 1.0, mj_scale = UNI ? -src[0].w : 1.0;

  f32x2 xi[kSymRP], yi[kSymRP], zi[kSymRP], nmi[kSymRP];
#pragma unroll
  for (int p = 0; p < kSymRP; p++) {
    float x[2] = {0.f, 0.f}, y[2] = {0.f, 0.f}, z[2] = {0.f, 0.f}, m[2] = {0.f, 0.f};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int i = ib + (2 * p + h) * 32;  // i-tiles of work items are full tiles (b < nt - 1)
      if (i < n) {
        const double4 q = src[i];
        x[h] = (float)(q.x - anc.x); y[h] = (float)(q.y - anc.y); z[h] = (float)(q.z - anc.z); m[h] = -(float)q.w;
      }
#pragma unroll
      for (int c = 0; c < 4; c++) iacc[(2 * p + h) * 4 + c][threadIdx.x] = 0.0;
    }
    xi[p] = pk2(x[0], x[1]); yi[p] = pk2(y[0], y[1]); zi[p] = pk2(z[0], z[1]); nmi[p] = pk2(m[0], m[1]);
  }
  const f32x2 e2 = pk2(eps2, eps2);
  int k = 0;
  for (int jb = j_lo; jb < j_hi; jb += 32, k ^= 1) {
    // padding source: massless at the anchor; UNI: far away (mj is unused)
    float xj = UNI ? 1e18f : 0.f, yj = xj, zj = xj, mj = 0.f;
    if (jb + l < j_hi) {
      const double4 q = src[jb + l];
      xj = (float)(q.x - anc.x); yj = (float)(q.y - anc.y); zj = (float)(q.z - anc.z); mj = UNI ? 1.f : (float)q.w;
    }
    float ajx = 0.f, ajy = 0.f, ajz = 0.f, ajp = 0.f;
    f32x2 px[kSymRP], py[kSymRP], pz[kSymRP], pp[kSymRP];
#pragma unroll
    for (int p = 0; p < kSymRP; p++) px[p] = py[p] = pz[p] = pp[p] = 0ull;
    // two source steps per iteration: the tail of one (its shuffles) overlaps
    // the head of the next (N = 1M: 315.7 -> 314.8 ms)
#pragma unroll 2
    for (int s = 0; s < 32; s++) {
      const f32x2 XJ = pk2(xj, xj), YJ = pk2(yj, yj), ZJ = pk2(zj, zj), MJ = pk2(mj, mj);
      f32x2 AX = pk2(ajx, 0.f), AY = pk2(ajy, 0.f), AZ = pk2(ajz, 0.f), AP = pk2(ajp, 0.f);
#pragma unroll
      for (int p = 0; p < kSymRP; p++) {
        const f32x2 dx = sub2(XJ, xi[p]), dy = sub2(YJ, yi[p]), dz = sub2(ZJ, zi[p]);
        f32x2 r2 = fma2(dx, dx, e2);
        r2 = fma2(dy, dy, r2);
        r2 = fma2(dz, dz, r2);
        float r2a, r2b;
        upk2(r2, r2a, r2b);
        const f32x2 inv = pk2(rsqrt_f32(r2a), rsqrt_f32(r2b));
        const f32x2 inv3 = mul2(mul2(inv, inv), inv);
        if (UNI) {
          px[p] = fma2(dx, inv3, px[p]);
          py[p] = fma2(dy, inv3, py[p]);
          pz[p] = fma2(dz, inv3, pz[p]);
          pp[p] = add2(pp[p], inv);
          AX = fma2(dx, inv3, AX);
          AY = fma2(dy, inv3, AY);
          AZ = fma2(dz, inv3, AZ);
          AP = add2(AP, inv);
        } else {
          const f32x2 sj = mul2(MJ, inv3), si = mul2(nmi[p], inv3);  // m_j / s^3, -m_i / s^3
          px[p] = fma2(dx, sj, px[p]);
          py[p] = fma2(dy, sj, py[p]);
          pz[p] = fma2(dz, sj, pz[p]);
          pp[p] = fma2(MJ, inv, pp[p]);
          AX = fma2(dx, si, AX);
          AY = fma2(dy, si, AY);
          AZ = fma2(dz, si, AZ);
          AP = fma2(nmi[p], inv, AP);
        }
      }
      float a0, a1;
      upk2(AX, a0, a1); ajx = a0 + a1;
      upk2(AY, a0, a1); ajy = a0 + a1;
      upk2(AZ, a0, a1); ajz = a0 + a1;
      upk2(AP, a0, a1); ajp = a0 + a1;
      xj = __shfl_sync(0xffffffffu, xj, nxt);
      yj = __shfl_sync(0xffffffffu, yj, nxt);
      zj = __shfl_sync(0xffffffffu, zj, nxt);
      if (!UNI) mj = __shfl_sync(0xffffffffu, mj, nxt);
      ajx = __shfl_sync(0xffffffffu, ajx, nxt);
      ajy = __shfl_sync(0xffffffffu, ajy, nxt);
      ajz = __shfl_sync(0xffffffffu, ajz, nxt);
      ajp = __shfl_sync(0xffffffffu, ajp, nxt);
    }
#pragma unroll
    for (int p = 0; p < kSymRP; p++) {
      const f32x2 part[4] = {px[p], py[p], pz[p], pp[p]};
#pragma unroll
      for (int c = 0; c < 4; c++) {
        float a0, a1;
        upk2(part[c], a0, a1);
        if (c == 3) a0 = -a0, a1 = -a1;  // pp holds +m/r (UNI: +1/r)
        iacc[(2 * p) * 4 + c][threadIdx.x] += a0;
        iacc[(2 * p + 1) * 4 + c][threadIdx.x] += a1;
      }
    }
    red[k][w][0][l] = ajx;
    red[k][w][1][l] = ajy;
    red[k][w][2][l] = ajz;
    red[k][w][3][l] = ajp;
    __syncthreads();  // also orders this batch's reads of red[k] before batch + 2 writes it
    for (int q = threadIdx.x; q < 128; q += kSymWarps * 32) {
      const int c = q >> 5, ll = q & 31;
      double s = 0.0;
#pragma unroll
      for (int v = 0; v < kSymWarps; v++) s += (double)red[k][v][c][ll];
      if (jb + ll < j_hi) atomicAdd(&reinterpret_cast<double *>(out + jb + ll)[c], G * mj_scale * s);
    }
  }
#pragma unroll
  for (int r = 0; r < 2 * kSymRP; r++) {
    const int i = ib + r * 32;
    if (i < n) {
      double *o = reinterpret_cast<double *>(out + i);
#pragma unroll
      for (int c = 0; c < 4; c++) atomicAdd(o + c, G * mi_scale * iacc[r * 4 + c][threadIdx.x]);
    }
  }
}

// mass_mixed: device word, 0 when all masses are equal (nullptr: general form);
// block b runs work item item0 + b
__global__ void __launch_bounds__(kSymWarps * 32, 4) k_grav_sym_plummer(int n, int nt, const double4 *__restrict__ src,
                                                                         double4 *__restrict__ out, float eps2,
                                                                         double G, const int *__restrict__ mass_mixed,
                                                                         long long item0) {
  __shared__ float red[2][kSymWarps][4][32];
  __shared__ double iacc[2 * kSymRP * 4][kSymWarps * 32];  // [i-slot * 4 + component][thread]
  const long long item = item0 + blockIdx.x;
  if (mass_mixed != nullptr && __ldg(mass_mixed) == 0)
    sym_plummer_item<true>(item, n, nt, src, out, eps2, G, red, iacc);
  else
    sym_plummer_item<false>(item, n, nt, src, out, eps2, G, red, iacc);
}

// ------------------- FP64, symmetric pair form ------------------------------
// The plain form of the symmetric Plummer kernel above: the same tiles, work
// items, travelling sources and block-combined j-side atomics, in FP64 with
// absolute coordinates (no anchor), kSym64R i-particles per lane and their
// FP64 sums in registers for the whole item.  Per pair: 3 sub, 3 FMA for
// s^2, the FP64 rsqrt (MUFU seed + one Householder step: 5 FP64 ops),
// 2 mul for s^-3, 2 for the mass-weighted s^-3 of each side, 8 FMA into the
// i- and j-side sums -- 23 FP64 operations against 36 for both directions;
// 21 in the equal-mass form (the mass applied to the sums at the end, as in
// the mixed kernel; padding sources 1e150 away, whose 1/s of about 6e-151
// vanishes in the potential sums, so no potential weight travels).  Each
// work item runs as two blocks of kSym64Warps warps, one per half of the
// i-tile (N = 1M: 756 -> 719 ms with the untravelled weight, against one
// block of twice the warps).
constexpr int kSym64Warps = 2;
constexpr int kSym64R = 8;
static_assert(2 * kSym64Warps * 32 * kSym64R == kSymTile, "the FP64 form shares the tile layout");

template <bool UNI>
__device__ __forceinline__ void sym_f64_item(long long item, int n, int nt, const double4 *__restrict__ src,
                                             double4 *__restrict__ out, double eps2, double G,
                                             double (&red)[2][kSym64Warps][4][32], int half) {
  int b, t_lo, t_hi;
  sym_item(item, nt, b, t_lo, t_hi);
  const int j_lo = t_lo * kSymTile, j_hi = min(t_hi * kSymTile, n);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nxt = (l + 1) & 31;
  const int ib = b * kSymTile + half * (kSymTile / 2) + w * 32 * kSym64R + l;
  const double4 far = src[b * kSymTile];  // position given to padding i-slots
  const double mi_scale = UNI ? src[0].w : 1.0, mj_scale = UNI ? -src[0].w : 1.0;

  double xi[kSym64R], yi[kSym64R], zi[kSym64R], nmi[kSym64R];
  double ax[kSym64R], ay[kSym64R], az[kSym64R], ap[kSym64R];
#pragma unroll
  for (int r = 0; r < kSym64R; r++) {
    const int i = ib + r * 32;  // i-tiles of work items are full tiles (b < nt - 1)
    const double4 q = i < n ? src[i] : make_double4(far.x, far.y, far.z, 0.0);
    xi[r] = q.x; yi[r] = q.y; zi[r] = q.z; nmi[r] = -q.w;
    ax[r] = ay[r] = az[r] = ap[r] = 0.0;
  }
  int k = 0;
  for (int jb = j_lo; jb < j_hi; jb += 32, k ^= 1) {
    // padding source: massless at a real position of the i-tile (s^2 >= eps^2 > 0);
    // UNI: 1e150 away (d / s^3 underflows to 0; mj is unused)
    const bool real = jb + l < j_hi;
    const double4 q = real ? src[jb + l] : (UNI ? make_double4(1e150, 1e150, 1e150, 0.0)
                                                : make_double4(far.x, far.y, far.z, 0.0));
    double xj = q.x, yj = q.y, zj = q.z, mj = UNI ? (real ? 1.0 : 0.0) : q.w;
    double bx = 0.0, by = 0.0, bz = 0.0, bp = 0.0;
#pragma unroll 1
    for (int s = 0; s < 32; s++) {
#pragma unroll
      for (int r = 0; r < kSym64R; r++) {
        const double dx = xj - xi[r], dy = yj - yi[r], dz = zj - zi[r];
        const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
        const double inv = rsqrt_f64(r2);
        const double inv3 = inv * inv * inv;
        if (UNI) {
          ax[r] = fma(dx, inv3, ax[r]);
          ay[r] = fma(dy, inv3, ay[r]);
          az[r] = fma(dz, inv3, az[r]);
          ap[r] -= inv;
          bx = fma(dx, inv3, bx);
          by = fma(dy, inv3, by);
          bz = fma(dz, inv3, bz);
          bp += inv;
        } else {
          const double sj = mj * inv3, si = nmi[r] * inv3;  // m_j / s^3, -m_i / s^3
          ax[r] = fma(dx, sj, ax[r]);
          ay[r] = fma(dy, sj, ay[r]);
          az[r] = fma(dz, sj, az[r]);
          ap[r] = fma(-mj, inv, ap[r]);
          bx = fma(dx, si, bx);
          by = fma(dy, si, by);
          bz = fma(dz, si, bz);
          bp = fma(nmi[r], inv, bp);
        }
      }
      xj = __shfl_sync(0xffffffffu, xj, nxt);
      yj = __shfl_sync(0xffffffffu, yj, nxt);
      zj = __shfl_sync(0xffffffffu, zj, nxt);
      if (!UNI) mj = __shfl_sync(0xffffffffu, mj, nxt);
      bx = __shfl_sync(0xffffffffu, bx, nxt);
      by = __shfl_sync(0xffffffffu, by, nxt);
      bz = __shfl_sync(0xffffffffu, bz, nxt);
      bp = __shfl_sync(0xffffffffu, bp, nxt);
    }
    red[k][w][0][l] = bx;
    red[k][w][1][l] = by;
    red[k][w][2][l] = bz;
    red[k][w][3][l] = bp;
    __syncthreads();  // also orders this batch's reads of red[k] before batch + 2 writes it
    for (int qq = threadIdx.x; qq < 128; qq += kSym64Warps * 32) {
      const int c = qq >> 5, ll = qq & 31;
      double sum = 0.0;
#pragma unroll
      for (int v = 0; v < kSym64Warps; v++) sum += red[k][v][c][ll];
      if (jb + ll < j_hi) atomicAdd(&reinterpret_cast<double *>(out + jb + ll)[c], G * mj_scale * sum);
    }
  }
#pragma unroll
  for (int r = 0; r < kSym64R; r++) {
    const int i = ib + r * 32;
    if (i < n) {
      double *o = reinterpret_cast<double *>(out + i);
      atomicAdd(o + 0, G * mi_scale * ax[r]);
      atomicAdd(o + 1, G * mi_scale * ay[r]);
      atomicAdd(o + 2, G * mi_scale * az[r]);
      atomicAdd(o + 3, G * mi_scale * ap[r]);
    }
  }
}

__global__ void __launch_bounds__(kSym64Warps * 32) k_grav_sym_f64(int n, int nt, const double4 *__restrict__ src,
                                                                  double4 *__restrict__ out, double eps2, double G,
                                                                  const int *__restrict__ mass_mixed, long long item0) {
  __shared__ double red[2][kSym64Warps][4][32];
  const long long item = item0 + (blockIdx.x >> 1);  // two blocks per item, one per half of the i-tile
  if (mass_mixed != nullptr && __ldg(mass_mixed) == 0)
    sym_f64_item<true>(item, n, nt, src, out, eps2, G, red, blockIdx.x & 1);
  else
    sym_f64_item<false>(item, n, nt, src, out, eps2, G, red, blockIdx.x & 1);
}

// blocks [lo, hi) of a one-sided or symmetric launch (nothing when empty)
struct Span {
  long long lo, hi;
  unsigned grid() const { return (unsigned)(hi - lo); }
  bool empty() const { return hi <= lo; }
};
static Span shard_span(long long count, int rank, int world) {
  Span sp;
  shard_range(count, rank, world, sp.lo, sp.hi);
  return sp;
}

// The direct-N work of one launch, and of shard `rank` of `world`: one-sided
// blocks of `block` particles -- each against the sources of its own tile of
// `tile` particles (the diagonal tiles), or against all sources when tile is
// 0 -- and the symmetric work items above the diagonal (tile pairs, each
// pair once).  Shards take contiguous shares of both lists.  Host code; the
// launch below and cudasph_gravity_plan both use it.
struct GravPlan {
  int tile;      // particles per symmetric tile; 0: the one-sided blocks cover all pairs
  int block;     // particles per one-sided block
  int nt;        // tiles
  int chunk;     // tiles per work item
  Span blocks;   // this shard's one-sided blocks
  Span items;    // this shard's symmetric work items
};

static GravPlan grav_plan(int n, int soft_mode, int precision, int rank, int world) {
  GravPlan g;
  g.nt = (n + kSymTile - 1) / kSymTile;
  g.chunk = g.nt >= 2 ? sym_chunk(g.nt) : 1;
  const bool sym = soft_mode == SPH_SOFT_PLUMMER;  // the spline kernels are one-sided over all pairs
  // FP64: R = 2 particles per thread; mixed Plummer: one packed i-pair per
  // thread (measured fastest at N = 1M: 68 registers, more resident warps to
  // cover the MUFU latency); mixed spline: R = 4
  g.block = precision == SPH_PREC_FP64 ? kGThreads * 2 : (sym ? kGThreads * 2 : kGThreads * 4);
  g.tile = sym && g.nt >= 2 ? kSymTile : 0;
  g.blocks = shard_span((n + g.block - 1) / g.block, rank, world);
  g.items = sym ? shard_span(sym_items(g.nt), rank, world) : Span{0, 0};
  return g;
}

// src = {x, y, z, m} per particle; h2src = range^2 (spline mode only).
// Shard `rank` of `world` (world > 1) computes its contiguous share of the
// one-sided blocks (diagonal tiles, or all pairs for small n / spline
// softening) and of the symmetric work items into `out`, which it zeroes
// first: the element-wise sum of the shards' outputs is the whole sum.
int launch_gravity(int n, const double4 *src, const double *h2src, double4 *out, int soft_mode, double eps, double G,
                   int precision, const int *mass_mixed, int rank, int world, cudaStream_t st) {
  if (n <= 0) return 0;
  if (world > 1) cudaMemsetAsync(out, 0, sizeof(double4) * n, st);
  const double eps2 = eps * eps;
  const GravPlan g = grav_plan(n, soft_mode, precision, rank, world);
  const int nt = g.nt;
  const Span &blocks = g.blocks, &items = g.items;
  int launches = 0;
  if (precision == SPH_PREC_FP64) {
    constexpr int R = 2;
    static_assert(kSymTile % (kGThreads * R) == 0, "diagonal tiles must hold whole blocks");
    if (soft_mode == SPH_SOFT_PLUMMER) {
      // diagonal tiles one-sided (all pairs when there is a single tile), then the items above them
      if (!blocks.empty()) {
        k_grav_f64<SPH_SOFT_PLUMMER, R><<<blocks.grid(), kGThreads, 0, st>>>(n, src, h2src, out, eps2, G, g.tile,
                                                                            (int)blocks.lo);
        launches++;
      }
      if (!items.empty()) {
        k_grav_sym_f64<<<items.grid() * 2, kSym64Warps * 32, 0, st>>>(n, nt, src, out, eps2, G, mass_mixed, items.lo);
        launches++;
      }
    } else if (!blocks.empty()) {
      k_grav_f64<SPH_SOFT_SPLINE, R><<<blocks.grid(), kGThreads, 0, st>>>(n, src, h2src, out, eps2, G, 0,
                                                                         (int)blocks.lo);
      launches++;
    }
  } else {
    if (soft_mode == SPH_SOFT_PLUMMER) {
      constexpr int RP = 1;
      static_assert(kSymTile % (kGThreads * 2 * RP) == 0, "diagonal tiles must hold whole blocks");
      // diagonal tiles store, the symmetric items add on top
      if (!blocks.empty()) {
        k_grav_f32x2_plummer<RP><<<blocks.grid(), kGThreads, 0, st>>>(n, src, out, (float)eps2, G, g.tile,
                                                                     (int)blocks.lo);
        launches++;
      }
      if (!items.empty()) {
        k_grav_sym_plummer<<<items.grid(), kSymWarps * 32, 0, st>>>(n, nt, src, out, (float)eps2, G, mass_mixed,
                                                                    items.lo);
        launches++;
      }
    } else {
      constexpr int R = 4;
      if (!blocks.empty()) {
        k_grav_f32<SPH_SOFT_SPLINE, R><<<blocks.grid(), kGThreads, 0, st>>>(n, src, h2src, out, (float)eps2, G,
                                                                           (int)blocks.lo);
        launches++;
      }
    }
  }
  return launches;
}

// pack the gravity sources {x, y, z, m} and range^2 from the state
// Also raises *mass_mixed (cleared before the launch) when some mass differs
// from the first particle's: the symmetric kernels take their equal-mass form
// when it stays 0.
__global__ void k_pack_sources(int n, const double4 *__restrict__ pos, const double4 *__restrict__ vel,
                               double4 *__restrict__ src, double *__restrict__ h2, int *__restrict__ mass_mixed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool differs = false;
  if (i < n) {
    const double4 p = pos[i];
    const double m = vel[i].w;
    src[i] = make_double4(p.x, p.y, p.z, m);
    h2[i] = p.w * p.w;
    differs = m != __ldg(&vel[0].w);
  }
  if (__syncthreads_or(differs) && threadIdx.x == 0) atomicOr(mass_mixed, 1);
}

int launch_pack_sources(int n, const double4 *pos, const double4 *vel, double4 *src, double *h2, int *mass_mixed,
                        cudaStream_t st) {
  cudaMemsetAsync(mass_mixed, 0, sizeof(int), st);
  k_pack_sources<<<(n + 255) / 256, 256, 0, st>>>(n, pos, vel, src, h2, mass_mixed);
  return 1;
}

__global__ void k_range_sq(int n, const double *__restrict__ r, double *__restrict__ h2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) h2[i] = r ? r[i] * r[i] : 0.0;
}

}  // namespace sph

extern "C" int cudasph_gravity_direct(int n, const double *pos4, const double *range, double *out4, int soft_mode,
                                      double eps, double G, int precision, void *stream) {
  if (n < 0 || (n > 0 && (!pos4 || !out4))) return SPH_ERR_ARG;
  if (soft_mode == SPH_SOFT_PLUMMER && !(eps > 0)) return SPH_ERR_ARG;
  if (soft_mode == SPH_SOFT_SPLINE && !range) return SPH_ERR_ARG;
  if (n == 0) return SPH_OK;
  cudaStream_t st = (cudaStream_t)stream;
  double *h2 = nullptr;
  if (soft_mode == SPH_SOFT_SPLINE) {
    SPH_CUDA_TRY(cudaMallocAsync((void **)&h2, sizeof(double) * n, st));
    sph::k_range_sq<<<(n + 255) / 256, 256, 0, st>>>(n, range, h2);
  }
  sph::launch_gravity(n, (const double4 *)pos4, h2, (double4 *)out4, soft_mode, eps, G, precision, nullptr, 0, 1, st);
  if (h2) SPH_CUDA_TRY(cudaFreeAsync(h2, st));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

// The gravity work plan without a device (the sharding's host-side logic).
extern "C" int cudasph_gravity_plan(int n, int precision, int soft_mode, int rank, int world, long long *out8) {
  if (n < 0 || !out8 || world < 1 || rank < 0 || rank >= world) return SPH_ERR_ARG;
  if (precision != SPH_PREC_FP64 && precision != SPH_PREC_MIXED) return SPH_ERR_ARG;
  if (soft_mode != SPH_SOFT_SPLINE && soft_mode != SPH_SOFT_PLUMMER) return SPH_ERR_ARG;
  const sph::GravPlan g = sph::grav_plan(n, soft_mode, precision, rank, world);
  out8[0] = g.tile;
  out8[1] = g.block;
  out8[2] = g.blocks.lo;
  out8[3] = g.blocks.hi;
  out8[4] = g.items.lo;
  out8[5] = g.items.hi;
  out8[6] = g.nt;
  out8[7] = g.chunk;
  return SPH_OK;
}

extern "C" int cudasph_gravity_item(int n, long long item, int *row, int *t_lo, int *t_hi) {
  if (n < 0 || !row || !t_lo || !t_hi) return SPH_ERR_ARG;
  const int nt = (n + sph::kSymTile - 1) / sph::kSymTile;
  if (item < 0 || item >= sph::sym_items(nt)) return SPH_ERR_ARG;
  sph::sym_item(item, nt, *row, *t_lo, *t_hi);
  return SPH_OK;
}
