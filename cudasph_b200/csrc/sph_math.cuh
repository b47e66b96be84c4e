// sph_math.cuh -- the M4 cubic-spline kernel family of dev_sph_kernels.cu:7-99,
// templated on the arithmetic type (double for the FP64 form, float for the
// pair terms of the mixed form).
//
// The expressions keep the reference's operation order (e.g. 4*pi*u*u*w(u),
// u3/3 - 0.3*u3*u*u + ...), so that translation units compiled without FMA
// contraction reproduce an FP64 CPU evaluation of the same formulas bit for
// bit.  The functions are the standard ones:
//   w(u)      = W normalised by 1/pi; dw = (1/u) dW/du; dwdh = dW/dh term;
//   dphidh    = d(softened potential)/dh term;
//   iw(x)     = integral of 4 pi x^2 w(x);  ig(u) = iw(4 (1 - |u - 1|)), the
//               smooth neighbour-count weight; digdh = u d(ig)/du; dig = (1/u) d(ig)/du.
#pragma once

namespace sph {

template <class R>
struct KC {
  static constexpr R pi = (R)3.141592653589793;
  static constexpr R ipi = (R)0.318309886183791;
};

template <class R>
__device__ __forceinline__ R k_w(R u) {
  if (u < 0) return KC<R>::ipi;
  if (u < 1) return KC<R>::ipi * ((R)1 - (R)1.5 * u * u + (R)0.75 * u * u * u);
  if (u < 2) return KC<R>::ipi * (R)0.25 * ((R)2 - u) * ((R)2 - u) * ((R)2 - u);
  return 0;
}
template <class R>
__device__ __forceinline__ R k_diw(R u) {
  return (R)4.0 * KC<R>::pi * u * u * k_w<R>(u);
}
template <class R>
__device__ __forceinline__ R k_iw(R u) {
  if (u < 0) return 0;
  if (u < 1) {
    R u3 = u * u * u;
    return (R)4 * (u3 / (R)3.0 - (R)0.3 * u3 * u * u + (R)0.125 * u3 * u3);
  }
  if (u < 2) {
    R u3 = u * u * u;
    return (R)4 * ((R)(-1.0 / 60) + (R)(2.0 / 3) * u3 - (R)0.75 * u3 * u + (R)0.3 * u3 * u * u - u3 * u3 / (R)24.0);
  }
  return 1;
}
template <class R>
__device__ __forceinline__ R k_ig(R u) {
  return k_iw<R>((R)4.0 * ((R)1.0 - fabs(u - (R)1.0)));
}
template <class R>
__device__ __forceinline__ R k_digdh(R u) {
  if (u <= 0) return 0;
  if (u < 1) return (R)4.0 * u * k_diw<R>((R)4.0 * u);
  if (u < 2) return (R)(-4.0) * u * k_diw<R>((R)4.0 * ((R)2 - u));
  return 0;
}
template <class R>
__device__ __forceinline__ R k_dig(R u) {
  if (u <= 0) return 0;
  if (u < 1) return (R)4.0 / u * k_diw<R>((R)4.0 * u);
  if (u < 2) return (R)(-4.0) / u * k_diw<R>((R)4.0 * ((R)2 - u));
  return 0;
}
template <class R>
__device__ __forceinline__ R k_dw(R u) {
  if (u < 1) return KC<R>::ipi * ((R)(-3) + (R)2.25 * u);
  if (u < 2) return -KC<R>::ipi * (R)0.75 * ((R)2 - u) * ((R)2 - u) / u;
  return 0;
}
template <class R>
__device__ __forceinline__ R k_dwdh(R u) {
  if (u < 1) return KC<R>::ipi * ((R)(-3) + (R)7.5 * u * u - (R)4.5 * u * u * u);
  if (u < 2) return KC<R>::ipi * ((R)(-6) + (R)12 * u - (R)7.5 * u * u + (R)1.5 * u * u * u);
  return 0;
}
template <class R>
__device__ __forceinline__ R k_dphidh(R u) {
  R u2 = u * u;
  if (u < 1) return (R)1.4 - (R)2 * u2 + (R)1.5 * u2 * u2 - (R)0.6 * u2 * u2 * u;
  if (u < 2) return (R)1.6 - (R)4 * u2 + (R)4 * u2 * u - (R)1.5 * u2 * u2 + (R)0.2 * u2 * u2 * u;
  return 0;
}

}  // namespace sph
