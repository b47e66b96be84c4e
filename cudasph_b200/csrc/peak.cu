// peak.cu -- FMA-pipe throughput probe, the denominator of the gravity
// roofline.  The measured-peaks file of the pool carries HBM and tensor-core
// figures only, while the direct-N gravity inner loop runs on the FP32 (mixed
// form) or FP64 (plain form) FMA pipe, so its peak is measured in the same
// run: every thread advances 8 independent FMA chains; the grid fills every
// SM several times over.  FP32 is measured both with scalar FFMA and with
// packed fma.rn.f32x2 (two FP32 FMAs per instruction, the form the gravity
// loop issues), and the larger rate is the peak (on B200 the packed form
// measured 74.2 TFLOP/s against 71.1 for scalar FFMA; mixing the two gave no
// more than the scalar form).
#include "common.cuh"
#include "pairmath.cuh"

namespace sph {

__global__ void __launch_bounds__(256) k_fma_peak_f32x2(int iters, float a, float b, float *out) {
  const f32x2 A = pk2(a, a), B = pk2(b, b);
  const float t = (float)threadIdx.x;
  f32x2 x[8];
#pragma unroll
  for (int c = 0; c < 8; c++) x[c] = pk2(t + (float)c, t - (float)c);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
#pragma unroll
      for (int c = 0; c < 8; c++) x[c] = fma2(x[c], A, B);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    float lo, hi;
    upk2(x[c], lo, hi);
    s += lo + hi;
  }
  if (s == -1.2345f) out[blockIdx.x] = s;  // keeps the chains alive
}

template <class R>
__global__ void __launch_bounds__(256) k_fma_peak(int iters, R a, R b, R *out) {
  R x0 = (R)threadIdx.x, x1 = x0 + (R)1, x2 = x0 + (R)2, x3 = x0 + (R)3;
  R x4 = x0 + (R)4, x5 = x0 + (R)5, x6 = x0 + (R)6, x7 = x0 + (R)7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const R s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (R)-1.2345) out[blockIdx.x] = s;  // keeps the chains alive
}

}  // namespace sph

// Runs the probe on `stream` and returns the achieved FLOP/s (2 per FMA)
// measured with CUDA events; precision 1 = FP32, 0 = FP64.
extern "C" double cudasph_fma_peak(int precision, int iters, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256;
  void *out = nullptr;
  if (cudaMallocAsync(&out, sizeof(double) * blocks, st) != cudaSuccess) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // each form: warm up, then time; FP32: scalar (form 0) and packed (form 1)
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  double best = -1;
  for (int form = 0; form < (precision == 1 ? 2 : 1); form++) {
    for (int rep = 0; rep < 2; rep++) {
      cudaEventRecord(e0, st);
      if (precision == 1 && form == 0)
        sph::k_fma_peak<float><<<blocks, threads, 0, st>>>(iters, 0.999999f, 1e-7f, (float *)out);
      else if (precision == 1)
        sph::k_fma_peak_f32x2<<<blocks, threads, 0, st>>>(iters, 0.999999f, 1e-7f, (float *)out);
      else
        sph::k_fma_peak<double><<<blocks, threads, 0, st>>>(iters, 0.999999999, 1e-12, (double *)out);
      cudaEventRecord(e1, st);
    }
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double f = ms > 0 ? flops * (form == 1 ? 2.0 : 1.0) / (ms * 1e-3) : -1;
    if (f > best) best = f;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(out, st);
  cudaStreamSynchronize(st);
  return best;
}

namespace sph {

// L2 read-bandwidth probe: a 48 MB buffer (well inside the 126 MB L2, after
// a first pass that brings it there) read by every SM in a grid-stride loop,
// 32 bytes per load, cached at L2 only (ld.global.cg), so the figure is the
// L2-to-SM read rate: the denominator of the gather rates of the neighbour
// loops, whose records come from L1 and L2.
__global__ void __launch_bounds__(256) k_l2_read(const double4 *__restrict__ buf, long long n4, int iters,
                                                 double *out) {
  double acc = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int it = 0; it < iters; it++) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
      double4 v;
      asm volatile("ld.global.cg.v4.f64 {%0, %1, %2, %3}, [%4];"
                   : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
                   : "l"(buf + i));
      acc += (v.x + v.y) + (v.z + v.w);
    }
  }
  if (acc == -1.2345) out[0] = acc;  // keeps the loads alive
}

}  // namespace sph

// Runs the L2 probe on `stream` and returns the achieved read bytes/s
// (CUDA events, the better of two timed launches after a warm-up).
extern "C" double cudasph_l2_peak(int iters, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long bytes = 48ll << 20, n4 = bytes / 32;
  if (iters < 1) return -1;
  void *buf = nullptr, *out = nullptr;
  if (cudaMallocAsync(&buf, (size_t)bytes, st) != cudaSuccess) return -1;
  if (cudaMallocAsync(&out, sizeof(double), st) != cudaSuccess) {
    cudaFreeAsync(buf, st);
    return -1;
  }
  cudaMemsetAsync(buf, 0, (size_t)bytes, st);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256;
  sph::k_l2_read<<<blocks, threads, 0, st>>>((const double4 *)buf, n4, 1, (double *)out);  // into L2
  double best = -1;
  for (int rep = 0; rep < 2; rep++) {
    cudaEventRecord(e0, st);
    sph::k_l2_read<<<blocks, threads, 0, st>>>((const double4 *)buf, n4, iters, (double *)out);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double r = ms > 0 ? (double)bytes * iters / (ms * 1e-3) : -1;
    if (r > best) best = r;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(buf, st);
  cudaFreeAsync(out, st);
  cudaStreamSynchronize(st);
  return best;
}
