// sort.cu -- Morton keys and a stable LSD radix sort (the space-filling-curve
// sort of sort_bodies.cpp:119-186, done on the device every step), and the
// reference's Peano-Hilbert keys as an optional sort key.
//
// Keys: positions quantised to 21 bits per dimension in the bounding cube
// (scale = 2^21 / max extent, like domain_fac of sort_bodies.cpp:135), bits
// interleaved x-y-z from the top.  The sort is an 8-bit-digit LSD radix sort
// (8 passes over 64-bit keys): per pass a per-block digit histogram, one
// exclusive scan over [digit][block], and a stable scatter in which each
// warp ranks equal digits with __match_any_sync.  Ties keep their input
// order, so with values = slot indices the permutation equals a stable sort.
#include <cstdio>

#include "common.cuh"

namespace sph {

constexpr int kRadixThreads = 256;
constexpr int kRadixChunk = 4096;  // keys per block per pass

__global__ void k_bbox_partial(int n, const double4 *__restrict__ pos, const double *__restrict__ x,
                               const double *__restrict__ y, const double *__restrict__ z, double *__restrict__ part) {
  double lo[3] = {1e308, 1e308, 1e308}, hi[3] = {-1e308, -1e308, -1e308};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double c[3];
    if (pos) {
      double4 p = pos[i];
      c[0] = p.x; c[1] = p.y; c[2] = p.z;
    } else {
      c[0] = x[i]; c[1] = y[i]; c[2] = z[i];
    }
#pragma unroll
    for (int d = 0; d < 3; d++) { lo[d] = fmin(lo[d], c[d]); hi[d] = fmax(hi[d], c[d]); }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  __shared__ double s[32][6];
  int w = threadIdx.x >> 5;
  if (lane_id() == 0)
    for (int d = 0; d < 3; d++) { s[w][d] = lo[d]; s[w][3 + d] = hi[d]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nw = blockDim.x >> 5;
    for (int k = 1; k < nw; k++)
      for (int d = 0; d < 3; d++) { s[0][d] = fmin(s[0][d], s[k][d]); s[0][3 + d] = fmax(s[0][3 + d], s[k][3 + d]); }
    for (int d = 0; d < 6; d++) part[blockIdx.x * 6 + d] = s[0][d];
  }
}

// box4 = {lo.x, lo.y, lo.z, scale}; scale = 2^21 / max extent (0 if degenerate)
__global__ void k_bbox_final(int nb, const double *__restrict__ part, double *__restrict__ box4) {
  if (threadIdx.x != 0) return;
  double lo[3] = {1e308, 1e308, 1e308}, hi[3] = {-1e308, -1e308, -1e308};
  for (int b = 0; b < nb; b++)
    for (int d = 0; d < 3; d++) { lo[d] = fmin(lo[d], part[b * 6 + d]); hi[d] = fmax(hi[d], part[b * 6 + 3 + d]); }
  double size = hi[0] - lo[0];
  if (hi[1] - lo[1] > size) size = hi[1] - lo[1];
  if (hi[2] - lo[2] > size) size = hi[2] - lo[2];
  box4[0] = lo[0]; box4[1] = lo[1]; box4[2] = lo[2];
  box4[3] = size > 0 ? __ddiv_rn(2097152.0, size) : 0.0;
}

__device__ __forceinline__ uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}

__device__ __forceinline__ uint32_t quant21(double c, double lo, double scale) {
  double v = __dmul_rn(__dsub_rn(c, lo), scale);
  return v >= 2097151.0 ? 2097151u : (uint32_t)v;
}

__global__ void k_morton(int n, const double4 *__restrict__ pos, const double *__restrict__ x,
                         const double *__restrict__ y, const double *__restrict__ z, const double *__restrict__ box4,
                         uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double c0, c1, c2;
  if (pos) {
    double4 p = pos[i];
    c0 = p.x; c1 = p.y; c2 = p.z;
  } else {
    c0 = x[i]; c1 = y[i]; c2 = z[i];
  }
  double s = box4[3];
  uint32_t qx = quant21(c0, box4[0], s), qy = quant21(c1, box4[1], s), qz = quant21(c2, box4[2], s);
  keys[i] = (spread3(qx) << 2) | (spread3(qy) << 1) | spread3(qz);
  if (vals) vals[i] = (uint32_t)i;
}

// per-block digit histogram, stored digit-major: hist[d * nb + block]
__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(int n, const uint64_t *__restrict__ keys, int shift,
                                                              unsigned *__restrict__ hist) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int beg = blockIdx.x * kRadixChunk, end = min(n, beg + kRadixChunk);
  for (int i = beg + threadIdx.x; i < end; i += kRadixThreads) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  __syncthreads();
  hist[threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// exclusive scan of m entries in one block of 1024 threads: warp w owns the
// contiguous segment [w * seg, (w + 1) * seg) and walks it in coalesced
// 32-entry chunks (warp shuffle scan per chunk); a first pass sums the
// segments, a block scan of the 32 segment sums gives each warp its offset,
// a second pass writes the prefixes.
__global__ void __launch_bounds__(1024) k_radix_scan(int m, unsigned *__restrict__ hist) {
  __shared__ unsigned seg_sum[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int seg = (m + 31) / 32;
  const int beg = w * seg, end = min(m, beg + seg);
  unsigned tot = 0;
  for (int i = beg + l; i < end; i += 32) tot += hist[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
  if (l == 0) seg_sum[w] = tot;
  __syncthreads();
  if (w == 0) {
    const unsigned v = seg_sum[l];
    unsigned inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
      if (l >= o) inc += t;
    }
    seg_sum[l] = inc - v;  // exclusive
  }
  __syncthreads();
  unsigned run = seg_sum[w];
  for (int c = beg; c < end; c += 32) {
    const int i = c + l;
    const unsigned v = i < end ? hist[i] : 0u;
    unsigned inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
      if (l >= o) inc += t;
    }
    if (i < end) hist[i] = run + inc - v;
    run += __shfl_sync(0xffffffffu, inc, 31);
  }
}

__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(int n, const uint64_t *__restrict__ kin,
                                                                 const uint32_t *__restrict__ vin,
                                                                 uint64_t *__restrict__ kout,
                                                                 uint32_t *__restrict__ vout, int shift,
                                                                 const unsigned *__restrict__ hist) {
  __shared__ unsigned s_base[256];
  __shared__ unsigned s_cnt[kRadixThreads / 32][256];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  s_base[t] = hist[t * gridDim.x + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kRadixThreads / 32; w++) s_cnt[w][t] = 0;
  __syncthreads();
  const int beg = blockIdx.x * kRadixChunk, end = min(n, beg + kRadixChunk);
  const unsigned lt = (1u << lane) - 1u;
  for (int base = beg; base < end; base += kRadixThreads) {
    int i = base + t;
    bool valid = i < end;
    uint64_t k = valid ? kin[i] : 0;
    uint32_t v = valid ? vin[i] : 0;
    unsigned d = valid ? (unsigned)((k >> shift) & 255u) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    unsigned rank = __popc(peers & lt);
    if (valid && rank == 0) s_cnt[warp][d] = __popc(peers);
    __syncthreads();
    {  // thread t owns digit t: exclusive prefix across warps
      unsigned run = s_base[t];
#pragma unroll
      for (int w = 0; w < kRadixThreads / 32; w++) {
        unsigned c = s_cnt[w][t];
        s_cnt[w][t] = run;
        run += c;
      }
      s_base[t] = run;
    }
    __syncthreads();
    if (valid) {
      unsigned o = s_cnt[warp][d] + rank;
      kout[o] = k;
      vout[o] = v;
    }
    __syncthreads();
#pragma unroll
    for (int w = 0; w < kRadixThreads / 32; w++) s_cnt[w][t] = 0;
    __syncthreads();
  }
}

size_t radix_scratch_bytes(int n) {
  size_t nb = (size_t)(n + kRadixChunk - 1) / kRadixChunk;
  if (nb == 0) nb = 1;
  size_t b = 0;
  b += ((size_t)n * 8 + 255) / 256 * 256;    // keys ping-pong
  b += ((size_t)n * 4 + 255) / 256 * 256;    // vals ping-pong
  b += (256 * nb * 4 + 255) / 256 * 256;     // histograms
  return b;
}

// Stable sort of (keys, vals); result in keys/vals.  Returns launches.
int radix_sort_u64(int n, uint64_t *keys, uint32_t *vals, void *scratch, cudaStream_t st) {
  if (n <= 1) return 0;
  int nb = (n + kRadixChunk - 1) / kRadixChunk;
  char *p = (char *)scratch;
  uint64_t *k2 = (uint64_t *)p;
  p += ((size_t)n * 8 + 255) / 256 * 256;
  uint32_t *v2 = (uint32_t *)p;
  p += ((size_t)n * 4 + 255) / 256 * 256;
  unsigned *hist = (unsigned *)p;
  uint64_t *ka = keys, *kb = k2;
  uint32_t *va = vals, *vb = v2;
  int launches = 0;
  for (int shift = 0; shift < 64; shift += 8) {
    k_radix_hist<<<nb, kRadixThreads, 0, st>>>(n, ka, shift, hist);
    k_radix_scan<<<1, 1024, 0, st>>>(256 * nb, hist);
    k_radix_scatter<<<nb, kRadixThreads, 0, st>>>(n, ka, va, kb, vb, shift, hist);
    launches += 3;
    uint64_t *tk = ka; ka = kb; kb = tk;
    uint32_t *tv = va; va = vb; vb = tv;
  }
  // 8 passes: the result is back in keys/vals
  return launches;
}

// bounding box + Morton keys of positions (double4 records or separate x/y/z)
int morton_keys(int n, const double4 *pos, const double *x, const double *y, const double *z, double *part,
                double *box4, uint64_t *keys, uint32_t *vals, cudaStream_t st) {
  int nb = 148 * 2;
  if (nb * 256 > n) nb = (n + 255) / 256;
  if (nb < 1) nb = 1;
  k_bbox_partial<<<nb, 256, 0, st>>>(n, pos, x, y, z, part);
  k_bbox_final<<<1, 32, 0, st>>>(nb, part, box4);
  k_morton<<<(n + 255) / 256, 256, 0, st>>>(n, pos, x, y, z, box4, keys, vals);
  return 3;
}

// ---------------------------------------------------------------------------
// Peano-Hilbert keys: the reference's space-filling curve (sort_bodies.cpp:
// 66-105), an optional sort key (sph_params.key_mode) for the reference's
// particle order.  Each level of a key descends into one octant of the
// current cell; the octant's rank along the curve is the level's 3-bit
// digit, and the octant's sub-cells are visited in a rotated frame, possibly
// in reverse.  Frames are proper rotations of the cube.  The curve is fixed
// by
//   * the visiting order in the unrotated frame: rank q visits the octant
//     whose (z, x, y) bits are the Gray code q ^ (q >> 1);
//   * per rank q, the child's frame: the parent's frame followed by
//     kPhTurnsX[q] quarter turns about x and kPhTurnsY[q] about y, and
//     whether the child's direction is the reverse of its parent's.
// Those per-rank turns and reversals carry the same information as
// rotx_table, roty_table and sense_table (sort_bodies.cpp:53-57): the keys
// agree only for the same curve.  The (frame, direction) pairs reachable
// from the root form a 24-state automaton, generated at compile time, so a
// key costs one shared-memory lookup per level: entry = next state * 8 +
// digit, indexed by state * 8 + (bx << 2 | by << 1 | bz).
// ---------------------------------------------------------------------------
struct PhFrame {
  int m[9];  // row-major signed permutation matrix
};

constexpr PhFrame ph_mul(const PhFrame &a, const PhFrame &b) {
  PhFrame r{};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      int v = 0;
      for (int k = 0; k < 3; k++) v += a.m[i * 3 + k] * b.m[k * 3 + j];
      r.m[i * 3 + j] = v;
    }
  return r;
}

constexpr bool ph_same(const PhFrame &a, const PhFrame &b) {
  for (int i = 0; i < 9; i++)
    if (a.m[i] != b.m[i]) return false;
  return true;
}

constexpr PhFrame kPhTurnX = {{1, 0, 0, 0, 0, 1, 0, -1, 0}};  // quarter turn about x
constexpr PhFrame kPhTurnY = {{0, 0, -1, 0, 1, 0, 1, 0, 0}};  // quarter turn about y
constexpr int kPhTurnsX[8] = {3, 0, 0, 2, 2, 0, 0, 1};
constexpr int kPhTurnsY[8] = {0, 1, 1, 2, 2, 3, 3, 0};
constexpr int kPhReverse[8] = {1, 1, 1, 0, 0, 1, 1, 1};
constexpr int kPhStates = 24;
constexpr int kPhMaxStates = 48;  // frames x directions

constexpr int ph_gray_rank(int g) {
  int q = 0;
  for (; g; g >>= 1) q ^= g;
  return q;
}

// rank along the curve, in frame f, of the world octant o = bx << 2 | by << 1 | bz
constexpr int ph_rank(const PhFrame &f, int o) {
  const int s[3] = {((o >> 2) & 1) * 2 - 1, ((o >> 1) & 1) * 2 - 1, (o & 1) * 2 - 1};
  int l[3] = {0, 0, 0};  // the octant's centre in the frame's own axes: f^T s
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) l[i] += f.m[j * 3 + i] * s[j];
  const int bx = (l[0] + 1) / 2, by = (l[1] + 1) / 2, bz = (l[2] + 1) / 2;
  return ph_gray_rank((bz << 2) | (bx << 1) | by);
}

struct PhTable {
  uint16_t e[kPhMaxStates * 8];
  int nstates;
};

constexpr PhTable make_ph_table() {
  PhFrame frame[kPhMaxStates] = {};
  int rev[kPhMaxStates] = {};
  frame[0] = PhFrame{{1, 0, 0, 0, 1, 0, 0, 0, 1}};
  int ns = 1;
  PhTable t{};
  for (int s = 0; s < ns; s++)
    for (int o = 0; o < 8; o++) {
      const int q = ph_rank(frame[s], o);
      PhFrame f = frame[s];
      for (int k = 0; k < kPhTurnsX[q]; k++) f = ph_mul(f, kPhTurnX);
      for (int k = 0; k < kPhTurnsY[q]; k++) f = ph_mul(f, kPhTurnY);
      const int r = rev[s] ^ kPhReverse[q];
      int id = 0;
      while (id < ns && !(rev[id] == r && ph_same(frame[id], f))) id++;
      if (id == ns) {  // a new state (at most kPhMaxStates exist)
        frame[ns] = f;
        rev[ns] = r;
        ns++;
      }
      t.e[s * 8 + o] = (uint16_t)(id * 8 + (rev[s] ? 7 - q : q));
    }
  t.nstates = ns;
  return t;
}

static_assert(make_ph_table().nstates == kPhStates, "the curve's automaton has 24 states");

__constant__ PhTable g_ph_table = make_ph_table();

__device__ __forceinline__ void ph_load_table(uint16_t *tab) {
  for (int i = threadIdx.x; i < kPhStates * 8; i += blockDim.x) tab[i] = g_ph_table.e[i];
  __syncthreads();
}

// key of the integer triplet: levels bits-1 .. 0 of each coordinate (higher
// bits are ignored, as the reference's mask does)
__device__ __forceinline__ uint64_t ph_key(const uint16_t *tab, uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint64_t key = 0;
  int s = 0;  // state * 8
  for (int l = bits - 1; l >= 0; l--) {
    const int o = (((x >> l) & 1u) << 2) | (((y >> l) & 1u) << 1) | ((z >> l) & 1u);
    const int e = tab[s + o];
    key = (key << 3) | (uint64_t)(e & 7);
    s = e & ~7;
  }
  return key;
}

__global__ void k_peano_int(int n, const int *__restrict__ x, const int *__restrict__ y, const int *__restrict__ z,
                            int bits, uint64_t *__restrict__ keys) {
  __shared__ uint16_t tab[kPhStates * 8];
  ph_load_table(tab);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keys[i] = ph_key(tab, (uint32_t)x[i], (uint32_t)y[i], (uint32_t)z[i], bits);
}

constexpr int kPhBits = 18;  // BITS_PER_DIMENSION, sort_bodies.cpp:3

// the reference's quantisation box (sort_bodies.cpp:121-135) in float, from
// the double bounding box (rounding is monotone, so the float box of the
// float-rounded positions is the rounded double box): box4 = {lo.x, lo.y,
// lo.z, domain_fac}, domain_fac = float(1.0 / size * 2^18) with size the
// largest float extent; 0 for a degenerate box (all keys 0)
__global__ void k_peano_box_final(int nb, const double *__restrict__ part, double *__restrict__ box4) {
  if (threadIdx.x != 0) return;
  double lo[3] = {1e308, 1e308, 1e308}, hi[3] = {-1e308, -1e308, -1e308};
  for (int b = 0; b < nb; b++)
    for (int d = 0; d < 3; d++) { lo[d] = fmin(lo[d], part[b * 6 + d]); hi[d] = fmax(hi[d], part[b * 6 + 3 + d]); }
  float lf[3], ext[3];
  for (int d = 0; d < 3; d++) {
    lf[d] = __double2float_rn(lo[d]);
    ext[d] = __fsub_rn(__double2float_rn(hi[d]), lf[d]);
  }
  const float size = fmaxf(ext[2], fmaxf(ext[1], ext[0]));
  const float fac = size > 0.f ? __double2float_rn(__dmul_rn(__ddiv_rn(1.0, (double)size), (double)(1 << kPhBits)))
                               : 0.f;
  box4[0] = lf[0]; box4[1] = lf[1]; box4[2] = lf[2]; box4[3] = fac;
}

// positions rounded to float (the reference's float4 state), offset and
// scaled in float and truncated (sort_bodies.cpp:155-159), then keyed
__global__ void k_peano_pos(int n, const double4 *__restrict__ pos, const double *__restrict__ x,
                            const double *__restrict__ y, const double *__restrict__ z,
                            const double *__restrict__ box4, uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  __shared__ uint16_t tab[kPhStates * 8];
  ph_load_table(tab);
  const float lx = (float)box4[0], ly = (float)box4[1], lz = (float)box4[2], fac = (float)box4[3];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double c0, c1, c2;
    if (pos) {
      const double4 p = pos[i];
      c0 = p.x; c1 = p.y; c2 = p.z;
    } else {
      c0 = x[i]; c1 = y[i]; c2 = z[i];
    }
    const int qx = __float2int_rz(__fmul_rn(__fsub_rn(__double2float_rn(c0), lx), fac));
    const int qy = __float2int_rz(__fmul_rn(__fsub_rn(__double2float_rn(c1), ly), fac));
    const int qz = __float2int_rz(__fmul_rn(__fsub_rn(__double2float_rn(c2), lz), fac));
    keys[i] = ph_key(tab, (uint32_t)qx, (uint32_t)qy, (uint32_t)qz, kPhBits);
    if (vals) vals[i] = (uint32_t)i;
  }
}

// bounding box + Peano-Hilbert keys of positions (double4 records or x/y/z)
int peano_keys(int n, const double4 *pos, const double *x, const double *y, const double *z, double *part,
               double *box4, uint64_t *keys, uint32_t *vals, cudaStream_t st) {
  int nb = 148 * 2;
  if (nb * 256 > n) nb = (n + 255) / 256;
  if (nb < 1) nb = 1;
  k_bbox_partial<<<nb, 256, 0, st>>>(n, pos, x, y, z, part);
  k_peano_box_final<<<1, 32, 0, st>>>(nb, part, box4);
  k_peano_pos<<<(n + 255) / 256, 256, 0, st>>>(n, pos, x, y, z, box4, keys, vals);
  return 3;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the radix sort.  Its scratch (ping-pong key and
// value buffers plus the per-block digit histograms) is a file-scope device
// array sized for kNoAllocMaxKeys keys; every GPU that loads this library
// holds those bytes until the process exits.
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxKeys = CUDASPH_SORT_NOALLOC_MAX_KEYS;
static_assert(kNoAllocMaxKeys == (1 << 18), "header and library disagree");
constexpr size_t round256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kNoAllocScratchBytes =
    round256((size_t)kNoAllocMaxKeys * 8) + round256((size_t)kNoAllocMaxKeys * 4) +
    round256(256 * (((size_t)kNoAllocMaxKeys + kRadixChunk - 1) / kRadixChunk) * 4);

static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[kNoAllocScratchBytes];

}  // namespace sph

#include <cuda.h>  // driver types only; the entry points come from cudaGetDriverEntryPoint

#include <mutex>

namespace {
// Host code cannot use the array's name as a device address (on the host it
// names a stand-in object), so the address is looked up with the device
// current and cached per device, together with the id of the context it was
// looked up in: after a cudaDeviceReset the library's module is loaded again
// into a new primary context, the array may move, and the next call looks the
// address up anew.
constexpr int kMaxDevices = 128;
std::mutex g_noalloc_mu;
struct NoAllocSlot {
  void *ptr;
  unsigned long long ctx_id;
};
NoAllocSlot g_noalloc[kMaxDevices] = {};

typedef CUresult (*ctx_get_current_fn)(CUcontext *);
typedef CUresult (*ctx_get_id_fn)(CUcontext, unsigned long long *);

ctx_get_current_fn g_get_current = nullptr;
ctx_get_id_fn g_get_id = nullptr;

// whether the driver gives context ids (resolved once)
bool context_ids_available() {
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr, *g = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &q2) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
      g_get_current = (ctx_get_current_fn)f;
      g_get_id = (ctx_get_id_fn)g;
    }
    (void)cudaGetLastError();
  });
  return g_get_current && g_get_id;
}

// id of the context current on this thread, 0 if none is
unsigned long long current_context_id() {
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (g_get_current(&c) != CUDA_SUCCESS || !c || g_get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

int noalloc_scratch(void **out) {
  int dev = 0;
  SPH_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    sph_internal_set_error("cudasph_radix_sort_u64_noalloc: device ordinal beyond the address cache");
    return SPH_ERR_ARG;
  }
  // without context ids from the driver the address is cached per device only
  const bool ids = context_ids_available();
  const unsigned long long ctx = ids ? current_context_id() : 0;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocSlot &slot = g_noalloc[dev];
  if (!slot.ptr || (ids && slot.ctx_id != ctx)) {
    void *p = nullptr;
    SPH_CUDA_TRY(cudaGetSymbolAddress(&p, sph::g_noalloc_sort_scratch));
    slot.ptr = p;
    // the lookup made the device's context current if none was
    slot.ctx_id = ids ? current_context_id() : 0;
  }
  *out = slot.ptr;
  return SPH_OK;
}
}  // namespace

extern "C" int cudasph_radix_sort_u64_noalloc(int n, uint64_t *keys, uint32_t *vals, void *stream) {
  if (n < 0 || n > sph::kNoAllocMaxKeys) {
    char msg[160];
    snprintf(msg, sizeof(msg), "cudasph_radix_sort_u64_noalloc: n = %d outside [0, %d], the size of its fixed scratch",
             n, sph::kNoAllocMaxKeys);
    sph_internal_set_error(msg);
    return SPH_ERR_ARG;
  }
  if (n > 0 && (!keys || !vals)) {
    sph_internal_set_error("cudasph_radix_sort_u64_noalloc: keys and vals must be device pointers (null given)");
    return SPH_ERR_ARG;
  }
  if (n <= 1) return SPH_OK;
  void *scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  // nothing in the scratch has to start at zero: every pass rewrites all
  // histogram entries and every key/value slot it later reads
  sph::radix_sort_u64(n, keys, vals, scratch, (cudaStream_t)stream);
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}


extern "C" size_t cudasph_sort_scratch_bytes(int n) { return sph::radix_scratch_bytes(n) + 148 * 2 * 6 * 8 + 256; }

extern "C" int cudasph_radix_sort_u64(int n, uint64_t *keys, uint32_t *vals, void *scratch, void *stream) {
  if (n < 0 || (n > 0 && (!keys || !vals || !scratch))) return SPH_ERR_ARG;
  sph::radix_sort_u64(n, keys, vals, scratch, (cudaStream_t)stream);
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_peano_keys(int n, const double *x, const double *y, const double *z, uint64_t *keys,
                                  double *box4, void *stream) {
  if (n <= 0) return n == 0 ? SPH_OK : SPH_ERR_ARG;
  if (!x || !y || !z || !keys || !box4) return SPH_ERR_ARG;
  double *part = nullptr;
  SPH_CUDA_TRY(cudaMallocAsync((void **)&part, 148 * 2 * 6 * sizeof(double), (cudaStream_t)stream));
  sph::peano_keys(n, nullptr, x, y, z, part, box4, keys, nullptr, (cudaStream_t)stream);
  SPH_CUDA_TRY(cudaFreeAsync(part, (cudaStream_t)stream));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_peano_hilbert_keys(int n, const int *x, const int *y, const int *z, int bits, uint64_t *keys,
                                          void *stream) {
  if (n < 0 || bits < 1 || bits > 21) return SPH_ERR_ARG;
  if (n == 0) return SPH_OK;
  if (!x || !y || !z || !keys) return SPH_ERR_ARG;
  int nb = (n + 255) / 256;
  if (nb > 148 * 8) nb = 148 * 8;
  sph::k_peano_int<<<nb, 256, 0, (cudaStream_t)stream>>>(n, x, y, z, bits, keys);
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}

extern "C" int cudasph_morton_keys(int n, const double *x, const double *y, const double *z, uint64_t *keys,
                                   double *box4, void *stream) {
  if (n <= 0) return n == 0 ? SPH_OK : SPH_ERR_ARG;
  if (!x || !y || !z || !keys || !box4) return SPH_ERR_ARG;
  double *part = nullptr;
  SPH_CUDA_TRY(cudaMallocAsync((void **)&part, 148 * 2 * 6 * sizeof(double), (cudaStream_t)stream));
  sph::morton_keys(n, nullptr, x, y, z, part, box4, keys, nullptr, (cudaStream_t)stream);
  SPH_CUDA_TRY(cudaFreeAsync(part, (cudaStream_t)stream));
  SPH_CUDA_TRY(cudaGetLastError());
  return SPH_OK;
}
