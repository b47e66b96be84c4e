// treegrav.cu -- tree-accelerated self-gravity (Barnes-Hut with quadrupoles)
// on the Morton order of the SPH phase, an opt-in alternative to the direct
// N^2 sum of sph_grav_kernel.cu:139-195 (grav_mode = SPH_GRAV_TREE).  The
// reference has no tree gravity; the direct sum stays the parity path and
// this mode trades a bounded force error (set by the opening angle theta)
// for O(N log N) work.
//
// Source tree: the binary radix tree of the sorted Morton keys (each
// internal node covers a contiguous run of particles that share a key
// prefix and splits it where the next key bit changes, so every node is a
// compact Morton cell or a half of one; equal keys split by index).  One
// thread per internal node finds its range and split from the keys alone
// (binary searches on common-prefix lengths).  Moments -- mass M, centre of
// mass c, traceless quadrupole Q_ab = sum m (3 d_a d_b - |d|^2 delta_ab)
// (d = x - c) and radius b = max |x - c| -- are FP64 and built bottom-up: one
// thread per particle climbs towards the root, and at every node the second
// of its two children's threads to arrive combines them (parallel-axis shift
// Q += M_k (3 s s - |s|^2 I), s = c_k - c; b = max(|s| + b_k)).
//
// Walk: one warp per SPH leaf of 32 targets, split into two groups where the
// leaf straddles a boundary of the curve (see "sub-groups" below); each group
// walks with the box of its own particles.  Each round pops up to sixteen
// internal nodes and tests their two children, one per lane: a child node is
// accepted for the whole group when b < theta * dmin, dmin = distance from c
// to the group's box (so every particle of the node lies at least
// (1 - theta) dmin from every target).  Accepted nodes go to a shared-memory
// list that all lanes sweep, two nodes per packed f32x2 instruction, with the
// softened monopole + quadrupole
//   a = M r / s^3 - Q r / s^5 + (5/2) (r.Q.r) r / s^7,
//   phi = -M / s - (1/2) (r.Q.r) / s^5,   r = c - x_i, s^2 = |r|^2 + eps^2;
// child particles and opened nodes of at most kBucket particles go to a ring
// of source particles swept 32 at a time with the Plummer pair term of the
// direct kernels; larger opened nodes are pushed.  Pair terms are FP32 on
// coordinates relative to the group's first particle (FP64 anchor); each
// sweep's FP32 partials fold into FP64.
#include <atomic>
#include <cstdint>

#include "common.cuh"
#include "pairmath.cuh"

namespace sph {

constexpr int kTgWarps = 4;     // warps (groups) per block
constexpr int kTgList = 96;     // accepted-node list entries per warp
constexpr int kTgRing = 576;    // source-particle ring per warp (a round adds at most 32 * kBucket)
constexpr int kTgStack = 1024;  // traversal stack entries per warp
constexpr int kBucket = 16;     // an opened node of at most this many particles is summed particle by particle
                                // (16 measured faster and more accurate than 4, 8 or 32 at N = 1M)
static_assert(32 * kBucket + 32 <= kTgRing, "a round's particles fit the ring");

// ------------------------------- workspace ----------------------------------
// per internal node (n - 1 of them): moments cm = {cx, cy, cz, M},
// q0 = {Qxx, Qyy, Qzz, Qxy}, q1 = {Qxz, Qyz, b, count}; children (an index
// >= 0 is an internal node, ~p a particle); particle range; parent; arrival
// counter of the bottom-up pass.  Per particle: its parent.  Per child slot
// of every internal node (2 (n - 1), indexed 2 node + side): what the walk
// tests that child with, so one load answers it.  One counter of the groups
// the walk has handed out.
struct __align__(16) ChildRec {
  float cx, cy, cz;  // centre of mass (float: the opening test only)
  float b;           // radius, rounded up; -1 for a massless node
  int ref;           // the child: an internal node, or ~particle
  int first, count;  // its particles
  int pad;
};
static_assert(sizeof(ChildRec) == 32, "one 32-byte record per child");

struct TgWork {
  double4 *cm, *q0, *q1;
  int2 *child, *range;
  int *parent, *lparent;
  unsigned *flag;
  ChildRec *rec;
  unsigned *next_group;
};

static size_t al256(size_t b) { return (b + 255) / 256 * 256; }

size_t tree_gravity_workspace_bytes(int n) {
  const size_t ni = n > 1 ? (size_t)n - 1 : 1;
  return 3 * al256(sizeof(double4) * ni) + 2 * al256(sizeof(int2) * ni) + al256(sizeof(int) * ni) +
         al256(sizeof(int) * (size_t)(n > 0 ? n : 1)) + al256(sizeof(unsigned) * ni) +
         al256(sizeof(ChildRec) * 2 * ni) + 256;
}

static TgWork carve(void *ws, int n) {
  const size_t ni = n > 1 ? (size_t)n - 1 : 1;
  char *p = (char *)ws;
  TgWork w;
  w.cm = (double4 *)p; p += al256(sizeof(double4) * ni);
  w.q0 = (double4 *)p; p += al256(sizeof(double4) * ni);
  w.q1 = (double4 *)p; p += al256(sizeof(double4) * ni);
  w.child = (int2 *)p; p += al256(sizeof(int2) * ni);
  w.range = (int2 *)p; p += al256(sizeof(int2) * ni);
  w.parent = (int *)p; p += al256(sizeof(int) * ni);
  w.lparent = (int *)p; p += al256(sizeof(int) * (size_t)(n > 0 ? n : 1));
  w.flag = (unsigned *)p; p += al256(sizeof(unsigned) * ni);
  w.rec = (ChildRec *)p; p += al256(sizeof(ChildRec) * 2 * ni);
  w.next_group = (unsigned *)p;
  return w;
}

// ------------------------------- topology ------------------------------------
// common-prefix length of keys i and j (64 + that of the indices for equal
// keys, -1 outside [0, n))
__device__ __forceinline__ int prefix(const uint64_t *__restrict__ k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint64_t a = k[i], b = k[j];
  if (a == b) return 64 + __clz((unsigned)(i ^ j));
  return __clzll((long long)(a ^ b));
}

__global__ void k_radix_tree(int n, const uint64_t *__restrict__ keys, TgWork w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  // direction of the node's range and its length by exponential + binary search
  const int d = prefix(keys, n, i, i + 1) - prefix(keys, n, i, i - 1) >= 0 ? 1 : -1;
  const int dmin = prefix(keys, n, i, i - d);
  int lmax = 2;
  while (prefix(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (prefix(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  // the split: the last position sharing more than the node's common prefix
  const int dnode = prefix(keys, n, i, j);
  int s = 0;
  for (int div = 2;; div <<= 1) {
    const int t = (l + div - 1) / div;
    if (prefix(keys, n, i, i + (s + t) * d) > dnode) s += t;
    if (t == 1) break;
  }
  const int gamma = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int left = (lo == gamma) ? ~gamma : gamma;
  const int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
  w.child[i] = make_int2(left, right);
  w.range[i] = make_int2(lo, hi);
  // a particle child's record is complete here; an internal child's is
  // finished by the moments pass
  const int cref[2] = {left, right};
#pragma unroll
  for (int k = 0; k < 2; k++) {
    ChildRec r;
    r.cx = r.cy = r.cz = 0.f;
    r.b = 0.f;
    r.ref = cref[k];
    r.first = cref[k] < 0 ? ~cref[k] : 0;
    r.count = 1;
    r.pad = 0;
    w.rec[2 * i + k] = r;
  }
  if (left < 0) w.lparent[gamma] = i;
  else w.parent[gamma] = i;
  if (right < 0) w.lparent[gamma + 1] = i;
  else w.parent[gamma + 1] = i;
  if (i == 0) w.parent[0] = -1;  // node 0 covers [0, n) and is the root
  w.flag[i] = 0u;
}

// a child's moments: a particle {x, m}, or an internal node written by
// another thread of this launch (read from L2, past the incoherent L1)
__device__ __forceinline__ void child_moments(int ref, const double4 *__restrict__ src, const TgWork &w, double4 &c,
                                              double4 &qa, double4 &qb) {
  if (ref < 0) {
    c = src[~ref];
    qa = make_double4(0, 0, 0, 0);
    qb = make_double4(0, 0, 0, 1);
    return;
  }
  const double2 *pc = reinterpret_cast<const double2 *>(w.cm + ref);
  const double2 *pa = reinterpret_cast<const double2 *>(w.q0 + ref);
  const double2 *pb = reinterpret_cast<const double2 *>(w.q1 + ref);
  const double2 c0 = __ldcg(pc), c1 = __ldcg(pc + 1), a0 = __ldcg(pa), a1 = __ldcg(pa + 1), b0 = __ldcg(pb),
                b1 = __ldcg(pb + 1);
  c = make_double4(c0.x, c0.y, c1.x, c1.y);
  qa = make_double4(a0.x, a0.y, a1.x, a1.y);
  qb = make_double4(b0.x, b0.y, b1.x, b1.y);
}

__global__ void k_tree_moments(int n, const double4 *__restrict__ src, TgWork w) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int node = w.lparent[p];
  while (node >= 0) {
    __threadfence();  // this thread's node writes (previous pass) before its arrival count
    if (atomicAdd(&w.flag[node], 1u) == 0u) return;  // the other child's thread combines
    const int2 ch = w.child[node];
    double4 ca, qaa, qab, cb, qba, qbb;
    child_moments(ch.x, src, w, ca, qaa, qab);
    child_moments(ch.y, src, w, cb, qba, qbb);
    const double M = ca.w + cb.w;
    double cx, cy, cz;
    if (M > 0) {
      cx = (ca.w * ca.x + cb.w * cb.x) / M;
      cy = (ca.w * ca.y + cb.w * cb.y) / M;
      cz = (ca.w * ca.z + cb.w * cb.z) / M;
    } else {
      cx = ca.x; cy = ca.y; cz = ca.z;
    }
    double Q[6] = {qaa.x + qba.x, qaa.y + qba.y, qaa.z + qba.z, qaa.w + qba.w, qab.x + qbb.x, qab.y + qbb.y};
    double b = 0;
    const double4 *cs[2] = {&ca, &cb};
    const double bs[2] = {qab.z, qbb.z};
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const double4 &ck = *cs[k];
      const double sx = ck.x - cx, sy = ck.y - cy, sz = ck.z - cz, s2 = sx * sx + sy * sy + sz * sz;
      Q[0] += ck.w * (3 * sx * sx - s2);
      Q[1] += ck.w * (3 * sy * sy - s2);
      Q[2] += ck.w * (3 * sz * sz - s2);
      Q[3] += ck.w * 3 * sx * sy;
      Q[4] += ck.w * 3 * sx * sz;
      Q[5] += ck.w * 3 * sy * sz;
      if (ck.w > 0) b = fmax(b, sqrt(s2) + bs[k]);
    }
    const int2 r = w.range[node];
    w.cm[node] = make_double4(cx, cy, cz, M);
    w.q0[node] = make_double4(Q[0], Q[1], Q[2], Q[3]);
    w.q1[node] = make_double4(Q[4], Q[5], b, (double)(r.y - r.x + 1));
    const int up = w.parent[node];
    if (up >= 0) {
      ChildRec rec;
      rec.cx = (float)cx; rec.cy = (float)cy; rec.cz = (float)cz;
      rec.b = M > 0 ? __double2float_ru(b) : -1.f;
      rec.ref = node;
      rec.first = r.x;
      rec.count = r.y - r.x + 1;
      rec.pad = 0;
      w.rec[2 * up + (w.child[up].x == node ? 0 : 1)] = rec;
    }
    node = up;
  }
}

// -------------------------------- the walk -----------------------------------
struct TreeGravArgs {
  TreeView t;          // the SPH tree: its leaves are the groups
  TgWork w;            // the gravity tree
  const double4 *src;  // {x, y, z, m} per particle, tree order
  const uint64_t *keys;  // the sorted keys of that order
  double4 *out;        // {gx, gy, gz, phi}
  unsigned *flags;
  float eps2, theta;
  double G;
  int leaf0, leaf1;    // groups (SPH leaves) of this launch
};

// Accepted nodes are stored in pairs, component-interleaved so that one
// packed f32x2 instruction advances both nodes of a pair against the lane's
// target: pair j holds entries 2j and 2j+1 as {a0, a1} for each component
// (coordinates relative to the group anchor), five 16-byte loads per pair.
struct __align__(16) NodePair {
  float x[2], y[2], z[2], m[2], qxx[2], qyy[2], qzz[2], qxy[2], qxz[2], qyz[2];
};
static_assert(sizeof(NodePair) == 80, "five 16-byte loads per pair");

// A ring sweep's 32 staged source particles, in pairs laid out the same way
// (particles 2j and 2j+1 as {p0, p1} per component).
struct __align__(16) PartPair {
  float x[2], y[2], z[2], m[2];
};
static_assert(sizeof(PartPair) == 32, "two 16-byte loads per pair");

struct TgSmem {
  NodePair list[kTgList / 2];
  PartPair part[16];     // a sweep's staged source particles
  int ring[kTgRing];     // source particles awaiting their sweep
  int stack[kTgStack];   // internal nodes to open
};

// ---- sub-groups ----
// A leaf of 32 consecutive particles can straddle a boundary of the curve and
// then spans two distant clumps; its box, and with it the set of opened
// nodes, is then far larger than either clump's (such a group sums most of a
// star directly).  The leaf is therefore split where its keys split in the
// radix tree (the first particle with the highest differing key bit set),
// up to kTgSplitLevels times, wherever the larger half's extent is below
// kTgSplitRatio of the whole part's: a compact group is not split, a
// straddling one walks once per clump, with that clump's box and anchor.
// Measured on the two-polytrope state (N = 262,144 and 1,048,576) and the
// 4M cold sphere: ratio 0.35 with one level is fastest (1M, theta 0.5:
// 12.0 ms unsplit, 5.6 ms); 0.5 or more levels also split compact leaves
// (6.4 - 6.7 ms), 0.25 or less leaves the costliest straddlers whole (13 ms).
constexpr int kTgSplitLevels = 1;
constexpr double kTgSplitRatio = 0.35;

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// bounding box of the lanes in `mask` (lo, hi; every lane gets the result)
__device__ __forceinline__ void lanes_box(bool in, double x, double y, double z, double *lo, double *hi) {
  lo[0] = warp_min(in ? x : 1e300); hi[0] = warp_max(in ? x : -1e300);
  lo[1] = warp_min(in ? y : 1e300); hi[1] = warp_max(in ? y : -1e300);
  lo[2] = warp_min(in ? z : 1e300); hi[2] = warp_max(in ? z : -1e300);
}

__device__ __forceinline__ double box_extent(const double *lo, const double *hi) {
  return fmax(fmax(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
}

// lanes [first, last] of the part that starts at lane `first` in the
// part-start mask `starts` (last = the lane before the next start, or cnt - 1)
__device__ __forceinline__ int part_last(unsigned starts, int first, int cnt) {
  const unsigned above = first < 31 ? starts & (0xffffffffu << (first + 1)) : 0u;
  return above ? __ffs(above) - 2 : cnt - 1;
}

__device__ __forceinline__ unsigned lane_range(int lo, int hi) {  // lanes lo..hi
  const unsigned up = hi >= 31 ? 0xffffffffu : ((1u << (hi + 1)) - 1u);
  return up & ~((1u << lo) - 1u);
}

// the walk of one group (SPH leaf `grp`) by the calling warp
__device__ __forceinline__ void tree_group(const TreeGravArgs &a, TgSmem &sm, int grp) {
  const unsigned lane = lane_id();
  const int n = a.t.n;
  const int s = grp * kLeaf + (int)lane;
  const int cnt = min(kLeaf, n - grp * kLeaf);  // targets of this group (lanes 0 .. cnt-1)
  const bool valid = (int)lane < cnt;
  const double4 me = valid ? a.src[s] : a.src[grp * kLeaf];
  const uint64_t key = valid ? a.keys[s] : 0ull;

  // the group's parts (bit L of `starts` set: a part starts at lane L)
  unsigned starts = 1u;
  for (int lev = 0; lev < kTgSplitLevels; lev++) {
    unsigned next = starts;
    for (unsigned m = starts; m; m &= m - 1u) {
      const int f = __ffs(m) - 1, l = part_last(starts, f, cnt);
      if (l <= f) continue;
      const uint64_t kf = __shfl_sync(0xffffffffu, key, f), kl = __shfl_sync(0xffffffffu, key, l);
      if (kf == kl) continue;
      const int top = 63 - __clzll((long long)(kf ^ kl));
      const unsigned in = lane_range(f, l);
      const unsigned upper = __ballot_sync(0xffffffffu, ((key >> top) & 1ull) != 0ull) & in;
      const int sp = __ffs(upper) - 1;  // first lane of the upper half (kl has the bit: sp in (f, l])
      const bool inp = (in >> lane) & 1u, ina = inp && (int)lane < sp, inb = inp && (int)lane >= sp;
      double plo[3], phi[3], alo[3], ahi[3], blo[3], bhi[3];
      lanes_box(inp, me.x, me.y, me.z, plo, phi);
      lanes_box(ina, me.x, me.y, me.z, alo, ahi);
      lanes_box(inb, me.x, me.y, me.z, blo, bhi);
      if (fmax(box_extent(alo, ahi), box_extent(blo, bhi)) < kTgSplitRatio * box_extent(plo, phi))
        next |= 1u << sp;
    }
    starts = next;
  }

  const float eps2 = a.eps2;
  const float theta = a.theta;
  double ax = 0, ay = 0, az = 0, ap = 0;
  int nlist = 0;
  unsigned head = 0, tail = 0;  // ring positions (mod kTgRing)
  bool ok = true;
  // per part: anchor, the lane's target relative to it, the part's box
  double4 anc = me;
  float xi = 0.f, yi = 0.f, zi = 0.f;
  double glo[3] = {0, 0, 0}, ghi[3] = {0, 0, 0};
  float flo[3] = {0.f, 0.f, 0.f}, fhi[3] = {0.f, 0.f, 0.f};  // the box rounded outward
  f32x2 X2 = 0ull, Y2 = 0ull, Z2 = 0ull;

  const f32x2 E2 = pk2(eps2, eps2);
  const f32x2 HALF5 = pk2(2.5f, 2.5f), MHALF = pk2(-0.5f, -0.5f), MONE = pk2(-1.f, -1.f);
  auto sweep_list = [&]() {
    __syncwarp();  // entries written by every lane are visible
    if (nlist & 1) {  // pad an odd list with a massless node far away
      if (lane == 0) {
        NodePair &e = sm.list[nlist >> 1];
        e.x[1] = e.y[1] = e.z[1] = 1e18f;
        e.m[1] = e.qxx[1] = e.qyy[1] = e.qzz[1] = e.qxy[1] = e.qxz[1] = e.qyz[1] = 0.f;
      }
      __syncwarp();
    }
    f32x2 px = 0ull, py = 0ull, pz = 0ull, pp = 0ull;
    const int npair = (nlist + 1) >> 1;
#pragma unroll 2
    for (int k = 0; k < npair; k++) {
      const NodePair &e = sm.list[k];
      const f32x2 ex = *reinterpret_cast<const f32x2 *>(e.x), ey = *reinterpret_cast<const f32x2 *>(e.y);
      const f32x2 ez = *reinterpret_cast<const f32x2 *>(e.z), em = *reinterpret_cast<const f32x2 *>(e.m);
      const f32x2 qxx = *reinterpret_cast<const f32x2 *>(e.qxx), qyy = *reinterpret_cast<const f32x2 *>(e.qyy);
      const f32x2 qzz = *reinterpret_cast<const f32x2 *>(e.qzz), qxy = *reinterpret_cast<const f32x2 *>(e.qxy);
      const f32x2 qxz = *reinterpret_cast<const f32x2 *>(e.qxz), qyz = *reinterpret_cast<const f32x2 *>(e.qyz);
      const f32x2 rx = sub2(ex, X2), ry = sub2(ey, Y2), rz = sub2(ez, Z2);
      f32x2 s2 = fma2(rx, rx, E2);
      s2 = fma2(ry, ry, s2);
      s2 = fma2(rz, rz, s2);
      float sa, sb;
      upk2(s2, sa, sb);
      const f32x2 inv = pk2(rsqrt_f32(sa), rsqrt_f32(sb));
      const f32x2 inv2 = mul2(inv, inv);
      const f32x2 inv3 = mul2(inv2, inv), inv5 = mul2(inv3, inv2);
      const f32x2 qx = fma2(qxz, rz, fma2(qxy, ry, mul2(qxx, rx)));
      const f32x2 qy = fma2(qyz, rz, fma2(qyy, ry, mul2(qxy, rx)));
      const f32x2 qz = fma2(qzz, rz, fma2(qyz, ry, mul2(qxz, rx)));
      const f32x2 rqr = fma2(rz, qz, fma2(ry, qy, mul2(rx, qx)));
      const f32x2 t = mul2(rqr, inv5);                             // (r.Q.r) / s^5
      const f32x2 c = fma2(HALF5, mul2(t, inv2), mul2(em, inv3));  // M / s^3 + (5/2) (r.Q.r) / s^7
      const f32x2 ni5 = mul2(inv5, MONE);
      px = fma2(ni5, qx, fma2(c, rx, px));
      py = fma2(ni5, qy, fma2(c, ry, py));
      pz = fma2(ni5, qz, fma2(c, rz, pz));
      pp = fma2(MHALF, t, sub2(pp, mul2(em, inv)));
    }
    float a0, a1;
    upk2(px, a0, a1); ax += (double)a0 + (double)a1;
    upk2(py, a0, a1); ay += (double)a0 + (double)a1;
    upk2(pz, a0, a1); az += (double)a0 + (double)a1;
    upk2(pp, a0, a1); ap += (double)a0 + (double)a1;
    nlist = 0;
    __syncwarp();  // every lane is done reading before the list is refilled
  };
  // sweep 32 ring entries from `head` (fewer at the end: the rest padded far
  // away and massless), two sources per packed instruction
  auto sweep_chunk = [&](unsigned cnt) {
    __syncwarp();
    float qx = 1e18f, qy = 1e18f, qz = 1e18f, qm = 0.f;
    if (lane < cnt) {
      const double4 p = a.src[sm.ring[(head + lane) % kTgRing]];
      qx = (float)(p.x - anc.x); qy = (float)(p.y - anc.y); qz = (float)(p.z - anc.z); qm = (float)p.w;
    }
    PartPair &d = sm.part[lane >> 1];
    d.x[lane & 1] = qx; d.y[lane & 1] = qy; d.z[lane & 1] = qz; d.m[lane & 1] = qm;
    __syncwarp();
    f32x2 px = 0ull, py = 0ull, pz = 0ull, pp = 0ull;
#pragma unroll 4
    for (int k = 0; k < 16; k++) {
      const PartPair &e = sm.part[k];
      const f32x2 ex = *reinterpret_cast<const f32x2 *>(e.x), ey = *reinterpret_cast<const f32x2 *>(e.y);
      const f32x2 ez = *reinterpret_cast<const f32x2 *>(e.z), em = *reinterpret_cast<const f32x2 *>(e.m);
      const f32x2 dx = sub2(ex, X2), dy = sub2(ey, Y2), dz = sub2(ez, Z2);
      f32x2 r2 = fma2(dx, dx, E2);
      r2 = fma2(dy, dy, r2);
      r2 = fma2(dz, dz, r2);
      float ra, rb;
      upk2(r2, ra, rb);
      const f32x2 inv = pk2(rsqrt_f32(ra), rsqrt_f32(rb));
      const f32x2 sj = mul2(em, inv);
      const f32x2 s3 = mul2(mul2(sj, inv), inv);
      px = fma2(dx, s3, px);
      py = fma2(dy, s3, py);
      pz = fma2(dz, s3, pz);
      pp = sub2(pp, sj);
    }
    float a0, a1;
    upk2(px, a0, a1); ax += (double)a0 + (double)a1;
    upk2(py, a0, a1); ay += (double)a0 + (double)a1;
    upk2(pz, a0, a1); az += (double)a0 + (double)a1;
    upk2(pp, a0, a1); ap += (double)a0 + (double)a1;
    head += cnt;
    __syncwarp();
  };

  for (unsigned parts = starts; parts && ok; parts &= parts - 1u) {
    const int f = __ffs(parts) - 1, l = part_last(starts, f, cnt);
    const bool mine = (int)lane >= f && (int)lane <= l;
    anc.x = __shfl_sync(0xffffffffu, me.x, f);
    anc.y = __shfl_sync(0xffffffffu, me.y, f);
    anc.z = __shfl_sync(0xffffffffu, me.z, f);
    lanes_box(mine, me.x, me.y, me.z, glo, ghi);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      flo[d] = __double2float_rd(glo[d]);
      fhi[d] = __double2float_ru(ghi[d]);
    }
    xi = (float)(me.x - anc.x); yi = (float)(me.y - anc.y); zi = (float)(me.z - anc.z);
    X2 = pk2(xi, xi); Y2 = pk2(yi, yi); Z2 = pk2(zi, zi);
    const double sx = ax, sy = ay, sz = az, sph = ap;  // lanes of other parts keep these

    int sp = 0;
    if (n < 2) {  // a single particle: no internal node
      if (lane == 0) sm.ring[0] = 0;
      tail = 1;
    } else {
      if (lane == 0) sm.stack[0] = 0;  // the root covers [0, n)
      sp = 1;
    }
    __syncwarp();
    while (sp > 0) {
      // pop up to sixteen nodes; lane L tests child (L & 1) of popped node (L >> 1)
      const int take = min(sp, 16);
      const int slot = (int)(lane >> 1);
      int node = -1;
      if (slot < take) node = sm.stack[sp - 1 - slot];
      sp -= take;
      __syncwarp();
      const bool live = slot < take;
      float4 r0 = make_float4(0.f, 0.f, 0.f, -1.f), r1 = make_float4(0.f, 0.f, 0.f, 0.f);
      if (live) {  // the child's record {cx, cy, cz, b}, {ref, first, count, -}
        const float4 *rp = reinterpret_cast<const float4 *>(a.w.rec + 2 * node + (int)(lane & 1u));
        r0 = __ldg(rp);
        r1 = __ldg(rp + 1);
      }
      const int ref = __float_as_int(r1.x);
      bool accept = false, open = false;
      int p0 = 0, pc = 0;  // source particles this lane hands to the ring
      if (live && ref < 0) {
        p0 = ~ref;
        pc = 1;
      } else if (live && r0.w >= 0.f) {
        const float ddx = fmaxf(fmaxf(flo[0] - r0.x, r0.x - fhi[0]), 0.f);
        const float ddy = fmaxf(fmaxf(flo[1] - r0.y, r0.y - fhi[1]), 0.f);
        const float ddz = fmaxf(fmaxf(flo[2] - r0.z, r0.z - fhi[2]), 0.f);
        accept = r0.w < theta * sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
        if (!accept) {
          const int count = __float_as_int(r1.z);
          if (count <= kBucket) {
            p0 = __float_as_int(r1.y);
            pc = count;
          } else {
            open = true;
          }
        }
      }
      // accepted nodes -> the list (swept first when it could overflow)
      const unsigned am = __ballot_sync(0xffffffffu, accept);
      if (am) {
        if (nlist + __popc(am) > kTgList) sweep_list();
        if (accept) {
          const double4 c = a.w.cm[ref], qa = a.w.q0[ref], qb = a.w.q1[ref];
          const int k = nlist + __popc(am & ((1u << lane) - 1u));
          NodePair &e = sm.list[k >> 1];
          const int h = k & 1;
          e.x[h] = (float)(c.x - anc.x); e.y[h] = (float)(c.y - anc.y); e.z[h] = (float)(c.z - anc.z);
          e.m[h] = (float)c.w;
          e.qxx[h] = (float)qa.x; e.qyy[h] = (float)qa.y; e.qzz[h] = (float)qa.z; e.qxy[h] = (float)qa.w;
          e.qxz[h] = (float)qb.x; e.qyz[h] = (float)qb.y;
        }
        nlist += __popc(am);
        __syncwarp();
      }
      // particles -> the ring (warp prefix sum of the counts), then every full chunk is swept
      int incl = pc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)lane >= o) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      if (total > 0) {
        for (int k = 0; k < pc; k++) sm.ring[(tail + (unsigned)(incl - pc + k)) % kTgRing] = p0 + k;
        tail += (unsigned)total;
        while (tail - head >= 32u) sweep_chunk(32u);
      }
      // opened larger nodes -> the stack
      const unsigned om = __ballot_sync(0xffffffffu, open);
      const int nopen = __popc(om);
      if (sp + nopen > kTgStack) {
        ok = false;
        break;
      }
      if (open) sm.stack[sp + nopen - 1 - __popc(om & ((1u << lane) - 1u))] = ref;
      sp += nopen;
      __syncwarp();
    }
    __syncwarp();
    if (nlist > 0) sweep_list();
    if (tail != head) sweep_chunk(tail - head);
    if (!mine) {
      ax = sx; ay = sy; az = sz; ap = sph;
    }
  }
  if (!ok && lane == 0) raise_flag(a.flags, SPH_FLAG_STACK_OVERFLOW);
  if (valid) a.out[s] = make_double4(a.G * ax, a.G * ay, a.G * az, a.G * ap);
}

// Persistent walk: one block per resident slot, and every warp takes the next
// group from a counter until none is left.  Group costs differ several-fold
// (a leaf in a sparse outer layer opens more nodes), and handing them out
// one at a time lets a long group overlap the rest instead of ending the
// launch alone on its SM.
__global__ void __launch_bounds__(kTgWarps * 32, 5) k_tree_gravity(TreeGravArgs a) {
  __shared__ TgSmem smem[kTgWarps];
  TgSmem &sm = smem[threadIdx.x >> 5];
  const unsigned groups = (unsigned)(a.leaf1 - a.leaf0);
  for (;;) {
    unsigned g = 0;
    if (lane_id() == 0) g = atomicAdd(a.w.next_group, 1u);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= groups) break;
    tree_group(a, sm, a.leaf0 + (int)g);
  }
}

// keys: the sorted Morton keys of the current particle order (the sort's
// output); ws: tree_gravity_workspace_bytes(n) bytes.  Shard `rank` of
// `world` computes the groups of its leaf range into `out`, zeroed first
// when world > 1 (the sum over shards is the whole field).
int launch_tree_gravity(const TreeView &t, const uint64_t *keys, const double4 *src, void *ws, double4 *out,
                        unsigned *flags, double eps, double theta, double G, int rank, int world, cudaStream_t st) {
  const int n = t.n;
  if (n <= 0) return 0;
  const TgWork w = carve(ws, n);
  int launches = 0;
  if (n > 1) {
    k_radix_tree<<<(n - 1 + 255) / 256, 256, 0, st>>>(n, keys, w);
    k_tree_moments<<<(n + 255) / 256, 256, 0, st>>>(n, src, w);
    launches += 2;
  }
  if (world > 1) cudaMemsetAsync(out, 0, sizeof(double4) * n, st);
  long long l0, l1;
  shard_range(t.count[0], rank, world, l0, l1);
  if (l1 <= l0) return launches;
  TreeGravArgs a;
  a.t = t; a.w = w; a.src = src; a.keys = keys; a.out = out; a.flags = flags;
  a.eps2 = (float)(eps * eps); a.theta = (float)theta; a.G = G;
  a.leaf0 = (int)l0; a.leaf1 = (int)l1;
  const int warps = (int)(l1 - l0);
  // resident blocks per SM (the same on every device of one architecture),
  // looked up once; contexts on several host threads may race to store it
  static std::atomic<int> cached_per_sm{0};
  int per_sm = cached_per_sm.load(std::memory_order_relaxed);
  if (per_sm == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tree_gravity, kTgWarps * 32, 0) == cudaSuccess &&
        per_sm >= 1) {
      cached_per_sm.store(per_sm, std::memory_order_relaxed);
    } else {
      // a failed query is neither cached nor left pending: the caller's
      // post-launch error check must only see the launch's own status
      (void)cudaGetLastError();
      per_sm = 1;
    }
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    (void)cudaGetLastError();
    sms = 148;
  }
  const int blocks = min((warps + kTgWarps - 1) / kTgWarps, sms * max(per_sm, 1));
  cudaMemsetAsync(w.next_group, 0, sizeof(unsigned), st);
  k_tree_gravity<<<blocks, kTgWarps * 32, 0, st>>>(a);
  return launches + 1;
}

}  // namespace sph
