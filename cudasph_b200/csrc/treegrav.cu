// treegrav.cu -- tree-accelerated self-gravity (Barnes-Hut with quadrupoles)
// on the Morton order of the SPH phase, an opt-in alternative to the direct
// N^2 sum of sph_grav_kernel.cu:139-195 (grav_mode = SPH_GRAV_TREE).  The
// reference has no tree gravity; the direct sum stays the parity path and
// this mode trades a bounded force error (set by the opening angle theta)
// for O(N log N) work.
//
// Source tree: its own implicit hierarchy over the Morton order, finer than
// the SPH tree: level 0 nodes are runs of 8 consecutive particles, every
// level above groups 8 consecutive nodes.  Every node gets its mass M,
// centre of mass c, traceless quadrupole Q_ab = sum m (3 d_a d_b - |d|^2
// delta_ab) (d = x - c) and radius b = max |x - c|, all in FP64: level 0 from
// its particles, parents from their 8 children by the parallel-axis shift
// Q += M_k (3 s s - |s|^2 I), s = c_k - c, and b = max(|s| + b_k).  Eight
// lanes build one node (four nodes per warp).
//
// Walk: one warp per SPH leaf (a "group" of 32 targets, whose float box the
// SPH tree holds).  Each round pops up to four nodes and tests their 8
// children, one per lane: a child is accepted for the whole group when
// b < theta * dmin, dmin = distance from c to the group's box (so every
// particle of the node lies at least (1 - theta) dmin from every target).
// Accepted nodes go to a shared-memory list that all lanes sweep, two nodes
// per packed f32x2 instruction, with the softened monopole + quadrupole
//   a = M r / s^3 - Q r / s^5 + (5/2) (r.Q.r) r / s^7,
//   phi = -M / s - (1/2) (r.Q.r) / s^5,   r = c - x_i, s^2 = |r|^2 + eps^2;
// opened level-0 nodes go to a list of source runs swept 32 particles at a
// time with the Plummer pair term of the direct kernels; opened higher nodes
// are pushed.  Pair terms are FP32 on coordinates relative to the group's
// first particle (FP64 anchor); each sweep's FP32 partials fold into FP64.
#include "common.cuh"
#include "pairmath.cuh"

namespace sph {

constexpr int kGFan = 8;        // children per gravity-tree node, particles per level-0 node
constexpr int kGLevels = 12;    // supports up to 8^12 particles
constexpr int kTgWarps = 4;     // warps (groups) per block
constexpr int kTgList = 96;     // accepted-node list entries per warp
constexpr int kTgRuns = 64;     // opened level-0 runs buffered per warp (a round opens at most 32)
constexpr int kTgStack = 512;   // traversal stack entries per warp

struct GTree {
  int levels;
  int count[kGLevels];
  long long base[kGLevels];
};

static GTree gtree_layout(int n) {
  GTree g;
  long long off = 0;
  int c = (n + kGFan - 1) / kGFan;
  if (c < 1) c = 1;
  g.levels = 0;
  while (true) {
    g.count[g.levels] = c;
    g.base[g.levels] = off;
    off += c;
    g.levels++;
    if (c == 1 || g.levels == kGLevels) break;
    c = (c + kGFan - 1) / kGFan;
  }
  return g;
}

// nodes of the gravity tree over n particles (moment arrays hold this many)
long long gtree_nodes(int n) {
  const GTree g = gtree_layout(n);
  return g.base[g.levels - 1] + g.count[g.levels - 1];
}

// ------------------------------- moments ------------------------------------
// sums over the 8 lanes of a node (lanes 8k .. 8k+7)
__device__ __forceinline__ double seg_sum(double v) {
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double seg_max(double v) {
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// cm = {cx, cy, cz, M}; q0 = {Qxx, Qyy, Qzz, Qxy}; q1 = {Qxz, Qyz, b, 0}.
// Level 0 (parent = false): member k of node `node` is particle 8 node + k
// with src = {x, y, z, m}.  Parents: member k is child node 8 node + k of
// the level below, read from (ccm, cq0, cq1).
template <bool PARENT>
__global__ void k_gtree_moments(int nmember, int nnode, const double4 *__restrict__ src,
                                const double4 *__restrict__ ccm, const double4 *__restrict__ cq0,
                                const double4 *__restrict__ cq1, double4 *__restrict__ cm, double4 *__restrict__ q0,
                                double4 *__restrict__ q1) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int node = tid >> 3, k = tid & 7;
  // every lane of the warp takes part in the shuffles; nodes past the end are empty
  const bool live = node < nnode;
  const int mbr = node * kGFan + k;
  double4 m = make_double4(0, 0, 0, 0), a = m, b4 = m;
  if (live && mbr < nmember) {
    if (PARENT) {
      m = ccm[mbr];
      a = cq0[mbr];
      b4 = cq1[mbr];
    } else {
      m = src[mbr];
    }
  }
  const double M = seg_sum(m.w);
  double cx = seg_sum(m.w * m.x), cy = seg_sum(m.w * m.y), cz = seg_sum(m.w * m.z);
  const int first = (int)(lane_id() & ~7u);
  if (M > 0) {
    cx /= M; cy /= M; cz /= M;
  } else {  // massless node: centre at its first member
    cx = __shfl_sync(0xffffffffu, m.x, first);
    cy = __shfl_sync(0xffffffffu, m.y, first);
    cz = __shfl_sync(0xffffffffu, m.z, first);
  }
  const double sx = m.x - cx, sy = m.y - cy, sz = m.z - cz, s2 = sx * sx + sy * sy + sz * sz;
  double Q[6];
  Q[0] = seg_sum(a.x + m.w * (3 * sx * sx - s2));
  Q[1] = seg_sum(a.y + m.w * (3 * sy * sy - s2));
  Q[2] = seg_sum(a.z + m.w * (3 * sz * sz - s2));
  Q[3] = seg_sum(a.w + m.w * 3 * sx * sy);
  Q[4] = seg_sum(b4.x + m.w * 3 * sx * sz);
  Q[5] = seg_sum(b4.y + m.w * 3 * sy * sz);
  const double b = seg_max((live && mbr < nmember && m.w > 0) ? sqrt(s2) + (PARENT ? b4.z : 0.0) : 0.0);
  if (live && k == 0) {
    cm[node] = make_double4(cx, cy, cz, M);
    q0[node] = make_double4(Q[0], Q[1], Q[2], Q[3]);
    q1[node] = make_double4(Q[4], Q[5], b, 0.0);
  }
}

static int gtree_moments(const GTree &g, int n, const double4 *src, double4 *cm, double4 *q0, double4 *q1,
                         cudaStream_t st) {
  int launches = 0;
  {
    const int nn = g.count[0];
    k_gtree_moments<false><<<(nn * kGFan + 255) / 256, 256, 0, st>>>(n, nn, src, nullptr, nullptr, nullptr,
                                                                     cm + g.base[0], q0 + g.base[0], q1 + g.base[0]);
    launches++;
  }
  for (int l = 1; l < g.levels; l++) {
    const int nn = g.count[l];
    k_gtree_moments<true><<<(nn * kGFan + 255) / 256, 256, 0, st>>>(
        g.count[l - 1], nn, nullptr, cm + g.base[l - 1], q0 + g.base[l - 1], q1 + g.base[l - 1], cm + g.base[l],
        q0 + g.base[l], q1 + g.base[l]);
    launches++;
  }
  return launches;
}

// -------------------------------- the walk -----------------------------------
struct TreeGravArgs {
  TreeView t;          // the SPH tree: the groups' boxes (level 0)
  GTree g;             // the gravity tree
  const double4 *src;  // {x, y, z, m} per particle, tree order
  const double4 *cm, *q0, *q1;
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

struct TgSmem {
  NodePair list[kTgList / 2];
  float4 part[32];        // a sweep's staged source particles {x, y, z, m}
  int runs[kTgRuns];      // opened level-0 nodes awaiting their sweep
  int stack[kTgStack];
};

__global__ void __launch_bounds__(kTgWarps * 32) k_tree_gravity(TreeGravArgs a) {
  __shared__ TgSmem smem[kTgWarps];
  TgSmem &sm = smem[threadIdx.x >> 5];
  const int grp = a.leaf0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (grp >= a.leaf1) return;
  const unsigned lane = lane_id();
  const int n = a.t.n;
  const int s = grp * kLeaf + (int)lane;
  const bool valid = s < n;
  const double4 anc = a.src[grp * kLeaf];
  float xi = 0.f, yi = 0.f, zi = 0.f;
  if (valid) {
    const double4 p = a.src[s];
    xi = (float)(p.x - anc.x); yi = (float)(p.y - anc.y); zi = (float)(p.z - anc.z);
  }
  const float4 gl = a.t.lo[a.t.base[0] + grp], gh = a.t.hi[a.t.base[0] + grp];
  const float eps2 = a.eps2;
  const double theta = a.theta;
  double ax = 0, ay = 0, az = 0, ap = 0;
  int nlist = 0, nruns = 0;
  bool ok = true;

  const f32x2 X2 = pk2(xi, xi), Y2 = pk2(yi, yi), Z2 = pk2(zi, zi), E2 = pk2(eps2, eps2);
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
      const f32x2 t = mul2(rqr, inv5);                          // (r.Q.r) / s^5
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
  // sweep the buffered level-0 runs, 32 source particles at a time
  auto sweep_runs = [&]() {
    __syncwarp();
    for (int r0 = 0; r0 < nruns; r0 += 4) {
      const int r = r0 + (int)(lane >> 3);
      float4 q = make_float4(1e18f, 1e18f, 1e18f, 0.f);  // padding: far away, massless
      if (r < nruns) {
        const int sj = sm.runs[r] * kGFan + (int)(lane & 7u);
        if (sj < n) {
          const double4 p = a.src[sj];
          q = make_float4((float)(p.x - anc.x), (float)(p.y - anc.y), (float)(p.z - anc.z), (float)p.w);
        }
      }
      __syncwarp();
      sm.part[lane] = q;
      __syncwarp();
      float px = 0.f, py = 0.f, pz = 0.f, pp = 0.f;
#pragma unroll 8
      for (int k = 0; k < 32; k++) {
        const float4 p = sm.part[k];
        const float dx = p.x - xi, dy = p.y - yi, dz = p.z - zi;
        const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
        const float inv = rsqrt_f32(r2);
        const float sj = p.w * inv;
        const float s3 = sj * inv * inv;
        px = fmaf(dx, s3, px);
        py = fmaf(dy, s3, py);
        pz = fmaf(dz, s3, pz);
        pp -= sj;
      }
      ax += px; ay += py; az += pz; ap += pp;
    }
    nruns = 0;
    __syncwarp();
  };

  const int top = a.g.levels - 1;
  int sp = 1;
  if (lane == 0) sm.stack[0] = (top << 26);  // the root
  __syncwarp();
  // the root itself is tested like any child: pretend its parent is popped
  bool root_round = true;
  while (sp > 0) {
    // pop up to four nodes; lane L tests child (L & 7) of popped node (L >> 3)
    const int take = min(sp, 4);
    const int slot = (int)(lane >> 3);
    int e = 0;
    if (slot < take) e = sm.stack[sp - 1 - slot];
    sp -= take;
    __syncwarp();
    const int plevel = e >> 26, pnode = e & ((1 << 26) - 1);
    int level, child;
    bool exists;
    if (root_round) {  // the root: lane 0 only
      level = top;
      child = 0;
      exists = lane == 0;
      root_round = false;
    } else {
      level = plevel - 1;
      child = pnode * kGFan + (int)(lane & 7u);
      exists = slot < take && child < a.g.count[level];
    }
    bool accept = false;
    double4 c = make_double4(0, 0, 0, 0);
    if (exists) {
      const long long k = a.g.base[level] + child;
      c = a.cm[k];
      const double b = a.q1[k].z;
      exists = c.w > 0;
      const double ddx = fmax(fmax((double)gl.x - c.x, c.x - (double)gh.x), 0.0);
      const double ddy = fmax(fmax((double)gl.y - c.y, c.y - (double)gh.y), 0.0);
      const double ddz = fmax(fmax((double)gl.z - c.z, c.z - (double)gh.z), 0.0);
      accept = exists && b < theta * sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
    }
    // accepted nodes -> the list (swept first when it could overflow)
    const unsigned am = __ballot_sync(0xffffffffu, accept);
    if (am) {
      if (nlist + __popc(am) > kTgList) sweep_list();
      if (accept) {
        const long long k = a.g.base[level] + child;
        const double4 qa = a.q0[k], qb = a.q1[k];
        const int slot = nlist + __popc(am & ((1u << lane) - 1u));
        NodePair &e = sm.list[slot >> 1];
        const int h = slot & 1;
        e.x[h] = (float)(c.x - anc.x); e.y[h] = (float)(c.y - anc.y); e.z[h] = (float)(c.z - anc.z);
        e.m[h] = (float)c.w;
        e.qxx[h] = (float)qa.x; e.qyy[h] = (float)qa.y; e.qzz[h] = (float)qa.z; e.qxy[h] = (float)qa.w;
        e.qxz[h] = (float)qb.x; e.qyz[h] = (float)qb.y;
      }
      nlist += __popc(am);
      __syncwarp();
    }
    const bool open = exists && !accept;
    // opened level-0 nodes -> the run buffer
    const unsigned rm = __ballot_sync(0xffffffffu, open && level == 0);
    if (rm) {
      if (nruns + __popc(rm) > kTgRuns) sweep_runs();
      if (open && level == 0) sm.runs[nruns + __popc(rm & ((1u << lane) - 1u))] = child;
      nruns += __popc(rm);
      __syncwarp();
    }
    // opened higher nodes -> the stack
    const unsigned om = __ballot_sync(0xffffffffu, open && level > 0);
    const int cnt = __popc(om);
    if (sp + cnt > kTgStack) {
      ok = false;
      break;
    }
    if (open && level > 0) sm.stack[sp + cnt - 1 - __popc(om & ((1u << lane) - 1u))] = (level << 26) | child;
    sp += cnt;
    __syncwarp();
  }
  __syncwarp();
  if (nlist > 0) sweep_list();
  if (nruns > 0) sweep_runs();
  if (!ok && lane == 0) raise_flag(a.flags, SPH_FLAG_STACK_OVERFLOW);
  if (valid) a.out[s] = make_double4(a.G * ax, a.G * ay, a.G * az, a.G * ap);
}

// Shard `rank` of `world` computes the groups of its leaf range into `out`,
// zeroed first when world > 1 (the sum over shards is the whole field).
int launch_tree_gravity(const TreeView &t, const double4 *src, double4 *cm, double4 *q0, double4 *q1, double4 *out,
                        unsigned *flags, double eps, double theta, double G, int rank, int world, cudaStream_t st) {
  if (t.n <= 0) return 0;
  const GTree g = gtree_layout(t.n);
  int launches = gtree_moments(g, t.n, src, cm, q0, q1, st);
  if (world > 1) cudaMemsetAsync(out, 0, sizeof(double4) * t.n, st);
  long long l0, l1;
  shard_range(t.count[0], rank, world, l0, l1);
  if (l1 <= l0) return launches;
  TreeGravArgs a;
  a.t = t; a.g = g; a.src = src; a.cm = cm; a.q0 = q0; a.q1 = q1; a.out = out; a.flags = flags;
  a.eps2 = (float)(eps * eps); a.theta = (float)theta; a.G = G;
  a.leaf0 = (int)l0; a.leaf1 = (int)l1;
  const int warps = (int)(l1 - l0);
  k_tree_gravity<<<(warps + kTgWarps - 1) / kTgWarps, kTgWarps * 32, 0, st>>>(a);
  return launches + 1;
}

}  // namespace sph
