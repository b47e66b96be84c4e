// treegrav.cu -- tree-accelerated self-gravity (Barnes-Hut with quadrupoles)
// on the Morton tree of the SPH phase, an opt-in alternative to the direct
// N^2 sum of sph_grav_kernel.cu:139-195 (grav_mode = SPH_GRAV_TREE).  The
// reference has no tree gravity; the direct sum stays the parity path and
// this mode trades a bounded force error (set by the opening angle theta)
// for O(N log N) work.
//
// Moments: every node of the implicit tree (leaves of 32 particles, fan-out
// 32) gets its mass M, centre of mass c, traceless quadrupole
// Q_ab = sum m (3 d_a d_b - |d|^2 delta_ab) (d = x - c) and the radius
// b = max |x - c| of its particles, all in FP64: leaves by one warp
// reduction over their particles, parents from their 32 children by the
// parallel-axis shift Q += M_k (3 s s - |s|^2 I), s = c_k - c, and
// b = max(|s| + b_k).
//
// Walk: one warp per leaf ("group" of 32 targets).  A node is accepted for
// the whole group when b < theta * dmin, dmin = distance from c to the
// group's bounding box (so every particle of the node lies at least
// (1 - theta) dmin from every target); accepted nodes go to a shared-memory
// list that all lanes sweep with the softened monopole + quadrupole
//   a = M r / s^3 - Q r / s^5 + (5/2) (r.Q.r) r / s^7,
//   phi = -M / s - (1/2) (r.Q.r) / s^5,   r = c - x_i, s^2 = |r|^2 + eps^2;
// leaves that are not accepted are summed particle by particle with the
// Plummer pair term of the direct kernels.  Pair terms are FP32 on
// coordinates relative to the group's first particle (FP64 anchor); each
// sweep's FP32 partial sums fold into FP64 accumulators.
#include "common.cuh"
#include "pairmath.cuh"

namespace sph {

constexpr int kTgWarps = 4;    // warps (groups) per block
constexpr int kTgList = 64;    // accepted-node list entries per warp
constexpr int kTgStack = 256;  // traversal stack entries per warp

// ------------------------------- moments ------------------------------------
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// cm = {cx, cy, cz, M}; q0 = {Qxx, Qyy, Qzz, Qxy}; q1 = {Qxz, Qyz, b, 0}
__device__ __forceinline__ void write_node(double4 *cm, double4 *q0, double4 *q1, int k, double M, double cx,
                                           double cy, double cz, const double *Q, double b) {
  cm[k] = make_double4(cx, cy, cz, M);
  q0[k] = make_double4(Q[0], Q[1], Q[2], Q[3]);
  q1[k] = make_double4(Q[4], Q[5], b, 0.0);
}

__global__ void k_leaf_moments(int n, int nleaf, const double4 *__restrict__ src, double4 *__restrict__ cm,
                               double4 *__restrict__ q0, double4 *__restrict__ q1) {
  const int leaf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (leaf >= nleaf) return;
  const int s = leaf * kLeaf + (int)lane_id();
  double4 p = make_double4(0, 0, 0, 0);
  if (s < n) p = src[s];
  const double M = warp_sum_d(p.w);
  double cx = warp_sum_d(p.w * p.x), cy = warp_sum_d(p.w * p.y), cz = warp_sum_d(p.w * p.z);
  if (M > 0) {
    cx /= M; cy /= M; cz /= M;
  } else {  // massless leaf: centre at its first particle
    cx = __shfl_sync(0xffffffffu, p.x, 0);
    cy = __shfl_sync(0xffffffffu, p.y, 0);
    cz = __shfl_sync(0xffffffffu, p.z, 0);
  }
  const double dx = p.x - cx, dy = p.y - cy, dz = p.z - cz, d2 = dx * dx + dy * dy + dz * dz;
  double Q[6];
  Q[0] = warp_sum_d(p.w * (3 * dx * dx - d2));
  Q[1] = warp_sum_d(p.w * (3 * dy * dy - d2));
  Q[2] = warp_sum_d(p.w * (3 * dz * dz - d2));
  Q[3] = warp_sum_d(p.w * 3 * dx * dy);
  Q[4] = warp_sum_d(p.w * 3 * dx * dz);
  Q[5] = warp_sum_d(p.w * 3 * dy * dz);
  const double b = warp_max_d(s < n ? sqrt(d2) : 0.0);
  if (lane_id() == 0) write_node(cm, q0, q1, leaf, M, cx, cy, cz, Q, b);
}

__global__ void k_parent_moments(int nchild, int nparent, const double4 *__restrict__ ccm,
                                 const double4 *__restrict__ cq0, const double4 *__restrict__ cq1,
                                 double4 *__restrict__ pcm, double4 *__restrict__ pq0, double4 *__restrict__ pq1) {
  const int node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (node >= nparent) return;
  const int c = node * kFan + (int)lane_id();
  double4 m = make_double4(0, 0, 0, 0), a = m, b4 = m;
  if (c < nchild) {
    m = ccm[c];
    a = cq0[c];
    b4 = cq1[c];
  }
  const double M = warp_sum_d(m.w);
  double cx = warp_sum_d(m.w * m.x), cy = warp_sum_d(m.w * m.y), cz = warp_sum_d(m.w * m.z);
  if (M > 0) {
    cx /= M; cy /= M; cz /= M;
  } else {
    cx = __shfl_sync(0xffffffffu, m.x, 0);
    cy = __shfl_sync(0xffffffffu, m.y, 0);
    cz = __shfl_sync(0xffffffffu, m.z, 0);
  }
  const double sx = m.x - cx, sy = m.y - cy, sz = m.z - cz, s2 = sx * sx + sy * sy + sz * sz;
  double Q[6];
  Q[0] = warp_sum_d(a.x + m.w * (3 * sx * sx - s2));
  Q[1] = warp_sum_d(a.y + m.w * (3 * sy * sy - s2));
  Q[2] = warp_sum_d(a.z + m.w * (3 * sz * sz - s2));
  Q[3] = warp_sum_d(a.w + m.w * 3 * sx * sy);
  Q[4] = warp_sum_d(b4.x + m.w * 3 * sx * sz);
  Q[5] = warp_sum_d(b4.y + m.w * 3 * sy * sz);
  const double b = warp_max_d((c < nchild && m.w > 0) ? sqrt(s2) + b4.z : 0.0);
  if (lane_id() == 0) write_node(pcm, pq0, pq1, node, M, cx, cy, cz, Q, b);
}

int tree_moments(const TreeView &t, const double4 *src, double4 *cm, double4 *q0, double4 *q1, cudaStream_t st) {
  int launches = 0;
  const int nleaf = t.count[0];
  k_leaf_moments<<<(nleaf * 32 + 255) / 256, 256, 0, st>>>(t.n, nleaf, src, cm + t.base[0], q0 + t.base[0],
                                                          q1 + t.base[0]);
  launches++;
  for (int l = 1; l < t.levels; l++) {
    const int np = t.count[l];
    k_parent_moments<<<(np * 32 + 255) / 256, 256, 0, st>>>(t.count[l - 1], np, cm + t.base[l - 1],
                                                           q0 + t.base[l - 1], q1 + t.base[l - 1], cm + t.base[l],
                                                           q0 + t.base[l], q1 + t.base[l]);
    launches++;
  }
  return launches;
}

// -------------------------------- the walk -----------------------------------
struct TreeGravArgs {
  TreeView t;
  const double4 *src;  // {x, y, z, m} per particle, tree order
  const double4 *cm, *q0, *q1;
  double4 *out;        // {gx, gy, gz, phi}
  unsigned *flags;
  float eps2, theta;
  double G;
  int leaf0, leaf1;    // groups (leaves) of this launch
};

struct NodeEntry {  // an accepted node, coordinates relative to the group anchor
  float x, y, z, m, qxx, qyy, qzz, qxy, qxz, qyz;
};

struct TgSmem {
  NodeEntry list[kTgList];
  float4 leaf[kLeaf];  // staged particles of an opened leaf {x, y, z, m}
  int stack[kTgStack];
};

__global__ void __launch_bounds__(kTgWarps * 32) k_tree_gravity(TreeGravArgs a) {
  __shared__ TgSmem smem[kTgWarps];
  TgSmem &sm = smem[threadIdx.x >> 5];
  const int g = a.leaf0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (g >= a.leaf1) return;
  const unsigned lane = lane_id();
  const int n = a.t.n;
  const int s = g * kLeaf + (int)lane;
  const bool valid = s < n;
  const double4 anc = a.src[g * kLeaf];
  float xi = 0.f, yi = 0.f, zi = 0.f;
  if (valid) {
    const double4 p = a.src[s];
    xi = (float)(p.x - anc.x); yi = (float)(p.y - anc.y); zi = (float)(p.z - anc.z);
  }
  // the group's box (level 0 of the tree, rounded outward)
  const float4 gl = a.t.lo[a.t.base[0] + g], gh = a.t.hi[a.t.base[0] + g];
  const float eps2 = a.eps2, theta = a.theta;
  double ax = 0, ay = 0, az = 0, ap = 0;
  int nlist = 0;
  bool ok = true;

  auto sweep_list = [&]() {
    __syncwarp();  // the list entries written by every lane are visible
    float px = 0.f, py = 0.f, pz = 0.f, pp = 0.f;
    for (int k = 0; k < nlist; k++) {
      const NodeEntry e = sm.list[k];
      const float rx = e.x - xi, ry = e.y - yi, rz = e.z - zi;
      const float s2 = fmaf(rz, rz, fmaf(ry, ry, fmaf(rx, rx, eps2)));
      const float inv = rsqrt_f32(s2), inv2 = inv * inv;
      const float inv3 = inv2 * inv, inv5 = inv3 * inv2;
      const float qx = e.qxx * rx + e.qxy * ry + e.qxz * rz;
      const float qy = e.qxy * rx + e.qyy * ry + e.qyz * rz;
      const float qz = e.qxz * rx + e.qyz * ry + e.qzz * rz;
      const float rqr = rx * qx + ry * qy + rz * qz;
      const float c = e.m * inv3 + 2.5f * rqr * inv5 * inv2;
      px += c * rx - inv5 * qx;
      py += c * ry - inv5 * qy;
      pz += c * rz - inv5 * qz;
      pp -= e.m * inv + 0.5f * rqr * inv5;
    }
    ax += px; ay += py; az += pz; ap += pp;
    nlist = 0;
    __syncwarp();  // every lane is done reading before the list is refilled
  };
  auto sweep_leaf = [&](int lj) {
    const int sj = lj * kLeaf + (int)lane;
    __syncwarp();
    float4 q = make_float4(1e18f, 1e18f, 1e18f, 0.f);  // padding: far away, massless
    if (sj < n) {
      const double4 p = a.src[sj];
      q = make_float4((float)(p.x - anc.x), (float)(p.y - anc.y), (float)(p.z - anc.z), (float)p.w);
    }
    sm.leaf[lane] = q;
    __syncwarp();
    float px = 0.f, py = 0.f, pz = 0.f, pp = 0.f;
#pragma unroll 8
    for (int k = 0; k < kLeaf; k++) {
      const float4 p = sm.leaf[k];
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
  };

  const int top = a.t.levels - 1;
  if (top == 0) {
    sweep_leaf(0);
  } else {
    int sp = 1;
    if (lane == 0) sm.stack[0] = (top << 26);
    __syncwarp();
    while (sp > 0) {
      --sp;
      const int e = sm.stack[sp];
      __syncwarp();
      const int level = e >> 26, node = e & ((1 << 26) - 1);
      const int cl = level - 1;
      const int child = node * kFan + (int)lane;
      bool exists = child < a.t.count[cl];
      bool accept = false;
      double4 c = make_double4(0, 0, 0, 0);
      double b = 0;
      if (exists) {
        const long long k = a.t.base[cl] + child;
        c = a.cm[k];
        b = a.q1[k].z;
        exists = c.w > 0;
        // distance from the node's centre of mass to the group's box
        const double ddx = fmax(fmax((double)gl.x - c.x, c.x - (double)gh.x), 0.0);
        const double ddy = fmax(fmax((double)gl.y - c.y, c.y - (double)gh.y), 0.0);
        const double ddz = fmax(fmax((double)gl.z - c.z, c.z - (double)gh.z), 0.0);
        const double dmin = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
        accept = exists && b < (double)theta * dmin;
      }
      // accepted nodes -> the list (flushed when it could overflow)
      const unsigned am = __ballot_sync(0xffffffffu, accept);
      if (am) {
        if (nlist + __popc(am) > kTgList) sweep_list();
        if (accept) {
          const long long k = a.t.base[cl] + child;
          const double4 qa = a.q0[k], qb = a.q1[k];
          NodeEntry en;
          en.x = (float)(c.x - anc.x); en.y = (float)(c.y - anc.y); en.z = (float)(c.z - anc.z);
          en.m = (float)c.w;
          en.qxx = (float)qa.x; en.qyy = (float)qa.y; en.qzz = (float)qa.z; en.qxy = (float)qa.w;
          en.qxz = (float)qb.x; en.qyz = (float)qb.y;
          sm.list[nlist + __popc(am & ((1u << lane) - 1u))] = en;
        }
        nlist += __popc(am);
        __syncwarp();
      }
      // nodes that must be opened
      const bool open = exists && !accept;
      unsigned om = __ballot_sync(0xffffffffu, open);
      if (cl == 0) {
        while (om) {
          const int bb = __ffs(om) - 1;
          om &= om - 1;
          sweep_leaf(node * kFan + bb);
        }
        continue;
      }
      const int cnt = __popc(om);
      if (sp + cnt > kTgStack) {
        ok = false;
        break;
      }
      if (open) sm.stack[sp + cnt - 1 - __popc(om & ((1u << lane) - 1u))] = (cl << 26) | child;
      sp += cnt;
      __syncwarp();
    }
    __syncwarp();
    if (nlist > 0) sweep_list();
  }
  if (!ok && lane == 0) raise_flag(a.flags, SPH_FLAG_STACK_OVERFLOW);
  if (valid) a.out[s] = make_double4(a.G * ax, a.G * ay, a.G * az, a.G * ap);
}

// Shard `rank` of `world` computes the groups of its leaf range into `out`,
// zeroed first when world > 1 (the sum over shards is the whole field).
int launch_tree_gravity(const TreeView &t, const double4 *src, double4 *cm, double4 *q0, double4 *q1, double4 *out,
                        unsigned *flags, double eps, double theta, double G, int rank, int world, cudaStream_t st) {
  if (t.n <= 0) return 0;
  int launches = tree_moments(t, src, cm, q0, q1, st);
  if (world > 1) cudaMemsetAsync(out, 0, sizeof(double4) * t.n, st);
  long long l0, l1;
  shard_range(t.count[0], rank, world, l0, l1);
  if (l1 <= l0) return launches;
  TreeGravArgs a;
  a.t = t; a.src = src; a.cm = cm; a.q0 = q0; a.q1 = q1; a.out = out; a.flags = flags;
  a.eps2 = (float)(eps * eps); a.theta = (float)theta; a.G = G;
  a.leaf0 = (int)l0; a.leaf1 = (int)l1;
  const int warps = (int)(l1 - l0);
  k_tree_gravity<<<(warps + kTgWarps - 1) / kTgWarps, kTgWarps * 32, 0, st>>>(a);
  return launches + 1;
}

}  // namespace sph
