// tree.cu -- the spatial tree over Morton-ordered particles.
//
// The reference builds a left-balanced kd-tree on the host every step
// (kd_tree.cpp:39-128, split dimension = depth % 3 at the median).  Here the
// particles are already in Morton order, whose bit interleaving is itself a
// kd split (x, y, z in turn at the cell midpoints), so the tree is implicit:
// leaves are runs of 32 consecutive particles (one warp), and every internal
// node covers 32 consecutive children.  Only the bounding boxes are built:
// one warp reduction per node, level by level, FP64 extrema rounded outward
// to float so a box test never rejects a true neighbour.
#include "common.cuh"

namespace sph {

__global__ void k_leaf_boxes(int n, const double4 *__restrict__ pos, float4 *__restrict__ lo, float4 *__restrict__ hi,
                             int nleaf) {
  int leaf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (leaf >= nleaf) return;
  int s = leaf * kLeaf + (int)lane_id();
  double l0 = 1e308, l1 = 1e308, l2 = 1e308, h0 = -1e308, h1 = -1e308, h2 = -1e308;
  if (s < n) {
    double4 p = pos[s];
    l0 = h0 = p.x; l1 = h1 = p.y; l2 = h2 = p.z;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l0 = fmin(l0, __shfl_xor_sync(0xffffffffu, l0, o));
    l1 = fmin(l1, __shfl_xor_sync(0xffffffffu, l1, o));
    l2 = fmin(l2, __shfl_xor_sync(0xffffffffu, l2, o));
    h0 = fmax(h0, __shfl_xor_sync(0xffffffffu, h0, o));
    h1 = fmax(h1, __shfl_xor_sync(0xffffffffu, h1, o));
    h2 = fmax(h2, __shfl_xor_sync(0xffffffffu, h2, o));
  }
  if (lane_id() == 0) {
    lo[leaf] = make_float4(__double2float_rd(l0), __double2float_rd(l1), __double2float_rd(l2), 0.f);
    hi[leaf] = make_float4(__double2float_ru(h0), __double2float_ru(h1), __double2float_ru(h2), 0.f);
  }
}

__global__ void k_parent_boxes(int nchild, const float4 *__restrict__ clo, const float4 *__restrict__ chi,
                               int nparent, float4 *__restrict__ plo, float4 *__restrict__ phi) {
  int node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (node >= nparent) return;
  int c = node * kFan + (int)lane_id();
  float4 l = make_float4(3e38f, 3e38f, 3e38f, 0.f), h = make_float4(-3e38f, -3e38f, -3e38f, 0.f);
  if (c < nchild) { l = clo[c]; h = chi[c]; }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l.x = fminf(l.x, __shfl_xor_sync(0xffffffffu, l.x, o));
    l.y = fminf(l.y, __shfl_xor_sync(0xffffffffu, l.y, o));
    l.z = fminf(l.z, __shfl_xor_sync(0xffffffffu, l.z, o));
    h.x = fmaxf(h.x, __shfl_xor_sync(0xffffffffu, h.x, o));
    h.y = fmaxf(h.y, __shfl_xor_sync(0xffffffffu, h.y, o));
    h.z = fmaxf(h.z, __shfl_xor_sync(0xffffffffu, h.z, o));
  }
  if (lane_id() == 0) { plo[node] = l; phi[node] = h; }
}

// level sizes for n particles; returns the number of levels and total nodes
int tree_layout(int n, TreeView *t) {
  t->n = n;
  int c = (n + kLeaf - 1) / kLeaf;
  if (c < 1) c = 1;
  int L = 0;
  long long off = 0;
  while (true) {
    t->count[L] = c;
    t->base[L] = off;
    off += c;
    L++;
    if (c == 1 || L == kMaxLevels) break;
    c = (c + kFan - 1) / kFan;
  }
  t->levels = L;
  return (int)off;
}

int build_tree(const TreeView &t, const double4 *pos, float4 *lo, float4 *hi, cudaStream_t st) {
  int launches = 0;
  int nleaf = t.count[0];
  k_leaf_boxes<<<(nleaf * 32 + 255) / 256, 256, 0, st>>>(t.n, pos, lo + t.base[0], hi + t.base[0], nleaf);
  launches++;
  for (int l = 1; l < t.levels; l++) {
    int np = t.count[l];
    k_parent_boxes<<<(np * 32 + 255) / 256, 256, 0, st>>>(t.count[l - 1], lo + t.base[l - 1], hi + t.base[l - 1], np,
                                                          lo + t.base[l], hi + t.base[l]);
    launches++;
  }
  return launches;
}

}  // namespace sph
