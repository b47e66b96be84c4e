// neighbours.cu -- smoothing-length solve (dev_solve_range.cu:17-189) and
// neighbour search (dev_find_ngb.cu:13-87) on the Morton tree.
//
// One warp owns one leaf (32 consecutive particles); lane l owns particle
// 32*leaf + l.  The warp walks the tree together: at every internal node each
// lane tests one child box, a ballot picks the children that overlap the
// union of the lanes' search boxes, and the hits are pushed in reverse order
// on a per-warp shared-memory stack, so leaves come out in ascending index
// order.  A visited leaf's 32 positions are staged in shared memory and every
// lane applies the exact FP64 predicate ds2 < range^2 to all of them.
//
// This translation unit is compiled without FMA contraction: the h solve and
// the predicate then perform the same IEEE operations, in the same order
// (ascending neighbour index), as an FP64 CPU evaluation of the reference's
// loops, which makes the solved ranges and the neighbour sets reproducible
// bit for bit against such an evaluation.
#include "common.cuh"
#include "sph_math.cuh"

namespace sph {

constexpr int kWarpsPerBlock = 4;
constexpr unsigned kFull = 0xffffffffu;

struct LaneBox {
  float lo[3], hi[3];
};

struct WarpSmem {
  LaneBox lbox[kLeaf];  // the lanes' query boxes of the current walk
  int stack[kStack];
  double sx[kLeaf], sy[kLeaf], sz[kLeaf];
  float4 sf[kLeaf];  // anchor-relative FP32 copies for the pre-filter
  double tx[kLeaf], ty[kLeaf], tz[kLeaf];  // the warp's own particles (the targets)
  // The speculative walk's per-target squared ranges and sliver bounds, and
  // the boxes of the children of the node being visited: every lane reads
  // them for the target or leaf at hand with one broadcast load, where a
  // shuffle from the owning lane took two instructions per double (N = 1M:
  // steady-state solve 3.83 -> 3.54 ms, the same ranges and lists).
  double tr2[kLeaf], ts2[kLeaf];
  float4 cbox[2 * kFan];  // lo of child k at [k], hi at [kFan + k]
};

// Conservative FP32 pre-filter of the neighbour predicate.  Coordinates are
// taken relative to a warp anchor (lane 0's particle) and rounded to FP32.
// For a pair that is truly within range w of lane l, |x_j - anchor| <= B + w
// where B bounds |x_l - anchor| over the warp, so the FP32 squared distance
// differs from the exact one by less than w^2 (4.2e-7 (B + w)/w + 2.6e-7).
// A candidate is rejected only when its FP32 squared distance exceeds
// w^2 (1 + m) with m = 1e-6 (B + w)/w + 1e-6, i.e. when it is certainly
// outside; everything else goes through the exact FP64 predicate, so the
// neighbour sets are unchanged.  Lanes with m > 1e-2 skip the pre-filter.
struct Prefilter {
  double ax, ay, az;  // warp anchor
  double B;           // sqrt(3) max |x_l - anchor| over the warp
  float xf, yf, zf;   // this lane, anchor-relative
};

__device__ __forceinline__ Prefilter make_prefilter(bool on, double x, double y, double z) {
  Prefilter f;
  f.ax = __shfl_sync(0xffffffffu, x, 0);
  f.ay = __shfl_sync(0xffffffffu, y, 0);
  f.az = __shfl_sync(0xffffffffu, z, 0);
  const double dx = x - f.ax, dy = y - f.ay, dz = z - f.az;
  double b = on ? fmax(fabs(dx), fmax(fabs(dy), fabs(dz))) : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  f.B = 1.7320508075688772 * b;
  f.xf = (float)dx;
  f.yf = (float)dy;
  f.zf = (float)dz;
  return f;
}

// the FP32 threshold for range w; negative = no pre-filter for this lane
__device__ __forceinline__ float prefilter_threshold(const Prefilter &f, double w) {
  if (!(w > 0)) return -1.f;
  const double m = 1e-6 * (f.B + w) / w + 1e-6;
  if (m > 1e-2) return -1.f;
  return (float)(w * w * (1.0 + m));
}

__device__ __forceinline__ bool certainly_outside(const Prefilter &f, float thr, float4 q) {
  const float dx = f.xf - q.x, dy = f.yf - q.y, dz = f.zf - q.z;
  const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
  return thr >= 0.f && d2 > thr;
}

// Query box over the lanes that take part: [x - r, x + r] widened by a
// relative 1e-15 of the magnitudes (covers the rounding of x - r) and
// rounded outward to float.
__device__ __forceinline__ void warp_query_box(bool on, double x, double y, double z, double r, float *ql, float *qh) {
  double m0 = (fabs(x) + r) * 1e-15, m1 = (fabs(y) + r) * 1e-15, m2 = (fabs(z) + r) * 1e-15;
  double l0 = on ? x - r - m0 : 1e308, l1 = on ? y - r - m1 : 1e308, l2 = on ? z - r - m2 : 1e308;
  double h0 = on ? x + r + m0 : -1e308, h1 = on ? y + r + m1 : -1e308, h2 = on ? z + r + m2 : -1e308;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l0 = fmin(l0, __shfl_xor_sync(kFull, l0, o));
    l1 = fmin(l1, __shfl_xor_sync(kFull, l1, o));
    l2 = fmin(l2, __shfl_xor_sync(kFull, l2, o));
    h0 = fmax(h0, __shfl_xor_sync(kFull, h0, o));
    h1 = fmax(h1, __shfl_xor_sync(kFull, h1, o));
    h2 = fmax(h2, __shfl_xor_sync(kFull, h2, o));
  }
  ql[0] = __double2float_rd(l0); ql[1] = __double2float_rd(l1); ql[2] = __double2float_rd(l2);
  qh[0] = __double2float_ru(h0); qh[1] = __double2float_ru(h1); qh[2] = __double2float_ru(h2);
}

// This lane's own query box [x - r, x + r], widened and rounded outward like
// warp_query_box.  A leaf whose box misses it holds no j with d2 < r^2 for
// this lane (both boxes contain everything they should), so the lane skips
// the leaf's candidates, and the walk descends only into nodes whose box
// meets the box of at least one active lane (not merely the union of the
// lanes' boxes): the sets are unchanged, the work drops by more than half.
__device__ __forceinline__ LaneBox lane_query_box(double x, double y, double z, double r) {
  const double m0 = (fabs(x) + r) * 1e-15, m1 = (fabs(y) + r) * 1e-15, m2 = (fabs(z) + r) * 1e-15;
  LaneBox b;
  b.lo[0] = __double2float_rd(x - r - m0); b.lo[1] = __double2float_rd(y - r - m1); b.lo[2] = __double2float_rd(z - r - m2);
  b.hi[0] = __double2float_ru(x + r + m0); b.hi[1] = __double2float_ru(y + r + m1); b.hi[2] = __double2float_ru(z + r + m2);
  return b;
}

// This lane's query ball for the box test below: centre rounded to float
// and the squared radius widened to cover every rounding of the float test
// (the centre's rounding, the subtractions, squares and sums: under
// 4e-7 (|x| + |y| + |z|) absolute and 1e-6 relative), so a leaf that holds a
// j with |x_j - x| < r always passes.
struct LaneBall {
  float x, y, z, r2;
};

__device__ __forceinline__ LaneBall lane_ball(double x, double y, double z, double r) {
  const double rr = r * (1.0 + 1e-6) + 4e-7 * (fabs(x) + fabs(y) + fabs(z));
  LaneBall b;
  b.x = (float)x; b.y = (float)y; b.z = (float)z;
  b.r2 = __double2float_ru(rr * rr);
  return b;
}

// does the box [bl, bh] come within the ball's radius of its centre?
__device__ __forceinline__ bool lane_ball_hits(const LaneBall &q, const float *bl, const float *bh) {
  const float dx = fmaxf(fmaxf(bl[0] - q.x, q.x - bh[0]), 0.f);
  const float dy = fmaxf(fmaxf(bl[1] - q.y, q.y - bh[1]), 0.f);
  const float dz = fmaxf(fmaxf(bl[2] - q.z, q.z - bh[2]), 0.f);
  return dx * dx + dy * dy + dz * dz <= q.r2;
}

__device__ __forceinline__ bool lane_box_hits(const LaneBox &q, const float *bl, const float *bh) {
  return (bl[0] <= q.hi[0]) & (bh[0] >= q.lo[0]) & (bl[1] <= q.hi[1]) & (bh[1] >= q.lo[1]) & (bl[2] <= q.hi[2]) &
         (bh[2] >= q.lo[2]);
}

// publish this lane's query box to the warp; returns the mask of active lanes
__device__ __forceinline__ unsigned share_lane_boxes(WarpSmem &sm, const LaneBox &lb, bool on) {
  __syncwarp();
  sm.lbox[lane_id()] = lb;
  const unsigned m = __ballot_sync(kFull, on);
  __syncwarp();
  return m;
}

// Visit, in ascending order, every leaf whose box overlaps [ql, qh] (the
// union of the lanes' query boxes) and the query box of at least one lane of
// `onmask` (boxes in lbs).  All lanes call visit(leaf, lo, hi) together,
// lo / hi = the leaf's box (float, rounded outward), read from cbox (2 kFan
// float4 of the warp's shared memory, which visit must not write).  Returns
// false on stack overflow.
template <class Visit>
__device__ bool walk_leaves(const TreeView &t, const float *ql, const float *qh, const LaneBox *lbs,
                            unsigned onmask, int *stack, float4 *cbox, Visit &&visit) {
  const unsigned lane = lane_id();
  const int top = t.levels - 1;
  if (top == 0) {
    const float bl[3] = {-3e38f, -3e38f, -3e38f}, bh[3] = {3e38f, 3e38f, 3e38f};
    visit(0, bl, bh);
    return true;
  }
  int sp = 1;
  if (lane == 0) stack[0] = (top << 26);
  __syncwarp();
  while (sp > 0) {
    --sp;
    const int e = stack[sp];
    __syncwarp();
    const int level = e >> 26, node = e & ((1 << 26) - 1);
    const int cl = level - 1;
    const int child = node * kFan + (int)lane;
    bool hit = false;
    float4 l = make_float4(0.f, 0.f, 0.f, 0.f), h = l;
    if (child < t.count[cl]) {
      l = __ldg(&t.lo[t.base[cl] + child]);
      h = __ldg(&t.hi[t.base[cl] + child]);
      hit = (l.x <= qh[0]) & (h.x >= ql[0]) & (l.y <= qh[1]) & (h.y >= ql[1]) & (l.z <= qh[2]) & (h.z >= ql[2]);
    }
    if (hit) {  // ... and the box of some active lane
      bool any = false;
      unsigned mm = onmask;
      while (mm && !any) {
        const int L = __ffs(mm) - 1;
        mm &= mm - 1;
        const LaneBox q = lbs[L];
        any = (l.x <= q.hi[0]) & (h.x >= q.lo[0]) & (l.y <= q.hi[1]) & (h.y >= q.lo[1]) & (l.z <= q.hi[2]) &
              (h.z >= q.lo[2]);
      }
      hit = any;
    }
    unsigned m = __ballot_sync(kFull, hit);
    if (cl == 0) {
      if (m) {  // the leaves' boxes, for every lane at each visit
        __syncwarp();
        cbox[lane] = l;
        cbox[kFan + lane] = h;
        __syncwarp();
      }
      while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        const float4 lb4 = cbox[b], hb4 = cbox[kFan + b];
        const float bl[3] = {lb4.x, lb4.y, lb4.z}, bh[3] = {hb4.x, hb4.y, hb4.z};
        visit(node * kFan + b, bl, bh);
      }
      continue;
    }
    const int cnt = __popc(m);
    if (sp + cnt > kStack) return false;
    if (hit) stack[sp + cnt - 1 - __popc(m & ((1u << lane) - 1u))] = (cl << 26) | child;
    sp += cnt;
    __syncwarp();
  }
  return true;
}

__device__ __forceinline__ void stage_leaf(const double4 *__restrict__ pos, int n, int leaf, WarpSmem &sm,
                                           const Prefilter &f) {
  const int s = leaf * kLeaf + (int)lane_id();
  __syncwarp();
  if (s < n) {
    const double4 p = ld4(pos + s);
    sm.sx[lane_id()] = p.x;
    sm.sy[lane_id()] = p.y;
    sm.sz[lane_id()] = p.z;
    sm.sf[lane_id()] = make_float4((float)(p.x - f.ax), (float)(p.y - f.ay), (float)(p.z - f.az), 0.f);
  }
  __syncwarp();
}

struct SolveArgs {
  TreeView t;
  double4 *pos;
  int *nevals;
  unsigned *flags;
  double n_target, rel_err, f_scale;
  int max_iter;
  int *n_ngb;      // hard count at the final range
  int *list;       // neighbour lists at the final range (layout of k_find_ngb)
  double *dcache;  // squared distances of the cached candidates, layout of list
  int cap;
  int leaf0, leaf1;  // leaves processed by this launch
  // the speculative first pass (k_solve_spec) hands the leaves it leaves
  // unfinished to k_solve_range through a queue (null: no speculative pass)
  int *queue;
  int *queue_count;
  struct SolveSave *save;  // per slot
};

enum { kBr0 = 0, kBr1 = 1, kSolve = 2, kDone = 3 };

// radius of a candidate cache relative to the range that fills it: one
// clamped Newton step of the bracket (f_scale = 10 %) stays inside it
constexpr double kCacheMargin = 1.15;
constexpr int kEvalBatch = 4;     // cache entries loaded ahead per evaluation step
constexpr int kSpecBlocks = 8;    // resident blocks per SM of the speculative pass
constexpr int kCompactBatch = 8;  // cache entries loaded ahead per compaction step

// A lane's iteration state: the bracket / Newton / bisection steps of
// dev_solve_range.cu:93-172 between evaluations.
struct LaneIter {
  double w, dx, f, x_left, f_try, rx, ry;
  int phase, iter, keep, nev;
};

// One evaluation's epilogue (compute_ngb, dev_solve_range.cu:77-87) with the
// smooth count sf and its derivative sum sg at it.w, and the step of the
// lane's iteration to its next evaluation or the end.
__device__ __forceinline__ void solve_advance(LaneIter &it, double sf, double sg, const SolveArgs &a) {
  const double rel = a.rel_err, fs = a.f_scale;
  it.nev++;
  it.f = sf - a.n_target;
  sg *= 1.0 / it.w;
  if (sg != 0) it.dx = it.f / sg;
  else it.dx = (it.f < 0) ? -it.w : +it.w;
  bool to_solve_init = false, to_br_check = false, to_solve_check = false;
  if (it.phase == kBr0 || it.phase == kBr1) {
    if (fabs(it.dx) < rel * it.w) {
      it.rx = it.w - 0.5 * fabs(it.dx);
      it.ry = it.w + 0.5 * fabs(it.dx);
      to_solve_init = true;
    } else {
      if (fabs(it.dx) > fs * it.w) it.dx = (it.dx < 0) ? -fs * it.w : fs * it.w;
      if (it.phase == kBr0) {
        it.x_left = it.w;
        it.f_try = it.f;
        it.iter = 0;
      }
      to_br_check = true;
    }
  } else {  // kSolve
    if (it.f < 0) it.rx = it.w;
    else it.ry = it.w;
    it.keep = fabs(it.dx) > rel * it.w;
    to_solve_check = true;
  }
  if (to_br_check) {
    if ((it.f_try * it.f >= 0) && (it.iter++ < a.max_iter)) {
      it.x_left = it.w;
      it.f_try = it.f;
      it.w -= it.dx;
      it.phase = kBr1;
    } else {
      if (it.x_left < it.w) { it.rx = it.x_left; it.ry = it.w; }
      else { it.rx = it.w; it.ry = it.x_left; }
      to_solve_init = true;
    }
  }
  if (to_solve_init) {
    it.w = 0.5 * (it.rx + it.ry);
    it.dx = 0;
    if (fabs(it.rx - it.ry) > rel * it.w) {
      it.iter = 0;
      it.keep = 1;
      to_solve_check = true;
    } else {
      it.phase = kDone;
    }
  }
  if (to_solve_check) {
    if (it.keep && (it.iter++ < a.max_iter)) {
      it.w -= it.dx;
      if ((it.w - it.ry) * (it.w - it.rx) >= 0) {
        it.dx = 0.5 * (it.ry - it.rx);
        it.w = 0.5 * (it.rx + it.ry);
      }
      it.phase = kSolve;
    } else {
      if (it.keep) raise_flag(a.flags, SPH_FLAG_H_NOT_CONVERGED);
      it.phase = kDone;
    }
  }
}

// a lane's state handed from the speculative pass to the resumed solve
struct SolveSave {
  double w, dx, f, x_left, f_try, rx, ry;
  int phase, iter, keep, nev, cnt_list, bits;  // bits: 1 direct, 2 pending, 4 listed by the speculative pass
};

// Speculative first evaluation.  In steady state the previous step's range
// (after the predictor) already passes the tolerance test for almost every
// particle, so the first evaluation is also the last: the warp walks the
// tree once at the ranges themselves, every hit (d2 < w^2) goes straight to
// its lane's list (index only), and each lane evaluates f and f' over its
// list in list order -- ascending index, the order of the walk and of the
// CPU loop -- recomputing the FP64 d2 of each entry from the positions (the
// same operations as the walk, so the same value).  No candidate cache is
// written or read.  A lane done after this evaluation keeps the list when
// its final range (w = (rx + ry) / 2, within a few ulp of the evaluated one)
// leaves the set unchanged: every entry inside the final range (the largest
// d2 checked), and, if the range grew, no candidate in the sliver just
// outside the evaluated range (flagged during the walk).  Otherwise the
// lane lists by a walk at its final range; lanes not done continue with the
// candidate cache below.
// This is its own kernel, with fewer registers (more resident warps) than
// the candidate-cache solve; a leaf with a lane not done after it saves its
// lanes' states and goes on a queue that k_solve_range then resumes.
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kSpecBlocks) k_solve_spec(SolveArgs a) {
  __shared__ WarpSmem smem[kWarpsPerBlock];
  WarpSmem &sm = smem[threadIdx.x >> 5];
  const int leaf = a.leaf0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (leaf >= a.leaf1) return;
  const int n = a.t.n;
  const int s = leaf * kLeaf + (int)lane_id();
  const bool valid = s < n;
  double xi = 0, yi = 0, zi = 0, w0 = 0;
  if (valid) {
    const double4 p = a.pos[s];
    xi = p.x; yi = p.y; zi = p.z; w0 = p.w;
  }
  const Prefilter pf = make_prefilter(valid && w0 > 0, xi, yi, zi);
  sm.tx[lane_id()] = xi;
  sm.ty[lane_id()] = yi;
  sm.tz[lane_id()] = zi;
  __syncwarp();
  const size_t colbase = (size_t)leaf * a.cap * kLeaf;  // the warp's block of list / dcache
  LaneIter it;
  it.w = w0;
  it.phase = (valid && w0 > 0) ? kBr0 : kDone;
  it.dx = it.f = it.x_left = it.f_try = it.rx = it.ry = 0;
  it.iter = it.keep = it.nev = 0;
  double &w = it.w;
  int &phase = it.phase, &nev = it.nev;
  bool stack_ok = true;
  const size_t col = (size_t)leaf * a.cap * kLeaf + lane_id();
  int *lst = a.list + col;
  const int cap = a.cap;
  int cnt_list = 0;
  bool direct = false;
  bool pending = false;
  auto advance = [&](double sf, double sg) { solve_advance(it, sf, sg, a); };
  int spec_cnt = -1;  // >= 0: the speculative list is this lane's final list
  if (__any_sync(kFull, phase != kDone)) {
    const bool on = phase != kDone;
    const double w_eval = w;
    const double r2 = __dmul_rn(w, w);
    const double r2hi = r2 * (1.0 + 0x1p-40);  // the sliver [w^2, r2hi)
    const double rw = w * (1.0 + 1e-12);       // boxes and ball cover the sliver
    float ql[3], qh[3];
    warp_query_box(on, xi, yi, zi, rw, ql, qh);
    const LaneBox lb = lane_query_box(xi, yi, zi, rw);
    const LaneBall lball = lane_ball(xi, yi, zi, rw);
    sm.tr2[lane_id()] = r2;  // published by the __syncwarp in share_lane_boxes
    sm.ts2[lane_id()] = r2hi;
    const unsigned onmask = share_lane_boxes(sm, lb, on);
    int c = 0;
    bool sliver = false;
    stack_ok &= walk_leaves(a.t, ql, qh, sm.lbox, onmask, sm.stack, sm.cbox, [&](int lj, const float *bl, const float *bh) {
      const int cntj = min(kLeaf, n - lj * kLeaf);
      const unsigned tm = __ballot_sync(kFull, on && lane_box_hits(lb, bl, bh) && lane_ball_hits(lball, bl, bh));
      if (!tm) return;
      double xk = 1e300, yk = 1e300, zk = 1e300;  // past the last particle: never a neighbour
      if ((int)lane_id() < cntj) {
        const double4 p = ld4(a.pos + lj * kLeaf + (int)lane_id());
        xk = p.x; yk = p.y; zk = p.z;
      }
      const int jk = lj * kLeaf + (int)lane_id();
      const unsigned below = (1u << lane_id()) - 1u;
      unsigned m = tm;
      while (m) {  // two targets per round, as in the candidate-cache fill of k_solve_range
        const int t0 = __ffs(m) - 1;
        m &= m - 1u;
        const int t1 = m ? __ffs(m) - 1 : t0;
        const bool two = m != 0u;
        m &= m - 1u;
        const double r20 = sm.tr2[t0], r21 = sm.tr2[t1];
        const double s20 = sm.ts2[t0], s21 = sm.ts2[t1];
        const double d20 = ds2_exact(sm.tx[t0] - xk, sm.ty[t0] - yk, sm.tz[t0] - zk);
        const double d21 = ds2_exact(sm.tx[t1] - xk, sm.ty[t1] - yk, sm.tz[t1] - zk);
        const bool h0 = d20 < r20, h1 = two && d21 < r21;
        const unsigned hm0 = __ballot_sync(kFull, h0), hm1 = __ballot_sync(kFull, h1);
        const unsigned sm0 = __ballot_sync(kFull, !h0 && d20 < s20), sm1 = __ballot_sync(kFull, two && !h1 && d21 < s21);
        const int b0 = __shfl_sync(kFull, c, t0), b1 = __shfl_sync(kFull, c, t1);
        if (h0) {
          const int idx = b0 + __popc(hm0 & below);
          if (idx < cap) a.list[colbase + (size_t)idx * kLeaf + (size_t)t0] = jk;
        }
        if (h1) {
          const int idx = b1 + __popc(hm1 & below);
          if (idx < cap) a.list[colbase + (size_t)idx * kLeaf + (size_t)t1] = jk;
        }
        if ((int)lane_id() == t0) { c += __popc(hm0); sliver |= sm0 != 0u; }
        if ((int)lane_id() == t1) { c += __popc(hm1); sliver |= sm1 != 0u; }  // t1 != t0 whenever hm1 | sm1 != 0
      }
    });
    if (on && c <= cap) {
      double sf = 0, sg = 0, dmax = -1.0;
      for (int k0 = 0; k0 < c; k0 += kEvalBatch) {
        int j[kEvalBatch];
#pragma unroll
        for (int q = 0; q < kEvalBatch; q++) j[q] = k0 + q < c ? lst[(size_t)(k0 + q) * kLeaf] : -1;
        double4 pj[kEvalBatch];
#pragma unroll
        for (int q = 0; q < kEvalBatch; q++) pj[q] = j[q] >= 0 ? ld4(a.pos + j[q]) : make_double4(xi, yi, zi, 0);
#pragma unroll
        for (int q = 0; q < kEvalBatch; q++) {
          if (j[q] >= 0) {
            const double d2 = ds2_exact(xi - pj[q].x, yi - pj[q].y, zi - pj[q].z);
            const double u = 2 * sqrt(d2) / w;
            sf += k_ig<double>(u);
            sg -= k_digdh<double>(u);
            dmax = fmax(dmax, d2);
          }
        }
      }
      advance(sf, sg);
      if (phase == kDone) {
        const double wf2 = __dmul_rn(w, w);
        const bool same = (w == w_eval) || (w < w_eval && dmax < wf2) || (w > w_eval && !sliver && wf2 < r2hi);
        if (same) {
          spec_cnt = c;
          cnt_list = c;
        } else {
          direct = true;  // list by a walk at the final range
          pending = true;
        }
      }
    }
  }
  if (!stack_ok && lane_id() == 0) raise_flag(a.flags, SPH_FLAG_STACK_OVERFLOW);
  const bool more = phase != kDone || pending;
  if (!__any_sync(kFull, more)) {
    if (valid) {
      a.pos[s].w = (w > 0) ? w : 0.0;
      a.n_ngb[s] = cnt_list;
      if (a.nevals) a.nevals[s] = nev;
    }
    return;
  }
  if (valid) {
    SolveSave v;
    v.w = it.w; v.dx = it.dx; v.f = it.f; v.x_left = it.x_left; v.f_try = it.f_try; v.rx = it.rx; v.ry = it.ry;
    v.phase = it.phase; v.iter = it.iter; v.keep = it.keep; v.nev = it.nev; v.cnt_list = cnt_list;
    v.bits = (direct ? 1 : 0) | (pending ? 2 : 0) | (spec_cnt >= 0 ? 4 : 0);
    a.save[s] = v;
  }
  if (lane_id() == 0) a.queue[atomicAdd(a.queue_count, 1)] = leaf;
}

// dev_solve_range (dev_solve_range.cu:137-189): per particle, bracket the
// root of f(w) = sum_j ig(2 r_ij / w) - N_target with clamped Newton steps
// (dev_bracket_root :93-135), then safeguarded Newton / bisection until
// |dx| < rel_err * w.  Each lane runs that iteration as a state machine.
//
// Candidate cache (find_ngb fused in): a lane whose range w is not covered
// by its cache walks the tree once at radius 1.15 w and stores every j with
// d2 < (1.15 w)^2 -- index in its column of the neighbour list, exact FP64
// d2 in the same column of dcache -- in the walk's ascending order.  Every
// evaluation of f (and of its derivative) then runs over the cached entries
// with d2 < w^2 in that order, the same operations in the same order as a
// walk at w, and the final list is the cache compacted in place to the final
// range.  The lanes that need a walk in a round share it.  A lane whose
// candidates exceed the list capacity falls back to walking at w for every
// evaluation, writing its list as it goes (`direct`), with one list-only walk
// when the final range differs from the last one evaluated (`pending`).
// 6 blocks (24 warps) per SM: at N = 1M the capped form (80 registers, a
// few spilled) took 12.1 ms per solve against 14.5 ms at 120 registers.
// The candidate-cache solve of one leaf-warp, from the initial ranges or
// (resume) from the states the speculative pass saved.
__device__ __forceinline__ void solve_leaf(const SolveArgs &a, WarpSmem &sm, int leaf, bool resume) {
  const int n = a.t.n;
  const int s = leaf * kLeaf + (int)lane_id();
  const bool valid = s < n;
  double xi = 0, yi = 0, zi = 0, w0 = 0;
  if (valid) {
    const double4 p = a.pos[s];
    xi = p.x; yi = p.y; zi = p.z; w0 = p.w;
  }
  const Prefilter pf = make_prefilter(valid && w0 > 0, xi, yi, zi);
  sm.tx[lane_id()] = xi;
  sm.ty[lane_id()] = yi;
  sm.tz[lane_id()] = zi;
  __syncwarp();
  const size_t colbase = (size_t)leaf * a.cap * kLeaf;  // the warp's block of list / dcache
  LaneIter it;
  it.w = w0;
  it.phase = (valid && w0 > 0) ? kBr0 : kDone;
  it.dx = it.f = it.x_left = it.f_try = it.rx = it.ry = 0;
  it.iter = it.keep = it.nev = 0;
  double &w = it.w;
  int &phase = it.phase, &nev = it.nev;
  bool stack_ok = true;
  const size_t col = (size_t)leaf * a.cap * kLeaf + lane_id();
  int *lst = a.list + col;
  const int cap = a.cap;
  int cnt_list = 0;
  bool direct = false;
  bool pending = false;
  auto advance = [&](double sf, double sg) { solve_advance(it, sf, sg, a); };
  double &dx = it.dx, &f = it.f, &x_left = it.x_left, &f_try = it.f_try, &rx = it.rx, &ry = it.ry;
  int &iter = it.iter, &keep = it.keep;
  (void)dx; (void)f; (void)x_left; (void)f_try; (void)rx; (void)ry; (void)iter; (void)keep;
  double *dc = a.dcache + col;
  int ncache = 0;           // cached entries
  double cache_r2 = -1.0;   // the cache holds every j with d2 < cache_r2
  double w_list = -1.0;     // direct lanes: range of the list last written
  int spec_cnt = -1;        // >= 0: the speculative pass listed this lane
  if (resume && valid) {
    const SolveSave v = a.save[s];
    it.w = v.w; it.dx = v.dx; it.f = v.f; it.x_left = v.x_left; it.f_try = v.f_try; it.rx = v.rx; it.ry = v.ry;
    it.phase = v.phase; it.iter = v.iter; it.keep = v.keep; it.nev = v.nev;
    cnt_list = v.cnt_list;
    direct = (v.bits & 1) != 0;
    pending = (v.bits & 2) != 0;
    spec_cnt = (v.bits & 4) ? v.cnt_list : -1;
  }
  while (true) {
    const bool iterate = phase != kDone;
    if (!__any_sync(kFull, iterate || pending)) break;
    const double w2 = __dmul_rn(w, w);
    const bool fill = iterate && !direct && !(w2 <= cache_r2);
    const bool dwalk = (iterate && direct) || pending;
    double sf = 0, sg = 0;
    bool evaluated = false;
    if (__any_sync(kFull, fill || dwalk)) {
      const bool on = fill || dwalk;
      const double r = fill ? w * kCacheMargin : w;
      const double r2 = __dmul_rn(r, r);
      float ql[3], qh[3];
      warp_query_box(on, xi, yi, zi, r, ql, qh);
      const float thr = prefilter_threshold(pf, r);
      int c = 0;
      const LaneBox lb = lane_query_box(xi, yi, zi, r);
      const LaneBall lball = lane_ball(xi, yi, zi, r);
      const unsigned onmask = share_lane_boxes(sm, lb, on);
      const bool any_dwalk = __any_sync(kFull, dwalk);
      stack_ok &= walk_leaves(a.t, ql, qh, sm.lbox, onmask, sm.stack, sm.cbox, [&](int lj, const float *bl, const float *bh) {
        const int cntj = min(kLeaf, n - lj * kLeaf);
        if (!any_dwalk) {
          // Cache fills only: transposed.  Lane k holds candidate k of the
          // leaf; for every lane t whose box meets the leaf, all 32 lanes
          // apply t's exact predicate at once and a ballot appends the hits
          // to t's column in ascending k -- the same entries, order and
          // FP64 d2 as t testing the leaf itself, in |targets| rounds
          // instead of 32 (a lane needs about half the leaves its warp
          // visits).
          const unsigned tm = __ballot_sync(kFull, on && lane_box_hits(lb, bl, bh) && lane_ball_hits(lball, bl, bh));
          if (!tm) return;
          double xk = 1e300, yk = 1e300, zk = 1e300;  // past the last particle: never a neighbour
          if ((int)lane_id() < cntj) {
            const double4 p = ld4(a.pos + lj * kLeaf + (int)lane_id());
            xk = p.x; yk = p.y; zk = p.z;
          }
          const int jk = lj * kLeaf + (int)lane_id();
          const unsigned below = (1u << lane_id()) - 1u;
          unsigned m = tm;
          while (m) {  // two targets per round: independent chains overlap
            const int t0 = __ffs(m) - 1;
            m &= m - 1u;
            const int t1 = m ? __ffs(m) - 1 : t0;
            const bool two = m != 0u;
            m &= m - 1u;
            const double r20 = __shfl_sync(kFull, r2, t0), r21 = __shfl_sync(kFull, r2, t1);
            const double d20 = ds2_exact(sm.tx[t0] - xk, sm.ty[t0] - yk, sm.tz[t0] - zk);
            const double d21 = ds2_exact(sm.tx[t1] - xk, sm.ty[t1] - yk, sm.tz[t1] - zk);
            const bool h0 = d20 < r20, h1 = two && d21 < r21;
            const unsigned hm0 = __ballot_sync(kFull, h0), hm1 = __ballot_sync(kFull, h1);
            const int b0 = __shfl_sync(kFull, c, t0), b1 = __shfl_sync(kFull, c, t1);
            if (h0) {
              const int idx = b0 + __popc(hm0 & below);
              if (idx < cap) {
                const size_t off = colbase + (size_t)idx * kLeaf + (size_t)t0;
                a.list[off] = jk;
                a.dcache[off] = d20;
              }
            }
            if (h1) {
              const int idx = b1 + __popc(hm1 & below);
              if (idx < cap) {
                const size_t off = colbase + (size_t)idx * kLeaf + (size_t)t1;
                a.list[off] = jk;
                a.dcache[off] = d21;
              }
            }
            if ((int)lane_id() == t0) c += __popc(hm0);
            if ((int)lane_id() == t1) c += __popc(hm1);  // t1 != t0 whenever hm1 != 0
          }
          return;
        }
        stage_leaf(a.pos, n, lj, sm, pf);
        if (on && lane_box_hits(lb, bl, bh)) {
#pragma unroll 8
          for (int k = 0; k < cntj; k++) {
            if (certainly_outside(pf, thr, sm.sf[k])) continue;
            const double d2 = ds2_exact(xi - sm.sx[k], yi - sm.sy[k], zi - sm.sz[k]);
            if (d2 < r2) {
              if (c < cap) {
                lst[(size_t)c * kLeaf] = lj * kLeaf + k;
                if (fill) dc[(size_t)c * kLeaf] = d2;
              }
              c++;
              if (dwalk && iterate) {
                const double u = 2 * sqrt(d2) / w;
                sf += k_ig<double>(u);
                sg -= k_digdh<double>(u);
              }
            }
          }
        }
      });
      if (fill) {
        if (c <= cap) {
          ncache = c;
          cache_r2 = r2;
        } else {
          direct = true;  // evaluated by a walk at w from the next round on
        }
      }
      if (dwalk) {
        w_list = w;
        cnt_list = c;
        if (iterate) evaluated = true;
        else pending = false;
      }
    }
    if (iterate && !direct && w2 <= cache_r2) {
      // the cache does not fit in L2 at large N: load a batch of entries
      // before using any (the sums keep the entries' order)
      for (int k0 = 0; k0 < ncache; k0 += kEvalBatch) {
        double d2[kEvalBatch];
#pragma unroll
        for (int q = 0; q < kEvalBatch; q++) d2[q] = k0 + q < ncache ? dc[(size_t)(k0 + q) * kLeaf] : w2;
#pragma unroll
        for (int q = 0; q < kEvalBatch; q++) {
          if (d2[q] < w2) {
            const double u = 2 * sqrt(d2[q]) / w;
            sf += k_ig<double>(u);
            sg -= k_digdh<double>(u);
          }
        }
      }
      evaluated = true;
    }
    if (!evaluated) continue;
    advance(sf, sg);
    if (phase == kDone) {
      if (direct) {
        pending = w != w_list;
      } else if (!(__dmul_rn(w, w) <= cache_r2)) {
        direct = true;  // final range outside the cache: list by a walk
        pending = true;
      }
    }
  }
  if (valid && !direct && cache_r2 >= 0 && spec_cnt < 0) {
    // the final list: the cached entries inside the final range, in order
    const double w2 = __dmul_rn(w, w);
    int c = 0;
    // batches loaded before any store: a store goes to a slot c <= k below
    // every slot a later batch reads
    for (int k0 = 0; k0 < ncache; k0 += kCompactBatch) {
      double d2[kCompactBatch];
      int j[kCompactBatch];
#pragma unroll
      for (int q = 0; q < kCompactBatch; q++) {
        const bool in = k0 + q < ncache;
        d2[q] = in ? dc[(size_t)(k0 + q) * kLeaf] : w2;
        j[q] = in ? lst[(size_t)(k0 + q) * kLeaf] : 0;
      }
#pragma unroll
      for (int q = 0; q < kCompactBatch; q++) {
        if (d2[q] < w2) {
          lst[(size_t)c * kLeaf] = j[q];
          c++;
        }
      }
    }
    cnt_list = c;
  }
  if (!stack_ok && lane_id() == 0) raise_flag(a.flags, SPH_FLAG_STACK_OVERFLOW);
  if (cnt_list > cap) raise_flag(a.flags, SPH_FLAG_NGB_OVERFLOW);
  if (valid) {
    a.pos[s].w = (w > 0) ? w : 0.0;
    a.n_ngb[s] = cnt_list;
    if (a.nevals) a.nevals[s] = nev;
  }
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32, 6) k_solve_range(SolveArgs a) {
  __shared__ WarpSmem smem[kWarpsPerBlock];
  WarpSmem &sm = smem[threadIdx.x >> 5];
  const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (!a.queue) {
    const int leaf = a.leaf0 + wid;
    if (leaf < a.leaf1) solve_leaf(a, sm, leaf, false);
    return;
  }
  // the leaves the speculative pass left, handed out to the resident warps
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int count = *a.queue_count;
  for (int q = wid; q < count; q += nw) {
    solve_leaf(a, sm, a.queue[q], true);
    __syncwarp();
  }
}

struct FindArgs {
  TreeView t;
  const double4 *pos;
  int *n_ngb;
  int *list;       // [leaf][k][lane], cap entries per lane
  int cap;
  unsigned *flags;
  int leaf0, leaf1;  // leaves processed by this launch
};

// dev_find_ngb (dev_find_ngb.cu:13-87): every j with ds2 < range_i^2, in
// ascending slot order, written to the leaf-sliced list (entry k of lane l of
// leaf L at ((L * cap) + k) * 32 + l: the lanes of a warp read and write
// their k-th neighbours in one 128-byte transaction).
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_find_ngb(FindArgs a) {
  __shared__ WarpSmem smem[kWarpsPerBlock];
  WarpSmem &sm = smem[threadIdx.x >> 5];
  const int leaf = a.leaf0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int n = a.t.n;
  if (leaf >= a.leaf1) return;
  const int s = leaf * kLeaf + (int)lane_id();
  const bool valid = s < n;
  double xi = 0, yi = 0, zi = 0, w = 0;
  if (valid) {
    const double4 p = a.pos[s];
    xi = p.x; yi = p.y; zi = p.z; w = p.w;
  }
  const bool on = valid && w > 0;
  float ql[3], qh[3];
  warp_query_box(on, xi, yi, zi, w, ql, qh);
  const double w2 = __dmul_rn(w, w);
  const Prefilter pf = make_prefilter(on, xi, yi, zi);
  const float thr = prefilter_threshold(pf, w);
  int cnt = 0;
  int *out = a.list + (size_t)leaf * a.cap * kLeaf + lane_id();
  const int cap = a.cap;
  bool ok = true;
  if (__any_sync(kFull, on)) {
    const LaneBox lb = lane_query_box(xi, yi, zi, w);
    const unsigned onmask = share_lane_boxes(sm, lb, on);
    ok = walk_leaves(a.t, ql, qh, sm.lbox, onmask, sm.stack, sm.cbox, [&](int lj, const float *bl, const float *bh) {
      stage_leaf(a.pos, n, lj, sm, pf);
      const int m = min(kLeaf, n - lj * kLeaf);
      if (on && lane_box_hits(lb, bl, bh)) {
#pragma unroll 8
        for (int k = 0; k < m; k++) {
          if (certainly_outside(pf, thr, sm.sf[k])) continue;
          const double d2 = ds2_exact(xi - sm.sx[k], yi - sm.sy[k], zi - sm.sz[k]);
          if (d2 < w2) {
            if (cnt < cap) out[(size_t)cnt * kLeaf] = lj * kLeaf + k;
            cnt++;
          }
        }
      }
    });
  }
  if (!ok && lane_id() == 0) raise_flag(a.flags, SPH_FLAG_STACK_OVERFLOW);
  if (cnt > cap) raise_flag(a.flags, SPH_FLAG_NGB_OVERFLOW);
  if (valid) a.n_ngb[s] = cnt;
}

// scratch of the two-kernel solve: the queue count, the queue, the saved states
size_t solve_work_bytes(int n, int nleaf) {
  return 256 + ((size_t)nleaf * sizeof(int) + 255) / 256 * 256 + (size_t)n * sizeof(SolveSave);
}

// leaves [leaf0, leaf1) (a shard's range, or 0 and the leaf count)
int launch_solve_range(const TreeView &t, double4 *pos, int *nevals, unsigned *flags, const sph_params &p,
                       int *n_ngb, int *list, double *dcache, int cap, void *work, int leaf0, int leaf1,
                       cudaStream_t st) {
  SolveArgs a;
  a.t = t; a.pos = pos; a.nevals = nevals; a.flags = flags;
  a.n_ngb = n_ngb; a.list = list; a.dcache = dcache; a.cap = cap;
  a.n_target = p.n_target; a.rel_err = p.rel_err; a.f_scale = p.f_scale; a.max_iter = p.max_iter;
  a.leaf0 = leaf0; a.leaf1 = leaf1;
  a.queue = nullptr; a.queue_count = nullptr; a.save = nullptr;
  const int warps = leaf1 - leaf0;
  if (warps <= 0) return 0;
  const int blocks = (warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
  // the speculative first evaluation pays when the previous range is likely
  // to pass the tolerance test already (not with a tight tolerance)
  if (p.rel_err < 1e-8 || !work) {
    k_solve_range<<<blocks, kWarpsPerBlock * 32, 0, st>>>(a);
    return 1;
  }
  char *w = (char *)work;
  a.queue_count = (int *)w;
  a.queue = (int *)(w + 256);
  a.save = (SolveSave *)(w + 256 + ((size_t)t.count[0] * sizeof(int) + 255) / 256 * 256);
  cudaMemsetAsync(a.queue_count, 0, sizeof(int), st);
  k_solve_spec<<<blocks, kWarpsPerBlock * 32, 0, st>>>(a);
  // the resumed leaves (about a tenth in steady state) on the resident warps
  const int resident = 148 * 6;
  k_solve_range<<<blocks < resident ? blocks : resident, kWarpsPerBlock * 32, 0, st>>>(a);
  return 2;
}

int launch_find_ngb(const TreeView &t, const double4 *pos, int *n_ngb, int *list, int cap, unsigned *flags,
                    int leaf0, int leaf1, cudaStream_t st) {
  FindArgs a;
  a.t = t; a.pos = pos; a.n_ngb = n_ngb; a.list = list; a.cap = cap; a.flags = flags;
  a.leaf0 = leaf0; a.leaf1 = leaf1;
  const int warps = leaf1 - leaf0;
  if (warps <= 0) return 0;
  k_find_ngb<<<(warps + kWarpsPerBlock - 1) / kWarpsPerBlock, kWarpsPerBlock * 32, 0, st>>>(a);
  return 1;
}

}  // namespace sph
