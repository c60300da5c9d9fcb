// knn_warp.cu -- warp-converged exact kNN for queries in leaf order (the default
// kernel of ckd_knn / ckd_forest_knn and of the learned-bound search).
//
// The reference walks the tree once per query (cosmokdtree.f90:549-675, the
// best-first queue; :782-853, the hyperplane DFS when periodic) and scans every
// visited leaf point by point (:654-664, :804-814).  Here the 32 lanes of a warp
// hold 32 queries adjacent in leaf order and the warp walks the tree once for all
// of them:
//  1. the distinct leaves the queries fall in are scanned first, which fills every
//     lane's heap with near points;
//  2. the walk starts at the lowest ancestor of the first query's leaf whose
//     sliding-midpoint cell strictly contains every lane's current k-th-distance
//     ball (cells partition space, so no point outside that subtree can enter any
//     heap), else at the root;
//  3. an internal node is expanded when at least one lane's FP32 lower bound
//     reaches it (ballot): both children are tested from the parent's child-pair
//     record, the child more lanes prefer is taken first and the other goes on a
//     warp stack held one entry per lane register, retested when popped;
//  4. a leaf's points are staged once in shared memory by one coalesced load and
//     every lane screens all of them for its own query (broadcast reads); the
//     points that pass are evaluated in FP64 with the reference arithmetic
//     (cosmokdtree.f90:1441-1465) from the chunk's FP64 records, staged the same
//     way, and offered to the lane's compact heap.
// Results equal the reference's under (d2, id) order.
//
// Screens.  Points are screened on their absolute coordinates rounded to FP32
// (v = fl32(p)) against q32 = fl32(q): fl32(v_j - q32_j) differs from p_j - q_j
// by at most 2^-23 (B_j + |q_j|) (three roundings of relative size 2^-24, B_j
// bounding every coordinate), so e_j = 2^-22 (B_j + |q_j|) is a bound with a
// factor-2 margin; with E = |e|, |p - q| >= |y| - E for the FP32 difference
// vector y, and the FP32 sum s of the y_j^2 satisfies s >= |y|^2 (1 - 2^-22).  A
// point whose FP64 squared distance is <= tau therefore has
// s <= (sqrt(tau) + E)^2 / (1 - 2^-20), the threshold used (rounded upwards).
// Node boxes are screened as in the per-lane kernel (outward-rounded FP32 boxes
// minus a per-axis slack).
//
// Periodic trees.  While every lane's k-th-distance ball lies strictly inside the
// fundamental box, the closest image of any point that can still enter a heap is
// the point itself (two points of the box never differ by a multiple of L inside
// a ball that does not reach its faces), so the direct (non-wrapping) box and
// point screens are valid lower bounds; they are used from the moment that holds
// for the whole warp (the balls only shrink).  Otherwise the minimum-image forms
// are used, with e_j widened by 2^-22 L_j.  Exact FP64 distances always use the
// minimum image (cosmokdtree.f90:1455).
//
// BOUNDED (learned path): heaps start full of sentinels at the predicted radius;
// lanes that still hold a sentinel at the end are appended to miss[] for the
// unbounded rerun and their rows are not written.
#include <algorithm>

#include "ckd_common.cuh"
#include "ckd_knn.cuh"

namespace ckd {

namespace {

constexpr int kWarpStack = 128;  // warp DFS stack entries, 4 registers per lane
constexpr int kChunk = 32;       // points staged per pass
constexpr int32_t kNone = -1;    // "no node" (leaves are stored as ~id, ids >= 1)
constexpr float kGrow = 1.0000020f;  // > 1 / (1 - 2^-20)

// shared memory per warp: the compact heaps and one staging buffer (a chunk's
// FP32 absolute points, then, when some lane has a pass, its FP64 records)
__host__ __device__ inline size_t warp_smem_per_warp(int k, int d) {
  return compact_heap_bytes(k) + (size_t)kChunk * ((d + 3) / 4) * sizeof(double4);
}

// Warp stack of node ids, entry i in register i / 32 of lane i % 32.
struct WarpStack {
  int32_t r0, r1, r2, r3;
  int top;
  __device__ __forceinline__ void push(int32_t v, int lane) {
    const int sr = top >> 5;
    if (lane == (top & 31)) {
      r0 = sr == 0 ? v : r0;
      r1 = sr == 1 ? v : r1;
      r2 = sr == 2 ? v : r2;
      r3 = sr == 3 ? v : r3;
    }
    ++top;
  }
  __device__ __forceinline__ int32_t pop() {
    --top;
    const int sr = top >> 5;
    const int32_t x = sr == 0 ? r0 : (sr == 1 ? r1 : (sr == 2 ? r2 : r3));
    return __shfl_sync(0xffffffffu, x, top & 31);
  }
};

// Per-lane query state of the warp search.
template <int D>
struct WarpQuery {
  double q[D];
  float q32[D];
  float dlt[D];  // node-box slack, 2^-21 (|q| + B)
  float xl[D];   // q32 + dlt (rounded up) and q32 - dlt (rounded down): the direct
  float xh[D];   // box gap on axis j is max(lo - xl, xh - hi, 0)
  float E;       // point-screen error bound, direct screen
  float Ew;      // point-screen error bound, minimum-image screen
};

// FP32 lower bound of the squared distance to a box [lo, hi] (registers).
template <int D, bool WRAP, int W>
__device__ __forceinline__ float box_lb(const TreeView& tv, const WarpQuery<D>& wq,
                                        const float (&lo)[W], const float (&hi)[W]) {
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    float g;
    if (!WRAP) {
      g = fmaxf(fmaxf(lo[j] - wq.xl[j], wq.xh[j] - hi[j]), 0.0f);
    } else {
      const float x = wq.q32[j];
      if (x >= lo[j] - wq.dlt[j] && x <= hi[j] + wq.dlt[j]) {
        g = 0.0f;
      } else {
        const float L = (float)tv.L[j];
        const float t1 = fabsf(x - lo[j]), t2 = fabsf(x - hi[j]);
        g = fmaxf(fminf(fminf(t1, L - t1), fminf(t2, L - t2)) - wq.dlt[j], 0.0f);
      }
    }
    s = fmaf(g, g, s);
  }
  return s * kShrink;
}

template <int D, bool WRAP>
__device__ __forceinline__ float node_lb(const TreeView& tv, const WarpQuery<D>& wq, int32_t node) {
  constexpr int NV = (D + 3) / 4;
  float lo[4 * NV], hi[4 * NV];
  const float2* b = reinterpret_cast<const float2*>(tv.box32 + (int64_t)node * 2 * D);
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const float2 lh = __ldg(b + j);
    lo[j] = lh.x;
    hi[j] = lh.y;
  }
#pragma unroll
  for (int j = D; j < 4 * NV; ++j) lo[j] = hi[j] = 0.0f;
  return box_lb<D, WRAP>(tv, wq, lo, hi);
}

// Screen leaf-ordered positions [start, start + count) for every lane in `ing`
// and offer the passes to the lanes' heaps.  Warp-uniform.
template <int D, bool PER, bool WRAP>
__device__ __forceinline__ void warp_scan_leaf(const TreeView& tv, int32_t start, int32_t count,
                                               bool ing, const WarpQuery<D>& wq, CompactHeap& hp,
                                               const CompactCtx<D, PER>& cx, int k,
                                               double4* stage, int lane,
                                               unsigned long long (&st)[8]) {
  constexpr int NV = (D + 3) / 4;
  constexpr unsigned FULL = 0xffffffffu;
  float4* stage32 = reinterpret_cast<float4*>(stage);
  if (lane == 0) {
    st[2] += 1;
    st[3] += count;
  }
  const float E = WRAP ? wq.Ew : wq.E;
  for (int base = 0; base < count; base += kChunk) {
    const int cnt = min(kChunk, count - base);
    const int32_t p0 = start + base;
    __syncwarp();  // the previous chunk's readers are done with the stage
    if (lane < cnt) {
#pragma unroll
      for (int h = 0; h < NV; ++h)
        stage32[lane * NV + h] = __ldg(&tv.pts32[(int64_t)(p0 + lane) * NV + h]);
    }
    __syncwarp();
    float thr = -1.0f;
    if (ing) {
      const float t = __fadd_ru(sqrt_up(hp.wd32), E);
      thr = __fmul_ru(__fmul_ru(t, t), kGrow);
    }
    unsigned mask = 0;
#pragma unroll 4
    for (int i = 0; i < cnt; ++i) {
      float v[4 * NV];
#pragma unroll
      for (int h = 0; h < NV; ++h) {
        const float4 f = stage32[i * NV + h];
        v[4 * h] = f.x;
        v[4 * h + 1] = f.y;
        v[4 * h + 2] = f.z;
        v[4 * h + 3] = f.w;
      }
      float s = 0.0f;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        float a = v[j] - wq.q32[j];
        if (WRAP) {
          a = fabsf(a);
          a = fminf(a, (float)tv.L[j] - a);
        }
        s = fmaf(a, a, s);
      }
      if (s <= thr) mask |= 1u << i;
    }
    if (!__any_sync(FULL, mask != 0)) continue;
    st[5] += __popc(mask);
    __syncwarp();
    if (lane < cnt) {
#pragma unroll
      for (int h = 0; h < NV; ++h) {
        const double2* r = reinterpret_cast<const double2*>(tv.pts64 + (int64_t)(p0 + lane) * NV + h);
        const double2 a = __ldg(r), b = __ldg(r + 1);
        stage[lane * NV + h] = make_double4(a.x, a.y, b.x, b.y);
      }
    }
    __syncwarp();
    while (mask) {
      const int i = __ffs(mask) - 1;
      mask &= mask - 1;
      double v[4 * NV];
#pragma unroll
      for (int h = 0; h < NV; ++h) {
        const double4 f = stage[i * NV + h];
        v[4 * h] = f.x;
        v[4 * h + 1] = f.y;
        v[4 * h + 2] = f.z;
        v[4 * h + 3] = f.w;
      }
      double d2 = 0.0;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        double dx = dsub(v[j], wq.q[j]);
        if (PER) dx = min_image(dx, tv.L[j]);
        d2 = (j == 0) ? dmul(dx, dx) : dadd(d2, dmul(dx, dx));
      }
      if (compact_offer<D, PER>(hp, k, cx, wq.q, d2, p0 + i)) st[6] += 1;
    }
  }
}

// Phase 3: the warp's walk from `node` over the subtree, for the lanes in `ing`.
template <int D, bool PER, bool WRAP>
__device__ __forceinline__ void warp_walk(const TreeView& tv, int32_t node, bool ing,
                                          int32_t myscan, const WarpQuery<D>& wq,
                                          CompactHeap& hp, const CompactCtx<D, PER>& cx, int k,
                                          double4* stage, int lane,
                                          unsigned long long (&st)[8]) {
  constexpr int NV = (D + 3) / 4;
  constexpr int PF = pair_f4(D);
  constexpr unsigned FULL = 0xffffffffu;
  WarpStack stk{kNone, kNone, kNone, kNone, 0};
  const NodeMeta m0 = load_meta(tv.meta, node);
  if (m0.left < 0) {  // the walk starts at a leaf
    if (!__any_sync(FULL, myscan == m0.start))
      warp_scan_leaf<D, PER, WRAP>(tv, m0.start, m0.count, ing, wq, hp, cx, k, stage, lane, st);
    return;
  }
  for (;;) {
    // ---- expand an internal node from its child-pair record
    if (lane == 0) st[0] += 1;
    const float4* rec = tv.pair + (int64_t)node * PF;
    float lo_l[4 * NV], hi_l[4 * NV], lo_r[4 * NV], hi_r[4 * NV];
#pragma unroll
    for (int h = 0; h < NV; ++h) {
      const float4 a = __ldg(rec + h), b = __ldg(rec + NV + h);
      const float4 c = __ldg(rec + 2 * NV + h), d = __ldg(rec + 3 * NV + h);
      lo_l[4 * h] = a.x; lo_l[4 * h + 1] = a.y; lo_l[4 * h + 2] = a.z; lo_l[4 * h + 3] = a.w;
      hi_l[4 * h] = b.x; hi_l[4 * h + 1] = b.y; hi_l[4 * h + 2] = b.z; hi_l[4 * h + 3] = b.w;
      lo_r[4 * h] = c.x; lo_r[4 * h + 1] = c.y; lo_r[4 * h + 2] = c.z; lo_r[4 * h + 3] = c.w;
      hi_r[4 * h] = d.x; hi_r[4 * h + 1] = d.y; hi_r[4 * h + 2] = d.z; hi_r[4 * h + 3] = d.w;
    }
    const int4 info = __ldg(reinterpret_cast<const int4*>(rec + 4 * NV));
    const int4 rng = __ldg(reinterpret_cast<const int4*>(rec + 4 * NV + 1));
    const float ml = box_lb<D, WRAP>(tv, wq, lo_l, hi_l);
    const float mr = box_lb<D, WRAP>(tv, wq, lo_r, hi_r);
    const bool nl = ing && ml <= hp.wd32, nr = ing && mr <= hp.wd32;
    const unsigned bl = __ballot_sync(FULL, nl), br = __ballot_sync(FULL, nr);
    if (bl | br) {
      bool lf = bl != 0;
      if (bl && br) {
        const unsigned vl = __ballot_sync(FULL, nl && (!nr || ml <= mr));
        lf = 2 * __popc(vl) >= __popc(bl | br);
        stk.push(lf ? (info.w ? ~info.y : info.y) : (info.z ? ~info.x : info.x), lane);
      }
      const bool leaf = lf ? info.z != 0 : info.w != 0;
      if (!leaf) {
        node = lf ? info.x : info.y;
        continue;
      }
      const int32_t ls = lf ? rng.x : rng.z, lc = lf ? rng.y : rng.w;
      if (!__any_sync(FULL, myscan == ls))
        warp_scan_leaf<D, PER, WRAP>(tv, ls, lc, ing, wq, hp, cx, k, stage, lane, st);
    }
    // ---- the most recently deferred subtree still within some lane's reach
    for (;;) {
      if (stk.top == 0) return;
      const int32_t e = stk.pop();
      if (lane == 0) st[1] += 1;
      const int32_t id = e < 0 ? ~e : e;
      const float mb = node_lb<D, WRAP>(tv, wq, id);
      if (!__any_sync(FULL, ing && mb <= hp.wd32)) continue;
      if (e >= 0) {
        node = e;
        break;
      }
      const NodeMeta lm = load_meta(tv.meta, id);
      if (!__any_sync(FULL, myscan == lm.start))
        warp_scan_leaf<D, PER, WRAP>(tv, lm.start, lm.count, ing, wq, hp, cx, k, stage, lane, st);
    }
  }
}

template <int D, bool PER, bool BOUNDED>
__global__ void __launch_bounds__(128, 6) k_knn_warp(TreeView tv, const double* __restrict__ Q,
                                                  const int32_t* __restrict__ order,
                                                  const int32_t* __restrict__ qleaf,
                                                  const int32_t* __restrict__ qroot, int64_t nq,
                                                  int k, int sorted, double* __restrict__ dist,
                                                  int64_t* __restrict__ idx,
                                                  unsigned long long* __restrict__ stats,
                                                  const double* __restrict__ r2,
                                                  int32_t* __restrict__ miss,
                                                  unsigned* __restrict__ nmiss) {
  constexpr int NV = (D + 3) / 4;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(32) unsigned char smem[];
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint2* H0 = reinterpret_cast<uint2*>(smem) + (size_t)w * 32 * (k + 1);
  double4* stage = reinterpret_cast<double4*>(smem + (size_t)nw * compact_heap_bytes(k)) +
                   (size_t)w * kChunk * NV;
  const int64_t gw = (int64_t)blockIdx.x * nw + w;
  const int64_t slot = gw * 32 + lane;
  const bool valid = slot < nq;
  const int64_t qi = valid ? (int64_t)order[slot] : 0;
  WarpQuery<D> wq;
  {
    float e2 = 0.0f, e2w = 0.0f;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      wq.q[j] = valid ? Q[qi * D + j] : 0.0;
      wq.q32[j] = __double2float_rn(wq.q[j]);
      wq.dlt[j] = kTwoM21 * (fabsf(wq.q32[j]) + tv.slack[j]) * 1.0001f;
      wq.xl[j] = __fadd_ru(wq.q32[j], wq.dlt[j]);
      wq.xh[j] = __fsub_rd(wq.q32[j], wq.dlt[j]);
      const float ej = __fmaf_ru(kTwoM22, __fadd_ru(tv.slack[j], fabsf(wq.q32[j])), 1e-37f);
      e2 = __fmaf_ru(ej, ej, e2);
      if (PER) {
        const float ejw = __fmaf_ru(kTwoM22, (float)tv.L[j], ej);
        e2w = __fmaf_ru(ejw, ejw, e2w);
      }
    }
    wq.E = sqrt_up(e2);
    wq.Ew = PER ? sqrt_up(e2w) : wq.E;
  }
  float skey = FLT_MAX;
  int32_t spos = kPosMissing;
  float wd32 = valid ? FLT_MAX : -1.0f;
  double rr = CKD_HUGE;
  if (BOUNDED && valid) {
    const double b = r2[qi];
    if (b < CKD_HUGE) {
      rr = b;
      skey = __double2float_rn(b);
      spos = kPosBound;
      wd32 = __double2float_ru(b);
    }
  }
  const CompactCtx<D, PER> cx{tv, rr};
  CompactHeap hp{H0 + lane, 0u, 0, 0.0f};
  compact_init<D, PER>(hp, k, skey, spos, wd32);
  const int32_t myleaf = valid ? qleaf[qi] : -1;
  const int32_t myroot = valid ? (qroot ? qroot[qi] : 0) : -1;

  // ---- 1. the warp's own leaves
  int32_t myscan = kNone;  // lane i holds the first position of the i-th leaf scanned
  {
    const unsigned peers = __match_any_sync(FULL, myleaf);
    unsigned todo = __ballot_sync(FULL, valid && (__ffs(peers) - 1) == lane);
    int nscan = 0;
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const int32_t leaf = __shfl_sync(FULL, myleaf, src);
      const int32_t lroot = __shfl_sync(FULL, myroot, src);
      const NodeMeta lm = load_meta(tv.meta, leaf);
      if (lane == nscan) myscan = lm.start;
      ++nscan;
      warp_scan_leaf<D, PER, PER>(tv, lm.start, lm.count, valid && myroot == lroot, wq, hp, cx, k,
                                  stage, lane, st);
    }
    if (lane == 0) st[4] += nscan;
  }

  // ---- 2./3. one walk per tree among the warp's queries (one tree unless a forest)
  unsigned pending = __ballot_sync(FULL, valid);
  while (pending) {
    const int src = __ffs(pending) - 1;
    const int32_t root = __shfl_sync(FULL, myroot, src);
    const bool ing = valid && myroot == root;
    pending &= ~__ballot_sync(FULL, ing);
    int32_t node = root;
    bool wrap_free = !PER;
    if (!__any_sync(FULL, ing && hp.wd32 >= FLT_MAX)) {
      const float r32 = ing ? sqrt_up(hp.wd32) : 0.0f;
      if (PER) {
        bool inside = true;
#pragma unroll
        for (int j = 0; j < D; ++j)
          inside = inside && __fadd_ru(__fadd_ru(fabsf(wq.q32[j]), r32), wq.dlt[j]) <
                                 0.5f * (float)tv.L[j];
        wrap_free = __all_sync(FULL, !ing || inside);
      }
      int32_t a = __shfl_sync(FULL, myleaf, src);
      while (a != root && a >= 0) {
        const float* c = tv.cell32 + (int64_t)a * 2 * D;
        bool inside = true;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          const float2 lh = __ldg(reinterpret_cast<const float2*>(c) + j);
          inside = inside && __fsub_rd(__fsub_rd(wq.q32[j], r32), wq.dlt[j]) > lh.x &&
                   __fadd_ru(__fadd_ru(wq.q32[j], r32), wq.dlt[j]) < lh.y;
        }
        if (__all_sync(FULL, !ing || inside)) break;
        a = __ldg(&tv.meta[a].parent);
        if (lane == 0) st[7] += 1;
      }
      node = a >= 0 ? a : root;
    }
    if (!PER || wrap_free)
      warp_walk<D, PER, false>(tv, node, ing, myscan, wq, hp, cx, k, stage, lane, st);
    else
      warp_walk<D, PER, PER>(tv, node, ing, myscan, wq, hp, cx, k, stage, lane, st);
  }

  if (stats) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = st[c];
      if (c == 5 || c == 6)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
  const bool missed = BOUNDED && valid && hp.wp == kPosBound;
  unsigned missmask = 0;
  if (BOUNDED) {
    missmask = __ballot_sync(FULL, missed);
    if (missmask) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(nmiss, (unsigned)__popc(missmask));
      base = __shfl_sync(FULL, base, 0);
      if (missed) miss[base + __popc(missmask & ((1u << lane) - 1u))] = (int32_t)qi;
    }
  }
  if (sorted && valid && !missed) compact_sort<D, PER>(hp.H, k, cx, wq.q);
  __syncwarp();
  compact_write<D, PER>(tv, H0, lane, gw, nq, order, wq.q, k, missmask, dist, idx);
}

template <int D, bool PER, bool BOUNDED>
ckd_status launch_one(const ckd_tree* t, const double* q, const int32_t* order,
                      const int32_t* qleaf, const int32_t* qroot, int64_t nq, int k, int sorted,
                      double* dist, int64_t* idx, const double* r2, int32_t* miss,
                      unsigned* nmiss, unsigned long long* stats, cudaStream_t s) {
  const int nw = 4;
  const size_t sm = (size_t)nw * warp_smem_per_warp(k, D);
  const unsigned blocks = (unsigned)cdiv(cdiv(nq, 32), nw);
  CKD_CUDA(cudaFuncSetAttribute(k_knn_warp<D, PER, BOUNDED>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_knn_warp<D, PER, BOUNDED><<<blocks, nw * 32, sm, s>>>(t->view(), q, order, qleaf, qroot, nq,
                                                          k, sorted, dist, idx, stats, r2, miss,
                                                          nmiss);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

}  // namespace

bool knn_warp_supported(const ckd_tree* t, int k) {
  return k >= 1 && k <= kSmemK && t->screen_ok && t->depth < kWarpStack - 1;
}

template <int D, bool PER>
ckd_status knn_warp_launch(const ckd_tree* t, const double* q, const int32_t* order,
                           const int32_t* qleaf, const int32_t* qroot, int64_t nq, int k,
                           int sorted, double* dist, int64_t* idx, const double* r2,
                           int32_t* miss, unsigned* nmiss, unsigned long long* stats,
                           cudaStream_t s) {
  if (nq <= 0) return CKD_OK;
  if (!order || !qleaf || !knn_warp_supported(t, k))
    return fail(CKD_ERR_BAD_ARG, "internal error: warp kNN kernel outside its limits");
  if (r2)
    return launch_one<D, PER, true>(t, q, order, qleaf, qroot, nq, k, sorted, dist, idx, r2, miss,
                                     nmiss, stats, s);
  return launch_one<D, PER, false>(t, q, order, qleaf, qroot, nq, k, sorted, dist, idx, nullptr,
                                    nullptr, nullptr, stats, s);
}

#define CKD_WI(DD)                                                                              \
  template ckd_status knn_warp_launch<DD, false>(const ckd_tree*, const double*, const int32_t*, \
                                                 const int32_t*, const int32_t*, int64_t, int,   \
                                                 int, double*, int64_t*, const double*,          \
                                                 int32_t*, unsigned*, unsigned long long*,       \
                                                 cudaStream_t);                                  \
  template ckd_status knn_warp_launch<DD, true>(const ckd_tree*, const double*, const int32_t*,  \
                                                const int32_t*, const int32_t*, int64_t, int,    \
                                                int, double*, int64_t*, const double*,           \
                                                int32_t*, unsigned*, unsigned long long*,        \
                                                cudaStream_t);
CKD_WI(1) CKD_WI(2) CKD_WI(3) CKD_WI(4) CKD_WI(5) CKD_WI(6) CKD_WI(7) CKD_WI(8)
#undef CKD_WI

}  // namespace ckd
