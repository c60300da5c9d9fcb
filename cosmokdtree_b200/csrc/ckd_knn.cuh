// ckd_knn.cuh -- device pieces shared by the kNN kernels: the FP32 screen of
// node boxes and leaf points, and the compact per-lane max-heap in shared memory
// (cosmokdtree.f90:859-905 keeps the k best in a max-heap whose root is the
// current k-th; here the heap is ordered by (FP64 d2, id) exactly).
#pragma once
#include "ckd_common.cuh"
#include "ckd_traverse.cuh"

namespace ckd {

CKD_LD_BEGIN

constexpr int kSmemK = 64;        // largest k whose heaps live in shared memory
constexpr int kLaneStack = 128;   // per-lane traversal stack of k_knn_lane2

constexpr float kTwoM21 = 4.76837158203125e-07f;  // 2^-21
constexpr float kTwoM22 = 2.384185791015625e-07f;  // 2^-22
constexpr float kShrink = 0.99999905f;             // 1 - 2^-20

template <int D, bool PER>
struct QueryScreen {
  float q32[D];
  float dlt[D];  // node-gap slack 2^-21 (|q| + B)
};

// FP32 lower bound of the FP64 squared distance from the query to a node's box
// (outward-rounded FP32 box minus the per-axis slack, then shrunk by the
// relative rounding of the sum).
template <int D, bool PER>
__device__ __forceinline__ float node_mind_lb(const TreeView& tv, const QueryScreen<D, PER>& qs,
                                              int32_t node) {
  const float* b = tv.box32 + (int64_t)node * 2 * D;
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    float2 lh = CKD_LDT(reinterpret_cast<const float2*>(b) + j);
    float x = qs.q32[j], g;
    if (x >= lh.x - qs.dlt[j] && x <= lh.y + qs.dlt[j]) {
      g = 0.0f;
    } else if (!PER) {
      g = fmaxf(lh.x - x, x - lh.y) - qs.dlt[j];
    } else {
      float L = (float)tv.L[j];
      float t1 = fabsf(x - lh.x), t2 = fabsf(x - lh.y);
      g = fminf(fminf(t1, L - t1), fminf(t2, L - t2)) - qs.dlt[j];
    }
    g = fmaxf(g, 0.0f);
    s = fmaf(g, g, s);
  }
  return s * kShrink;
}

// node_mind_lb for a box held in registers (lo/hi padded to a multiple of 4)
template <int D, bool PER, int W>
__device__ __forceinline__ float box_mind_lb(const TreeView& tv, const QueryScreen<D, PER>& qs,
                                             const float (&lo)[W], const float (&hi)[W]) {
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    float x = qs.q32[j], g;
    if (x >= lo[j] - qs.dlt[j] && x <= hi[j] + qs.dlt[j]) {
      g = 0.0f;
    } else if (!PER) {
      g = fmaxf(lo[j] - x, x - hi[j]) - qs.dlt[j];
    } else {
      float L = (float)tv.L[j];
      float t1 = fabsf(x - lo[j]), t2 = fabsf(x - hi[j]);
      g = fminf(fminf(t1, L - t1), fminf(t2, L - t2)) - qs.dlt[j];
    }
    g = fmaxf(g, 0.0f);
    s = fmaf(g, g, s);
  }
  return s * kShrink;
}

// Upper bound of sqrt(x) for finite x >= 0, used only for screening thresholds:
// the PTX approximate square root (a few ulps of relative error) raised by 2^-15
// and rounded up; subnormal inputs are flushed to zero, so 2^-63 (> the square
// root of any subnormal) is added.
__device__ __forceinline__ float sqrt_up(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return __fmaf_ru(r, 1.0000305f, 1.0842022e-19f);
}

template <int D, bool PER>
__device__ __forceinline__ void init_query_screen(const TreeView& tv, const double (&q)[D],
                                                  QueryScreen<D, PER>& qs) {
#pragma unroll
  for (int j = 0; j < D; ++j) {
    qs.q32[j] = __double2float_rn(q[j]);
    qs.dlt[j] = kTwoM21 * (fabsf(qs.q32[j]) + tv.slack[j]) * 1.0001f;
  }
}

// ------------------------------------------------------------ compact heap
// Each entry is the FP32 rounding of its FP64 squared distance (round to nearest
// is monotone, so a < b in FP32 implies a < b exactly) and the point's
// leaf-ordered position, 8 bytes.  Ties in FP32 are resolved exactly by
// recomputing the FP64 distances from the positions and then comparing ids; the
// FP64 distances of the results are recomputed once for the output.  Slot s
// (1-based) of lane l lives at H[s * 32 + l], so every lane always addresses its
// own bank pair.  Sentinels: position -1 = (HUGE, id -1), position -2 = (r2,
// INT32_MAX) for the bounded search.  The first k entries that enter are placed
// by sifting up from the next free slot (a heap of the entries so far, the
// sentinels parked in the slots past it), so none of them is sifted down through
// k sentinels; once k have entered, every new one replaces the root.
__host__ __device__ inline size_t compact_heap_bytes(int k) { return (size_t)(k + 1) * 32 * 8; }

constexpr int32_t kPosMissing = -1;
constexpr int32_t kPosBound = -2;

// Exact (d2, id) comparisons of heap entries by position.  The query
// coordinates are passed to each call rather than held here, so they stay in
// registers.
template <int D, bool PER>
struct CompactCtx {
  const TreeView& tv;
  double rr;  // bounded sentinel's squared distance
  __device__ __forceinline__ double exact(const double (&q)[D], int32_t p) const {
    return p >= 0 ? point_d2_rec<D, PER>(tv, q, p) : (p == kPosMissing ? CKD_HUGE : rr);
  }
  __device__ __forceinline__ int32_t id(int32_t p) const {
    return p >= 0 ? CKD_LDT(&tv.ids[p]) : (p == kPosMissing ? -1 : 0x7fffffff);
  }
  // exact (d2, id) order of two entries whose FP32 keys are equal
  __device__ __forceinline__ bool tie_before(const double (&q)[D], int32_t a, int32_t b) const {
    const double da = exact(q, a), db = exact(q, b);
    if (da != db) return da < db;
    return id(a) < id(b);
  }
};

// Per-lane heap state: H points at this lane's slot 0 (slot s at H[s * 32]);
// wk / wp are the root's key bits and position, wd32 an FP32 upper bound of the
// root's squared distance (the next float above its key).
struct CompactHeap {
  uint2* H;
  unsigned wk;
  int32_t wp;
  float wd32;
  int cnt;  // entries offered so far while fewer than k (then k)
};

template <int D, bool PER>
__device__ __forceinline__ void compact_init(CompactHeap& h, int k, float skey, int32_t spos,
                                             float wd32) {
  for (int s = 1; s <= k; ++s) h.H[s * 32] = make_uint2(__float_as_uint(skey), (unsigned)spos);
  h.wk = __float_as_uint(skey);
  h.wp = spos;
  h.wd32 = wd32;
  h.cnt = 0;
}

// Offer leaf-ordered point p at exact squared distance d2: it enters iff it ranks
// strictly before the root under (d2, id) (the strict test of cosmokdtree.f90:658
// in canonical form); while fewer than k have entered it is sifted up from the
// next free slot, afterwards the root is replaced and sifted down.  Returns true
// when the heap changed.  BND: a bounded search (its root sentinel is the bound,
// tested before filling; a HUGE root sentinel is beaten by every point).
template <int D, bool PER, bool BND = false>
__device__ __forceinline__ bool compact_offer(CompactHeap& h, int k, const CompactCtx<D, PER>& cx,
                                              const double (&q)[D], double d2, int32_t p) {
  const unsigned kc = __float_as_uint(__double2float_rn(d2));
  // the entry test against the root: for a bounded search the root is the bound's
  // sentinel from the start; otherwise it is a HUGE sentinel, which every point
  // beats, until the heap is full
  auto beats_root = [&]() -> bool {
    if (kc > h.wk) return false;
    if (kc == h.wk) {  // FP32 tie with the root: exact comparison
      const double dr = cx.exact(q, h.wp);
      if (d2 > dr) return false;
      if (d2 == dr && CKD_LDT(&cx.tv.ids[p]) >= cx.id(h.wp)) return false;
    }
    return true;
  };
  if (BND && !beats_root()) return false;
  uint2* H = h.H;
  if (h.cnt < k) {
    // filling: the root is still a sentinel (HUGE, or the bound of a bounded
    // search); sift up from slot cnt + 1 over the real entries, slots past cnt
    // keep their sentinels until the heap is full
    int s = ++h.cnt;
    while (s > 1) {
      const int par = s >> 1;
      const uint2 pe = H[par * 32];
      bool up = kc > pe.x;  // the candidate ranks after its parent
      if (kc == pe.x) {
        const double dp = cx.exact(q, (int32_t)pe.y);
        up = d2 > dp || (d2 == dp && CKD_LDT(&cx.tv.ids[p]) > cx.id((int32_t)pe.y));
      }
      if (!up) break;
      H[s * 32] = pe;
      s = par;
    }
    H[s * 32] = make_uint2(kc, (unsigned)p);
    if (h.cnt == k) {
      const uint2 root = H[32];
      h.wk = root.x;
      h.wp = (int32_t)root.y;
      h.wd32 = __uint_as_float(h.wk + 1u);
    }
    return true;
  }
  if (!BND && !beats_root()) return false;
  int s = 1;
  for (;;) {
    const int l = 2 * s;
    if (l > k) break;
    uint2 ch = H[l * 32];
    int c = l;
    if (l < k) {
      const uint2 r = H[(l + 1) * 32];
      if (ch.x < r.x || (ch.x == r.x && cx.tie_before(q, (int32_t)ch.y, (int32_t)r.y))) {
        ch = r;
        c = l + 1;
      }
    }
    const unsigned kch = ch.x;
    const int32_t pch = (int32_t)ch.y;
    // the candidate stays above the child iff it ranks after it
    bool cand_before = kc < kch;
    if (kc == kch) {
      const double dch = cx.exact(q, pch);
      cand_before = d2 < dch || (d2 == dch && CKD_LDT(&cx.tv.ids[p]) < cx.id(pch));
    }
    if (!cand_before) break;
    H[s * 32] = ch;
    s = c;
  }
  H[s * 32] = make_uint2(kc, (unsigned)p);
  const uint2 root = H[32];
  h.wk = root.x;
  h.wp = (int32_t)root.y;
  h.wd32 = __uint_as_float(h.wk + 1u);
  return true;
}

// After a search that offered fewer than k points, slots cnt + 1 .. k still hold
// sentinels below real entries: sift each one up so the k slots form a heap.
template <int D, bool PER>
__device__ __forceinline__ void compact_finish(CompactHeap& h, int k, const CompactCtx<D, PER>& cx,
                                               const double (&q)[D]) {
  uint2* H = h.H;
  for (int s0 = h.cnt + 1; s0 <= k; ++s0) {
    const uint2 e = H[s0 * 32];
    int s = s0;
    while (s > 1) {
      const int par = s >> 1;
      const uint2 pe = H[par * 32];
      if (!(e.x > pe.x || (e.x == pe.x && cx.tie_before(q, (int32_t)pe.y, (int32_t)e.y)))) break;
      H[s * 32] = pe;
      s = par;
    }
    H[s * 32] = e;
  }
  h.cnt = k;
}

// Heap sort into ascending (d2, id) (replaces the quicksort of
// cosmokdtree.f90:1553-1643): slot 1 ends up holding the nearest.
template <int D, bool PER>
__device__ __forceinline__ void compact_sort(uint2* H, int k, const CompactCtx<D, PER>& cx,
                                             const double (&q)[D]) {
  for (int end = k; end > 1; --end) {
    const uint2 e = H[end * 32];
    H[end * 32] = H[32];
    int s = 1;
    for (;;) {
      const int l = 2 * s;
      if (l >= end) break;
      int c = l;
      uint2 ch = H[l * 32];
      if (l + 1 < end) {
        const uint2 r = H[(l + 1) * 32];
        if (ch.x < r.x || (ch.x == r.x && cx.tie_before(q, (int32_t)ch.y, (int32_t)r.y))) {
          c = l + 1;
          ch = r;
        }
      }
      if (!(e.x < ch.x || (e.x == ch.x && cx.tie_before(q, (int32_t)e.y, (int32_t)ch.y)))) break;
      H[s * 32] = ch;
      s = c;
    }
    H[s * 32] = e;
  }
}

// Warp-cooperative write-out of the warp's 32 result rows (query slot gw*32+qq):
// exact FP64 distances recomputed from the positions, one coalesced row at a
// time.  Rows whose bit is set in `skip` (bounded-search misses) are not written.
// H0 is the warp's heap base (lane 0, slot 0).
template <int D, bool PER>
__device__ __forceinline__ void compact_write(const TreeView& tv, const uint2* H0, int lane,
                                              int64_t gw, int64_t nq, const int32_t* order,
                                              const double (&q)[D], int k, unsigned skip,
                                              double* __restrict__ dist,
                                              int64_t* __restrict__ idx) {
  for (int qq = 0; qq < 32; ++qq) {
    const int64_t s2 = gw * 32 + qq;
    if (s2 >= nq) break;
    double qx[D];
#pragma unroll
    for (int j = 0; j < D; ++j) qx[j] = __shfl_sync(0xffffffffu, q[j], qq);
    if ((skip >> qq) & 1u) continue;
    const int64_t row = order ? (int64_t)order[s2] : s2;
    const uint2* rp = H0 + qq + 32;  // query qq's slot 1
    for (int j = lane; j < k; j += 32) {
      const int32_t p = (int32_t)rp[j * 32].y;
      double d2 = CKD_HUGE;
      int64_t id = -2;
      if (p >= 0) {
        d2 = point_d2_rec<D, PER>(tv, qx, p);
        id = (int64_t)CKD_LDT(&tv.ids[p]);
      }
      dist[row * k + j] = sqrt(d2);
      idx[row * k + j] = id;
    }
  }
}

CKD_LD_END

}  // namespace ckd
