// knn.cu -- exact k-nearest-neighbour search (cosmokdtree.f90:504-905).
//
// One query per lane; the 32 lanes of a warp hold spatially adjacent queries and
// walk the tree together (packet traversal): a node is visited when at least
// one lane's pruning bound reaches it, near child first by majority vote.  Each
// lane keeps its k best (squared distance, id) in a max-heap (root = current
// k-th); a candidate enters iff it ranks strictly before the root under
// (d2, id) order, the canonical form of the strict test at cosmokdtree.f90:658.
// The heap starts full of (HUGE(0.0), -1) sentinels (cosmokdtree.f90:517-518).
// Heaps live lane-major in shared memory for k <= kSmemK, otherwise in the
// caller's output rows.  Distances are FP64, separately rounded, so results are
// bit-identical to the CPU restatement.
#include <algorithm>
#include <mutex>

#include "ckd_common.cuh"
#include "ckd_mlp.cuh"
#include "ckd_scan.cuh"
#include "ckd_traverse.cuh"

namespace ckd {

namespace {

constexpr int kStack = 96;   // per-warp traversal stack in shared memory
float knn_bucket_alpha_v = 1.5f;
float knn_bucket_alpha() { return knn_bucket_alpha_v; }
}  // namespace
void set_knn_bucket_alpha(float a) { knn_bucket_alpha_v = a; }
namespace {

// process-wide traversal statistics of the screened kernel (diagnostics)
__device__ unsigned long long g_knn_stats[8];
bool g_stats_on = false;
unsigned long long* knn_stats_buffer() {
  if (!g_stats_on) return nullptr;
  void* p = nullptr;
  cudaGetSymbolAddress(&p, g_knn_stats);
  return reinterpret_cast<unsigned long long*>(p);
}
constexpr int kSmemK = 64;   // largest k kept in shared memory

// ---------------------------------------------------------- heap storage
// Shared-memory heap: slot s of lane l at [s * 32 + l].
struct SmemHeap {
  double* key;
  int32_t* id;
  int lane;
  __device__ __forceinline__ double k(int s) const { return key[s * 32 + lane]; }
  __device__ __forceinline__ int64_t i(int s) const { return id[s * 32 + lane]; }
  __device__ __forceinline__ void set(int s, double d, int64_t x) {
    key[s * 32 + lane] = d;
    id[s * 32 + lane] = (int32_t)x;
  }
};
// Heap in the caller's output row (keys in dist, ids in idx).
struct RowHeap {
  double* key;
  int64_t* id;
  __device__ __forceinline__ double k(int s) const { return key[s]; }
  __device__ __forceinline__ int64_t i(int s) const { return id[s]; }
  __device__ __forceinline__ void set(int s, double d, int64_t x) {
    key[s] = d;
    id[s] = x;
  }
};

__device__ __forceinline__ bool before(double d1, int64_t i1, double d2, int64_t i2) {
  return d1 < d2 || (d1 == d2 && i1 < i2);
}

// cosmokdtree.f90:859-905: the root is replaced, then sifted down.
template <typename H>
__device__ __forceinline__ void heap_replace_root(H& h, int k, double d2, int64_t id) {
  int i = 0;
  for (;;) {
    int l = 2 * i + 1;
    if (l >= k) break;
    int c = l;
    double dc = h.k(l);
    int64_t ic = h.i(l);
    if (l + 1 < k) {
      double dr = h.k(l + 1);
      int64_t ir = h.i(l + 1);
      if (before(dc, ic, dr, ir)) {
        c = l + 1;
        dc = dr;
        ic = ir;
      }
    }
    if (!before(d2, id, dc, ic)) break;
    h.set(i, dc, ic);
    i = c;
  }
  h.set(i, d2, id);
}

// sift-down inside [0, end) used by the final heap sort
template <typename H>
__device__ __forceinline__ void heap_sift(H& h, int end, double d2, int64_t id) {
  int i = 0;
  for (;;) {
    int l = 2 * i + 1;
    if (l >= end) break;
    int c = l;
    double dc = h.k(l);
    int64_t ic = h.i(l);
    if (l + 1 < end) {
      double dr = h.k(l + 1);
      int64_t ir = h.i(l + 1);
      if (before(dc, ic, dr, ir)) {
        c = l + 1;
        dc = dr;
        ic = ir;
      }
    }
    if (!before(d2, id, dc, ic)) break;
    h.set(i, dc, ic);
    i = c;
  }
  h.set(i, d2, id);
}

// ascending (d2, id) in place (replaces the quicksort of cosmokdtree.f90:1553-1643)
template <typename H>
__device__ __forceinline__ void heap_sort(H& h, int k) {
  for (int end = k - 1; end > 0; --end) {
    double dr = h.k(0);
    int64_t ir = h.i(0);
    double de = h.k(end);
    int64_t ie = h.i(end);
    h.set(end, dr, ir);
    heap_sift(h, end, de, ie);
  }
}

// Packet traversal shared by the shared-memory and output-row heap variants.
template <int D, bool PER, typename H>
__device__ __forceinline__ void knn_walk(const TreeView& tv, const double (&q)[D], bool valid, H& h,
                                         int k, int32_t* stk, int lane) {
  double wd = valid ? CKD_HUGE : -1.0;  // lanes without a query never need a node
  int64_t wid = -1;
  int top = 0;
  if (lane == 0) stk[0] = 0;
  __syncwarp();
  while (top >= 0) {
    int32_t node = stk[top];
    --top;
    __syncwarp();
    NodeMeta m = load_meta(tv.meta, node);
    double md = box_mind2<D, PER>(tv, q, node);
    bool need = md <= wd;
    unsigned nm = __ballot_sync(0xffffffffu, need);
    if (nm == 0) continue;
    if (m.left < 0) {
      for (int i = 0; i < m.count; ++i) {
        int32_t p = m.start + i;
        double d2 = point_d2<D, PER>(tv, q, p);
        if (need && d2 <= wd) {
          int64_t id = __ldg(&tv.ids[p]);
          if (before(d2, id, wd, wid)) {
            heap_replace_root(h, k, d2, id);
            wd = h.k(0);
            wid = h.i(0);
          }
        }
      }
    } else {
      double qa = 0.0;
#pragma unroll
      for (int j = 0; j < D; ++j)
        if (j == m.axis) qa = q[j];
      unsigned lv = __ballot_sync(0xffffffffu, need && qa < m.split);
      bool left_first = 2 * __popc(lv) >= __popc(nm);
      int32_t nearc = left_first ? m.left : m.left + 1;
      int32_t farc = left_first ? m.left + 1 : m.left;
      if (lane == 0) {
        stk[top + 1] = farc;
        stk[top + 2] = nearc;
      }
      top += 2;
      __syncwarp();
    }
  }
}

template <int D, bool PER>
__global__ void __launch_bounds__(128) k_knn_smem(TreeView tv, const double* __restrict__ Q,
                                                  const int32_t* __restrict__ order, int64_t nq,
                                                  int k, int sorted, int32_t* __restrict__ gstack,
                                                  int stack_len, double* __restrict__ dist,
                                                  int64_t* __restrict__ idx) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* keys = reinterpret_cast<double*>(smem) + (size_t)w * k * 32;
  int32_t* ids = reinterpret_cast<int32_t*>(reinterpret_cast<double*>(smem) + (size_t)nw * k * 32) +
                 (size_t)w * k * 32;
  int32_t* stk;
  int64_t gw = (int64_t)blockIdx.x * nw + w;
  if (gstack)
    stk = gstack + gw * stack_len;
  else
    stk = reinterpret_cast<int32_t*>(reinterpret_cast<int32_t*>(reinterpret_cast<double*>(smem) +
                                                                (size_t)nw * k * 32) +
                                     (size_t)nw * k * 32) +
          (size_t)w * kStack;
  int64_t slot = gw * 32 + lane;
  bool valid = slot < nq;
  int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
#pragma unroll
  for (int j = 0; j < D; ++j) q[j] = valid ? Q[qi * D + j] : 0.0;
  SmemHeap h{keys, ids, lane};
  for (int s = 0; s < k; ++s) h.set(s, CKD_HUGE, -1);
  knn_walk<D, PER>(tv, q, valid, h, k, stk, lane);
  if (sorted) heap_sort(h, k);
  __syncwarp();
  // coalesced write-out: for each lane's query, the warp writes its row
  for (int qq = 0; qq < 32; ++qq) {
    int64_t s2 = gw * 32 + qq;
    if (s2 >= nq) break;
    int64_t row = order ? (int64_t)order[s2] : s2;
    for (int j = lane; j < k; j += 32) {
      double d2 = keys[j * 32 + qq];
      int32_t id = ids[j * 32 + qq];
      dist[row * k + j] = sqrt(d2);
      idx[row * k + j] = id < 0 ? -2 : (int64_t)id;
    }
  }
}

template <int D, bool PER>
__global__ void __launch_bounds__(128) k_knn_rows(TreeView tv, const double* __restrict__ Q,
                                                  const int32_t* __restrict__ order, int64_t nq,
                                                  int k, int sorted, int32_t* __restrict__ gstack,
                                                  int stack_len, double* __restrict__ dist,
                                                  int64_t* __restrict__ idx) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t gw = (int64_t)blockIdx.x * nw + w;
  int32_t* stk = gstack + gw * stack_len;
  int64_t slot = gw * 32 + lane;
  bool valid = slot < nq;
  int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
#pragma unroll
  for (int j = 0; j < D; ++j) q[j] = valid ? Q[qi * D + j] : 0.0;
  double dummy_k[1];
  int64_t dummy_i[1];
  RowHeap h{valid ? dist + qi * k : dummy_k, valid ? idx + qi * k : dummy_i};
  int kk = valid ? k : 1;
  for (int s = 0; s < kk; ++s) h.set(s, CKD_HUGE, -1);
  knn_walk<D, PER>(tv, q, valid, h, kk, stk, lane);
  if (!valid) return;
  if (sorted) heap_sort(h, k);
  for (int s = 0; s < k; ++s) {
    double d2 = h.k(s);
    int64_t id = h.i(s);
    h.set(s, sqrt(d2), id < 0 ? -2 : id);
  }
}

// ====================================================== FP32-screened search
// Same traversal and result as k_knn_smem, with two changes that cut the
// instruction count per query:
//  * leaves are screened in FP32 on leaf-relative coordinates: a point's FP32
//    lower bound of its FP64 squared distance is compared with the current k-th
//    (rounded up); only points that can still enter are evaluated in FP64 with
//    the reference arithmetic and ranked exactly by (d2, id);
//  * inserts are deferred per 32-point chunk (candidate bitmask first), and the
//    heap keys are the FP64 bit patterns compared as uint64, siblings adjacent
//    (1-based heap) so one 16-byte shared load reads both children.
// Node pruning uses the outward-rounded FP32 boxes minus a rounding slack.

constexpr float kTwoM21 = 4.76837158203125e-07f;  // 2^-21
constexpr float kShrink = 0.99999905f;             // 1 - 2^-20

// heap stride per lane (in slots): >= k + 1 and == 2 mod 16, so the 8 lanes of a
// 16-byte shared-memory phase hit distinct banks for the same slot
__host__ __device__ inline int heap_stride(int k) {
  int s = k + 1;
  return s + ((2 - s) % 16 + 16) % 16;
}

template <int D, bool PER>
struct QueryScreen {
  float q32[D];
  float dlt[D];  // node-gap slack 2^-21 (|q| + B)
};

template <int D, bool PER>
__device__ __forceinline__ float node_mind_lb(const TreeView& tv, const QueryScreen<D, PER>& qs,
                                              int32_t node) {
  const float* b = tv.box32 + (int64_t)node * 2 * D;
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    float2 lh = __ldg(reinterpret_cast<const float2*>(b) + j);
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

template <int D, bool PER>
__global__ void __launch_bounds__(128) k_knn_screen(TreeView tv, const double* __restrict__ Q,
                                                    const int32_t* __restrict__ order, int64_t nq,
                                                    int k, int sorted, int32_t* __restrict__ gstack,
                                                    int stack_len, double* __restrict__ dist,
                                                    int64_t* __restrict__ idx,
                                                    unsigned long long* __restrict__ stats) {
  constexpr int NV = (D + 3) / 4;
  // traversal statistics (only when `stats` is given): pops, needed pops, leaf
  // visits, points screened, warp phase-2 rounds, FP64 evaluations, inserts,
  // lanes active on leaf visits
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int KS = heap_stride(k);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem) + (size_t)w * 32 * KS;
  int32_t* ids = reinterpret_cast<int32_t*>(reinterpret_cast<unsigned long long*>(smem) +
                                            (size_t)nw * 32 * KS) +
                 (size_t)w * 32 * KS;
  int64_t gw = (int64_t)blockIdx.x * nw + w;
  int32_t* stk = gstack ? gstack + gw * stack_len
                        : reinterpret_cast<int32_t*>(reinterpret_cast<int32_t*>(
                              reinterpret_cast<unsigned long long*>(smem) + (size_t)nw * 32 * KS) +
                                                     (size_t)nw * 32 * KS) +
                              (size_t)w * kStack;
  int64_t slot = gw * 32 + lane;
  const bool valid = slot < nq;
  const int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
  QueryScreen<D, PER> qs;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    q[j] = valid ? Q[qi * D + j] : 0.0;
    qs.q32[j] = __double2float_rn(q[j]);
    qs.dlt[j] = kTwoM21 * (fabsf(qs.q32[j]) + tv.slack[j]) * 1.0001f;
  }
  unsigned long long* hk = keys + lane * KS;  // 1-based: slots 1..k
  int32_t* hi = ids + lane * KS;
  const unsigned long long kHugeKey = (unsigned long long)__double_as_longlong(CKD_HUGE);
  for (int s = 1; s <= k; ++s) {
    hk[s] = kHugeKey;
    hi[s] = -1;
  }
  unsigned long long wkey = kHugeKey;
  int32_t wid = -1;
  float wd32 = valid ? FLT_MAX : -1.0f;

  int top = 0;
  if (lane == 0) stk[0] = 0;
  __syncwarp();
  while (top >= 0) {
    int32_t node = stk[top];
    --top;
    __syncwarp();
    NodeMeta m = load_meta(tv.meta, node);
    bool need = node_mind_lb<D, PER>(tv, qs, node) <= wd32;
    unsigned nm = __ballot_sync(0xffffffffu, need);
    if (stats) st[0] += 1;
    if (nm == 0) continue;
    if (stats) st[1] += 1;
    if (m.left >= 0) {
      float qa = 0.0f;
#pragma unroll
      for (int j = 0; j < D; ++j)
        if (j == m.axis) qa = qs.q32[j];
      unsigned lv = __ballot_sync(0xffffffffu, need && (double)qa < m.split);
      bool left_first = 2 * __popc(lv) >= __popc(nm);
      if (lane == 0) {
        stk[top + 1] = left_first ? m.left + 1 : m.left;
        stk[top + 2] = left_first ? m.left : m.left + 1;
      }
      top += 2;
      __syncwarp();
      continue;
    }
    // ---- leaf: frame (query relative to the leaf centre) and error bounds
    if (stats) {
      st[2] += 1;
      st[3] += m.count;
      st[7] += __popc(nm);
    }
    float qr[D], e[D];
    {
      const double* b = tv.box + (int64_t)node * 2 * D;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        double lo = __ldg(&b[2 * j]), hh = __ldg(&b[2 * j + 1]);
        double c = leaf_centre(lo, hh);
        double r = fmax(c - lo, hh - c);
        double x = q[j] - c;
        if (PER) {
          double h = 0.5 * tv.L[j];
          if (x > h) x -= tv.L[j];
          else if (x < -h) x += tv.L[j];
        }
        qr[j] = __double2float_rn(x);
        e[j] = kTwoM21 * (float)(r + fabs(x) + (PER ? tv.L[j] : 0.0)) * 1.0001f + 1e-37f;
      }
    }
    for (int base = 0; base < m.count; base += 32) {
      const int cnt = min(32, m.count - base);
      const int32_t p0 = m.start + base;
      unsigned mask = 0;
      for (int i = 0; i < cnt; ++i) {
        float v[4 * NV];
#pragma unroll
        for (int h = 0; h < NV; ++h) {
          float4 f = __ldg(&tv.pts32[(int64_t)(p0 + i) * NV + h]);
          v[4 * h] = f.x;
          v[4 * h + 1] = f.y;
          v[4 * h + 2] = f.z;
          v[4 * h + 3] = f.w;
        }
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          float a = fabsf(v[j] - qr[j]);
          if (PER) a = fminf(a, (float)tv.L[j] - a);
          a = fmaxf(a - e[j], 0.0f);
          s = fmaf(a, a, s);
        }
        if (s * kShrink <= wd32) mask |= 1u << i;
      }
      if (!need) mask = 0;
      if (stats) {
        st[4] += __reduce_max_sync(0xffffffffu, (unsigned)__popc(mask));
        st[5] += __popc(mask);
      }
      while (mask) {
        int i = __ffs(mask) - 1;
        mask &= mask - 1;
        int32_t p = p0 + i;
        double d2 = point_d2<D, PER>(tv, q, p);
        unsigned long long key = (unsigned long long)__double_as_longlong(d2);
        if (key > wkey) continue;
        int32_t id = __ldg(&tv.ids[p]);
        if (key == wkey && id >= wid) continue;
        // replace the root (slot 1) and sift down
        if (stats) st[6] += 1;
        int s = 1;
        for (;;) {
          int l = 2 * s;
          if (l > k) break;
          unsigned long long kc;
          int32_t ic;
          int c;
          if (l < k) {
            ulonglong2 kk = *reinterpret_cast<const ulonglong2*>(hk + l);
            int2 ii = *reinterpret_cast<const int2*>(hi + l);
            bool right = kk.x < kk.y || (kk.x == kk.y && ii.x < ii.y);
            kc = right ? kk.y : kk.x;
            ic = right ? ii.y : ii.x;
            c = right ? l + 1 : l;
          } else {
            kc = hk[l];
            ic = hi[l];
            c = l;
          }
          if (!(key < kc || (key == kc && id < ic))) break;
          hk[s] = kc;
          hi[s] = ic;
          s = c;
        }
        hk[s] = key;
        hi[s] = id;
        wkey = hk[1];
        wid = hi[1];
        wd32 = __double2float_ru(__longlong_as_double((long long)wkey));
      }
    }
  }
  if (stats) {
    // pops, needed, leaves, points and rounds are warp-uniform: count them once
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = st[c];
      if (c == 5 || c == 6) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      }
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
  // ---- ascending (d2, id) by heap sort, then a coalesced write-out
  if (sorted) {
    for (int end = k; end > 1; --end) {
      unsigned long long key = hk[end];
      int32_t id = hi[end];
      hk[end] = hk[1];
      hi[end] = hi[1];
      int s = 1;
      for (;;) {
        int l = 2 * s;
        if (l >= end) break;
        int c = l;
        unsigned long long kc = hk[l];
        int32_t ic = hi[l];
        if (l + 1 < end) {
          unsigned long long kr = hk[l + 1];
          int32_t ir = hi[l + 1];
          if (kc < kr || (kc == kr && ic < ir)) {
            c = l + 1;
            kc = kr;
            ic = ir;
          }
        }
        if (!(key < kc || (key == kc && id < ic))) break;
        hk[s] = kc;
        hi[s] = ic;
        s = c;
      }
      hk[s] = key;
      hi[s] = id;
    }
  }
  __syncwarp();
  for (int qq = 0; qq < 32; ++qq) {
    int64_t s2 = gw * 32 + qq;
    if (s2 >= nq) break;
    int64_t row = order ? (int64_t)order[s2] : s2;
    const unsigned long long* rk = keys + qq * KS + 1;
    const int32_t* ri = ids + qq * KS + 1;
    for (int j = lane; j < k; j += 32) {
      int32_t id = ri[j];
      dist[row * k + j] = sqrt(__longlong_as_double((long long)rk[j]));
      idx[row * k + j] = id < 0 ? -2 : (int64_t)id;
    }
  }
}

// ================================================= per-lane traversal variant
// Each lane walks the tree for its own query: both children's FP32 boxes are
// tested when a node is expanded, the nearer child is taken and the other pushed
// with its bound on a per-lane stack (registers / local memory), so entries that
// the shrinking k-th distance has pruned are dropped without reloading a node.
// Lanes descend until they reach a leaf, then scan leaves together
// (while-while structure), with the same FP32 screen, FP64 recheck and heap as
// k_knn_screen.
//
// BOUNDED: every query starts with its heap full of k sentinels (key r2[q],
// id INT32_MAX) instead of HUGE, so pruning starts at the root.  A point is
// accepted iff (d2, id) < the current worst, so every point with d2 <= r2[q] is
// still seen; when no sentinel is left the heap holds the exact k nearest.  A
// query that ends with a sentinel (fewer than k points within the bound) is
// appended to miss[] for the unbounded rerun and its output row is not written.
constexpr int kLaneStack = 128;

template <int D, bool PER, bool BOUNDED = false>
__global__ void __launch_bounds__(128) k_knn_lane(TreeView tv, const double* __restrict__ Q,
                                                  const int32_t* __restrict__ order, int64_t nq,
                                                  int k, int sorted, double* __restrict__ dist,
                                                  int64_t* __restrict__ idx,
                                                  unsigned long long* __restrict__ stats,
                                                  const double* __restrict__ r2 = nullptr,
                                                  int32_t* __restrict__ miss = nullptr,
                                                  unsigned* __restrict__ nmiss = nullptr,
                                                  const int32_t* __restrict__ qleaf = nullptr,
                                                  const int32_t* __restrict__ qroot = nullptr) {
  constexpr int NV = (D + 3) / 4;
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int KS = heap_stride(k);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem) + (size_t)w * 32 * KS;
  int32_t* ids = reinterpret_cast<int32_t*>(reinterpret_cast<unsigned long long*>(smem) +
                                            (size_t)nw * 32 * KS) +
                 (size_t)w * 32 * KS;
  int64_t gw = (int64_t)blockIdx.x * nw + w;
  int64_t slot = gw * 32 + lane;
  const bool valid = slot < nq;
  const int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
  QueryScreen<D, PER> qs;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    q[j] = valid ? Q[qi * D + j] : 0.0;
    qs.q32[j] = __double2float_rn(q[j]);
    qs.dlt[j] = kTwoM21 * (fabsf(qs.q32[j]) + tv.slack[j]) * 1.0001f;
  }
  unsigned long long* hk = keys + lane * KS;
  int32_t* hi = ids + lane * KS;
  const unsigned long long kHugeKey = (unsigned long long)__double_as_longlong(CKD_HUGE);
  unsigned long long skey = kHugeKey;
  int32_t sid = -1;
  float wd32 = FLT_MAX;
  if (BOUNDED && valid) {
    const double rr = r2[qi];
    if (rr < CKD_HUGE) {
      skey = (unsigned long long)__double_as_longlong(rr);
      sid = 0x7fffffff;
      wd32 = __double2float_ru(rr);
    }
  }
  for (int s = 1; s <= k; ++s) {
    hk[s] = skey;
    hi[s] = sid;
  }
  unsigned long long wkey = skey;
  int32_t wid = sid;

  int32_t sn[kLaneStack];
  float sd[kLaneStack];
  int top = 0;
  // a forest query starts at its own tree's root
  int32_t node = valid ? (qroot ? qroot[qi] : 0) : -1;
  if (BOUNDED && valid && qleaf && sid == 0x7fffffff) {
    // Start at the lowest ancestor of the query's leaf whose cell strictly
    // contains the cube [q - r, q + r]^D: every point within the bound lies
    // strictly inside that cell, hence in its subtree (and, periodic, is its own
    // minimum image).  Inward-rounded FP32 cells and outward-rounded tests keep
    // this conservative.
    const float r32 = __fsqrt_ru(wd32);
    int32_t a = qleaf[qi];
    while (a >= 0) {
      const float* c = tv.cell32 + (int64_t)a * 2 * D;
      bool inside = true;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        const float2 lh = __ldg(reinterpret_cast<const float2*>(c) + j);
        inside = inside && __fsub_rd(__fsub_rd(qs.q32[j], r32), qs.dlt[j]) > lh.x &&
                 __fadd_ru(__fadd_ru(qs.q32[j], r32), qs.dlt[j]) < lh.y;
      }
      if (inside) break;
      a = load_meta(tv.meta, a).parent;
    }
    node = a < 0 ? node : a;
  }
  while (node >= 0) {
    // ---- descend to a leaf, nearer child first
    NodeMeta m = load_meta(tv.meta, node);
    while (node >= 0 && m.left >= 0) {
      if (stats) st[0] += 1;
      float ml = node_mind_lb<D, PER>(tv, qs, m.left);
      float mr = node_mind_lb<D, PER>(tv, qs, m.left + 1);
      bool nl = ml <= wd32, nr = mr <= wd32;
      if (nl && nr) {
        bool lf = ml <= mr;
        sn[top] = lf ? m.left + 1 : m.left;
        sd[top] = lf ? mr : ml;
        ++top;
        node = lf ? m.left : m.left + 1;
      } else if (nl || nr) {
        node = nl ? m.left : m.left + 1;
      } else {
        node = -1;
        while (top > 0) {
          --top;
          if (sd[top] <= wd32) {
            node = sn[top];
            break;
          }
        }
      }
      if (node >= 0) m = load_meta(tv.meta, node);
    }
    if (node < 0) break;
    // ---- scan the leaf
    if (stats) {
      st[2] += 1;
      st[3] += m.count;
    }
    float qr[D], e[D];
    {
      const double* b = tv.box + (int64_t)node * 2 * D;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        double lo = __ldg(&b[2 * j]), hh = __ldg(&b[2 * j + 1]);
        double c = leaf_centre(lo, hh);
        double r = fmax(c - lo, hh - c);
        double x = q[j] - c;
        if (PER) {
          double h = 0.5 * tv.L[j];
          if (x > h) x -= tv.L[j];
          else if (x < -h) x += tv.L[j];
        }
        qr[j] = __double2float_rn(x);
        e[j] = kTwoM21 * (float)(r + fabs(x) + (PER ? tv.L[j] : 0.0)) * 1.0001f + 1e-37f;
      }
    }
    for (int base = 0; base < m.count; base += 32) {
      const int cnt = min(32, m.count - base);
      const int32_t p0 = m.start + base;
      unsigned mask = 0;
      for (int i = 0; i < cnt; ++i) {
        float v[4 * NV];
#pragma unroll
        for (int h = 0; h < NV; ++h) {
          float4 f = __ldg(&tv.pts32[(int64_t)(p0 + i) * NV + h]);
          v[4 * h] = f.x;
          v[4 * h + 1] = f.y;
          v[4 * h + 2] = f.z;
          v[4 * h + 3] = f.w;
        }
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          float a = fabsf(v[j] - qr[j]);
          if (PER) a = fminf(a, (float)tv.L[j] - a);
          a = fmaxf(a - e[j], 0.0f);
          s = fmaf(a, a, s);
        }
        if (s * kShrink <= wd32) mask |= 1u << i;
      }
      if (stats) st[5] += __popc(mask);
      while (mask) {
        int i = __ffs(mask) - 1;
        mask &= mask - 1;
        int32_t p = p0 + i;
        double d2 = point_d2<D, PER>(tv, q, p);
        unsigned long long key = (unsigned long long)__double_as_longlong(d2);
        if (key > wkey) continue;
        int32_t id = __ldg(&tv.ids[p]);
        if (key == wkey && id >= wid) continue;
        if (stats) st[6] += 1;
        int s = 1;
        for (;;) {
          int l = 2 * s;
          if (l > k) break;
          unsigned long long kc;
          int32_t ic;
          int c;
          if (l < k) {
            ulonglong2 kk = *reinterpret_cast<const ulonglong2*>(hk + l);
            int2 ii = *reinterpret_cast<const int2*>(hi + l);
            bool right = kk.x < kk.y || (kk.x == kk.y && ii.x < ii.y);
            kc = right ? kk.y : kk.x;
            ic = right ? ii.y : ii.x;
            c = right ? l + 1 : l;
          } else {
            kc = hk[l];
            ic = hi[l];
            c = l;
          }
          if (!(key < kc || (key == kc && id < ic))) break;
          hk[s] = kc;
          hi[s] = ic;
          s = c;
        }
        hk[s] = key;
        hi[s] = id;
        wkey = hk[1];
        wid = hi[1];
        wd32 = __double2float_ru(__longlong_as_double((long long)wkey));
      }
    }
    // ---- next: pop the nearest pending subtree still within reach
    node = -1;
    while (top > 0) {
      --top;
      if (sd[top] <= wd32) {
        node = sn[top];
        break;
      }
    }
  }
  if (stats) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = st[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
  const bool missed = BOUNDED && valid && wid == 0x7fffffff;
  unsigned missmask = 0;
  if (BOUNDED) {
    missmask = __ballot_sync(0xffffffffu, missed);
    if (missmask) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(nmiss, (unsigned)__popc(missmask));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (missed) miss[base + __popc(missmask & ((1u << lane) - 1u))] = (int32_t)qi;
    }
  }
  if (sorted && valid && !missed) {
    for (int end = k; end > 1; --end) {
      unsigned long long key = hk[end];
      int32_t id = hi[end];
      hk[end] = hk[1];
      hi[end] = hi[1];
      int s = 1;
      for (;;) {
        int l = 2 * s;
        if (l >= end) break;
        int c = l;
        unsigned long long kc = hk[l];
        int32_t ic = hi[l];
        if (l + 1 < end) {
          unsigned long long kr = hk[l + 1];
          int32_t ir = hi[l + 1];
          if (kc < kr || (kc == kr && ic < ir)) {
            c = l + 1;
            kc = kr;
            ic = ir;
          }
        }
        if (!(key < kc || (key == kc && id < ic))) break;
        hk[s] = kc;
        hi[s] = ic;
        s = c;
      }
      hk[s] = key;
      hi[s] = id;
    }
  }
  __syncwarp();
  for (int qq = 0; qq < 32; ++qq) {
    int64_t s2 = gw * 32 + qq;
    if (s2 >= nq) break;
    if (BOUNDED && ((missmask >> qq) & 1u)) continue;
    int64_t row = order ? (int64_t)order[s2] : s2;
    const unsigned long long* rk = keys + qq * KS + 1;
    const int32_t* ri = ids + qq * KS + 1;
    for (int j = lane; j < k; j += 32) {
      int32_t id = ri[j];
      dist[row * k + j] = sqrt(__longlong_as_double((long long)rk[j]));
      idx[row * k + j] = id < 0 ? -2 : (int64_t)id;
    }
  }
}

// ============================================ per-lane traversal, compact heap
// Same search as k_knn_lane with a heap half the size: each entry is the FP32
// rounding of its FP64 squared distance (round to nearest is monotone, so
// a < b in FP32 implies a < b exactly) and the point's leaf-ordered position.
// Ties in FP32 are resolved exactly by recomputing the FP64 distances from the
// positions and then comparing ids; the FP64 distances of the results are
// recomputed once for the output.  8 bytes per entry instead of 12 lets 1.5x
// more warps stay resident; heap comparisons are 32-bit.  Sentinels: position -1
// = (HUGE, id -1), position -2 = (r2, INT32_MAX) for the bounded search.
// shared memory of the compact per-lane kernel per warp: k heap slots (1-based) x 32 lanes
__host__ __device__ inline size_t compact_heap_bytes(int k) { return (size_t)(k + 1) * 32 * 8; }

constexpr int32_t kPosMissing = -1;
constexpr int32_t kPosBound = -2;

template <int D, bool PER>
struct CompactCtx {
  const TreeView& tv;
  const double (&q)[D];
  double rr;  // bounded sentinel's squared distance
  __device__ __forceinline__ double exact(int32_t p) const {
    return p >= 0 ? point_d2_rec<D, PER>(tv, q, p) : (p == kPosMissing ? CKD_HUGE : rr);
  }
  __device__ __forceinline__ int32_t id(int32_t p) const {
    return p >= 0 ? __ldg(&tv.ids[p]) : (p == kPosMissing ? -1 : 0x7fffffff);
  }
  // exact (d2, id) order of two entries whose FP32 keys are equal
  __device__ __forceinline__ bool tie_before(int32_t a, int32_t b) const {
    const double da = exact(a), db = exact(b);
    if (da != db) return da < db;
    return id(a) < id(b);
  }
};

template <int D, bool PER, bool BOUNDED = false, bool PAIR = false>
__global__ void __launch_bounds__(128, 6) k_knn_lane2(TreeView tv, const double* __restrict__ Q,
                                                   const int32_t* __restrict__ order, int64_t nq,
                                                   int k, int sorted, double* __restrict__ dist,
                                                   int64_t* __restrict__ idx,
                                                   unsigned long long* __restrict__ stats,
                                                   const double* __restrict__ r2 = nullptr,
                                                   int32_t* __restrict__ miss = nullptr,
                                                   unsigned* __restrict__ nmiss = nullptr,
                                                   const int32_t* __restrict__ qleaf = nullptr,
                                                   const int32_t* __restrict__ qroot = nullptr) {
  constexpr int NV = (D + 3) / 4;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // heap slot s of this lane at H[s * 32 + lane]: (key bits, position); keys are
  // non-negative floats, so their bit patterns order as unsigned integers, and
  // every lane always addresses its own bank pair (no conflicts between lanes
  // at different heap levels)
  uint2* H = reinterpret_cast<uint2*>(smem) + (size_t)w * 32 * (k + 1) + lane;
  const int64_t gw = (int64_t)blockIdx.x * nw + w;
  const int64_t slot = gw * 32 + lane;
  const bool valid = slot < nq;
  const int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
  QueryScreen<D, PER> qs;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    q[j] = valid ? Q[qi * D + j] : 0.0;
    qs.q32[j] = __double2float_rn(q[j]);
    qs.dlt[j] = kTwoM21 * (fabsf(qs.q32[j]) + tv.slack[j]) * 1.0001f;
  }
  float skey = FLT_MAX;
  int32_t spos = kPosMissing;
  float wd32 = FLT_MAX;
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
  const CompactCtx<D, PER> cx{tv, q, rr};
  for (int s = 1; s <= k; ++s) H[s * 32] = make_uint2(__float_as_uint(skey), (unsigned)spos);
  unsigned wk = __float_as_uint(skey);  // root key bits
  int32_t wp = spos;                    // root position

  int32_t sn[kLaneStack];
  float sd[kLaneStack];
  int top = 0;
  int32_t node = valid ? (qroot ? qroot[qi] : 0) : -1;
  if (BOUNDED && valid && qleaf && spos == kPosBound) {
    // start at the lowest ancestor whose cell strictly contains [q - r, q + r]^D
    const float r32 = __fsqrt_ru(wd32);
    int32_t a = qleaf[qi];
    while (a >= 0) {
      const float* c = tv.cell32 + (int64_t)a * 2 * D;
      bool inside = true;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        const float2 lh = __ldg(reinterpret_cast<const float2*>(c) + j);
        inside = inside && __fsub_rd(__fsub_rd(qs.q32[j], r32), qs.dlt[j]) > lh.x &&
                 __fadd_ru(__fadd_ru(qs.q32[j], r32), qs.dlt[j]) < lh.y;
      }
      if (inside) break;
      a = load_meta(tv.meta, a).parent;
    }
    node = a < 0 ? node : a;
  }
  // PAIR: stack entries and `node` carry the leaf flag (a leaf is stored as ~id,
  // < -1 because children ids are >= 1; -1 means "no node") and internal nodes are
  // expanded from their child-pair record alone (both children's FP32 boxes, ids
  // and leaf flags), one dependent load per level.  Otherwise the node's meta is
  // read first, then both children's FP32 boxes.
  constexpr int PF = pair_f4(D);
  bool is_leaf = node >= 0 && PAIR && load_meta(tv.meta, node).left < 0;
  NodeMeta m;
  while (node >= 0) {
    // ---- descend to a leaf, nearer child first
    if (!PAIR) {
      m = load_meta(tv.meta, node);
      while (node >= 0 && m.left >= 0) {
        if (stats) st[0] += 1;
        const float ml = node_mind_lb<D, PER>(tv, qs, m.left);
        const float mr = node_mind_lb<D, PER>(tv, qs, m.left + 1);
        const bool nl = ml <= wd32, nr = mr <= wd32;
        if (nl && nr) {
          const bool lf = ml <= mr;
          sn[top] = lf ? m.left + 1 : m.left;
          sd[top] = lf ? mr : ml;
          ++top;
          node = lf ? m.left : m.left + 1;
        } else if (nl || nr) {
          node = nl ? m.left : m.left + 1;
        } else {
          node = -1;
          while (top > 0) {
            --top;
            if (sd[top] <= wd32) {
              node = sn[top];
              break;
            }
          }
        }
        if (node >= 0) m = load_meta(tv.meta, node);
      }
      if (node < 0) break;
    } else {
      while (!is_leaf) {
        if (stats) st[0] += 1;
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
        const float ml = box_mind_lb<D, PER>(tv, qs, lo_l, hi_l);
        const float mr = box_mind_lb<D, PER>(tv, qs, lo_r, hi_r);
        const bool nl = ml <= wd32, nr = mr <= wd32;
        const int32_t el = info.z ? ~info.x : info.x, er = info.w ? ~info.y : info.y;
        int32_t nxt = -1;
        if (nl && nr) {
          const bool lf = ml <= mr;
          sn[top] = lf ? er : el;
          sd[top] = lf ? mr : ml;
          ++top;
          nxt = lf ? el : er;
        } else if (nl || nr) {
          nxt = nl ? el : er;
        } else {
          while (top > 0) {
            --top;
            if (sd[top] <= wd32) {
              nxt = sn[top];
              break;
            }
          }
          if (nxt == -1) break;
        }
        is_leaf = nxt < 0;
        node = is_leaf ? ~nxt : nxt;
      }
      if (!is_leaf) break;
      m = load_meta(tv.meta, node);
    }

    // ---- scan the leaf
    if (stats) {
      st[2] += 1;
      st[3] += m.count;
    }
    float qr[D], e[D];
    // near: on every axis the whole leaf lies within half a box side of the
    // query's image, so the minimum image of each point difference is the
    // direct difference and the screen skips the wrap (exactly: every |v - qr|
    // stays below L/2 even after rounding)
    bool near = true;
    {
      const double* b = tv.box + (int64_t)node * 2 * D;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        double lo = __ldg(&b[2 * j]), hh = __ldg(&b[2 * j + 1]);
        double c = leaf_centre(lo, hh);
        double r = fmax(c - lo, hh - c);
        double x = q[j] - c;
        if (PER) {
          double h = 0.5 * tv.L[j];
          if (x > h) x -= tv.L[j];
          else if (x < -h) x += tv.L[j];
          near = near && fabs(x) + r < 0.49 * tv.L[j];
        }
        qr[j] = __double2float_rn(x);
        e[j] = kTwoM21 * (float)(r + fabs(x) + (PER ? tv.L[j] : 0.0)) * 1.0001f + 1e-37f;
      }
    }
    for (int base = 0; base < m.count; base += 32) {
      const int cnt = min(32, m.count - base);
      const int32_t p0 = m.start + base;
      unsigned mask = 0;
      if (!PER || near) {
        for (int i = 0; i < cnt; ++i) {
          float v[4 * NV];
#pragma unroll
          for (int h = 0; h < NV; ++h) {
            float4 f = __ldg(&tv.pts32[(int64_t)(p0 + i) * NV + h]);
            v[4 * h] = f.x;
            v[4 * h + 1] = f.y;
            v[4 * h + 2] = f.z;
            v[4 * h + 3] = f.w;
          }
          float s = 0.0f;
#pragma unroll
          for (int j = 0; j < D; ++j) {
            float a = fmaxf(fabsf(v[j] - qr[j]) - e[j], 0.0f);
            s = fmaf(a, a, s);
          }
          if (s * kShrink <= wd32) mask |= 1u << i;
        }
      } else {
        for (int i = 0; i < cnt; ++i) {
          float v[4 * NV];
#pragma unroll
          for (int h = 0; h < NV; ++h) {
            float4 f = __ldg(&tv.pts32[(int64_t)(p0 + i) * NV + h]);
            v[4 * h] = f.x;
            v[4 * h + 1] = f.y;
            v[4 * h + 2] = f.z;
            v[4 * h + 3] = f.w;
          }
          float s = 0.0f;
#pragma unroll
          for (int j = 0; j < D; ++j) {
            float a = fabsf(v[j] - qr[j]);
            a = fminf(a, (float)tv.L[j] - a);
            a = fmaxf(a - e[j], 0.0f);
            s = fmaf(a, a, s);
          }
          if (s * kShrink <= wd32) mask |= 1u << i;
        }
      }
      if (stats) st[5] += __popc(mask);
      while (mask) {
        const int i = __ffs(mask) - 1;
        mask &= mask - 1;
        const int32_t p = p0 + i;
        const double d2 = point_d2_rec<D, PER>(tv, q, p);
        const unsigned kc = __float_as_uint(__double2float_rn(d2));
        if (kc > wk) continue;
        if (kc == wk) {  // FP32 tie with the root: exact comparison
          const double dr = cx.exact(wp);
          if (d2 > dr) continue;
          if (d2 == dr && __ldg(&tv.ids[p]) >= cx.id(wp)) continue;
        }
        if (stats) st[6] += 1;
        // replace the root, sift down
        int s = 1;
        for (;;) {
          const int l = 2 * s;
          if (l > k) break;
          uint2 ch = H[l * 32];
          int c = l;
          if (l < k) {
            const uint2 r = H[(l + 1) * 32];
            if (ch.x < r.x || (ch.x == r.x && cx.tie_before((int32_t)ch.y, (int32_t)r.y))) {
              ch = r;
              c = l + 1;
            }
          }
          const unsigned kch = ch.x;
          const int32_t pch = (int32_t)ch.y;
          // the candidate stays above the child iff it ranks after it
          bool cand_before = kc < kch;
          if (kc == kch) {
            const double dch = cx.exact(pch);
            cand_before = d2 < dch || (d2 == dch && __ldg(&tv.ids[p]) < cx.id(pch));
          }
          if (!cand_before) break;
          H[s * 32] = ch;
          s = c;
        }
        H[s * 32] = make_uint2(kc, (unsigned)p);
        const uint2 root = H[32];
        wk = root.x;
        wp = (int32_t)root.y;
        wd32 = __uint_as_float(wk + 1u);
      }
    }
    // ---- next: pop the nearest pending subtree still within reach
    int32_t nxt = -1;
    while (top > 0) {
      --top;
      if (sd[top] <= wd32) {
        nxt = sn[top];
        break;
      }
    }
    if (nxt == -1) break;
    if (PAIR) {
      is_leaf = nxt < 0;
      node = is_leaf ? ~nxt : nxt;
    } else {
      node = nxt;
    }
  }
  if (stats) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = st[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
  const bool missed = BOUNDED && valid && wp == kPosBound;
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
  if (sorted && valid && !missed) {
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
          if (ch.x < r.x || (ch.x == r.x && cx.tie_before((int32_t)ch.y, (int32_t)r.y))) {
            c = l + 1;
            ch = r;
          }
        }
        if (!(e.x < ch.x || (e.x == ch.x && cx.tie_before((int32_t)e.y, (int32_t)ch.y)))) break;
        H[s * 32] = ch;
        s = c;
      }
      H[s * 32] = e;
    }
  }
  __syncwarp();
  // warp-cooperative write-out: exact FP64 distances recomputed from positions
  for (int qq = 0; qq < 32; ++qq) {
    const int64_t s2 = gw * 32 + qq;
    if (s2 >= nq) break;
    double qx[D];
#pragma unroll
    for (int j = 0; j < D; ++j) qx[j] = __shfl_sync(FULL, q[j], qq);
    if (BOUNDED && ((missmask >> qq) & 1u)) continue;
    const int64_t row = order ? (int64_t)order[s2] : s2;
    const uint2* rp = H - lane + qq + 32;  // query qq's slot 1
    for (int j = lane; j < k; j += 32) {
      const int32_t p = (int32_t)rp[j * 32].y;
      double d2 = CKD_HUGE;
      int64_t id = -2;
      if (p >= 0) {
        d2 = point_d2_rec<D, PER>(tv, qx, p);
        id = (int64_t)__ldg(&tv.ids[p]);
      }
      dist[row * k + j] = sqrt(d2);
      idx[row * k + j] = id;
    }
  }
}

// ===================================================== bottom-up search (v4)
// Per-lane search that starts at the query's own leaf and climbs: after a
// subtree C is exhausted, the search stops if the ball of the current k-th
// distance lies inside C's sliding-midpoint cell (cells partition the box, so no
// point outside C can be closer; under periodic wrap the ball then lies inside
// the fundamental box, so no image can be closer either); otherwise C's sibling
// subtree is explored top-down, nearer child first, pruned by FP32 boxes, and C
// moves to its parent.  Leaves are screened in FP32 and ranked exactly in FP64
// as in k_knn_screen.

struct LaneHeap {
  unsigned long long* hk;  // 1-based slots 1..k (FP64 bit patterns)
  int32_t* hi;
  int k;
  int n;  // real entries so far; below k the slots are an unordered list
  unsigned long long wkey;
  int32_t wid;
  float wd32;  // current k-th squared distance rounded up to FP32
};

// sift (key, id) down from slot s within slots 1..end
__device__ __forceinline__ void lane_sift(LaneHeap& H, int s, int end, unsigned long long key,
                                          int32_t id) {
  for (;;) {
    int l = 2 * s;
    if (l > end) break;
    unsigned long long kc;
    int32_t ic;
    int c;
    if (l < end) {
      ulonglong2 kk = *reinterpret_cast<const ulonglong2*>(H.hk + l);
      int2 ii = *reinterpret_cast<const int2*>(H.hi + l);
      bool right = kk.x < kk.y || (kk.x == kk.y && ii.x < ii.y);
      kc = right ? kk.y : kk.x;
      ic = right ? ii.y : ii.x;
      c = right ? l + 1 : l;
    } else {
      kc = H.hk[l];
      ic = H.hi[l];
      c = l;
    }
    if (!(key < kc || (key == kc && id < ic))) break;
    H.hk[s] = kc;
    H.hi[s] = ic;
    s = c;
  }
  H.hk[s] = key;
  H.hi[s] = id;
}

__device__ __forceinline__ void lane_heapify(LaneHeap& H, int end) {
  for (int s = end / 2; s >= 1; --s) lane_sift(H, s, end, H.hk[s], H.hi[s]);
}

// A candidate that ranks before the current k-th.  While fewer than k entries
// are held it is appended (the k-th is still the HUGE(0.0) sentinel); the k-th
// append heapifies once, later candidates replace the root and sift down.
__device__ __forceinline__ void lane_heap_insert(LaneHeap& H, unsigned long long key, int32_t id) {
  if (H.n < H.k) {
    ++H.n;
    H.hk[H.n] = key;
    H.hi[H.n] = id;
    if (H.n < H.k) return;
    lane_heapify(H, H.k);
  } else {
    lane_sift(H, 1, H.k, key, id);
  }
  H.wkey = H.hk[1];
  H.wid = H.hi[1];
  H.wd32 = __double2float_ru(__longlong_as_double((long long)H.wkey));
}

// pad with (HUGE(0.0), -1) sentinels when fewer than k points were found
__device__ __forceinline__ void lane_heap_finish(LaneHeap& H) {
  if (H.n == H.k) return;
  const unsigned long long kHugeKey = (unsigned long long)__double_as_longlong(CKD_HUGE);
  for (int s = H.n + 1; s <= H.k; ++s) {
    H.hk[s] = kHugeKey;
    H.hi[s] = -1;
  }
  H.n = H.k;
  lane_heapify(H, H.k);
}

__device__ __forceinline__ void lane_heap_sort(LaneHeap& H) {
  for (int end = H.k; end > 1; --end) {
    unsigned long long key = H.hk[end];
    int32_t id = H.hi[end];
    H.hk[end] = H.hk[1];
    H.hi[end] = H.hi[1];
    lane_sift(H, 1, end - 1, key, id);
  }
}

// FP32 lower bound of a child box gap from a child-pair record side
template <int D, bool PER>
__device__ __forceinline__ float rec_mind_lb(const TreeView& tv, const QueryScreen<D, PER>& qs,
                                             const float (&lo)[4 * ((D + 3) / 4)],
                                             const float (&hi)[4 * ((D + 3) / 4)]) {
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

// Screen one leaf and insert the points that can enter (see k_knn_screen).
template <int D, bool PER>
__device__ __forceinline__ void lane_scan_leaf(const TreeView& tv, const double (&q)[D],
                                               int32_t node, int32_t start, int32_t count,
                                               LaneHeap& H, unsigned long long* st) {
  constexpr int NV = (D + 3) / 4;
  float qr[D], e[D];
  const float* b32 = tv.box32 + (int64_t)node * 2 * D;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double c = __ldg(&tv.centre[(int64_t)node * D + j]);
    float2 lh = __ldg(reinterpret_cast<const float2*>(b32) + j);
    double r = fmax(c - (double)lh.x, (double)lh.y - c);  // >= |p - c| for every point
    double x = q[j] - c;
    double wrap = 0.0;
    if (PER) {
      double h = 0.5 * tv.L[j];
      if (x > h) x -= tv.L[j];
      else if (x < -h) x += tv.L[j];
      if (r + fabs(x) > 0.45 * tv.L[j]) wrap = tv.L[j];  // minimum image may wrap
    }
    qr[j] = __double2float_rn(x);
    e[j] = kTwoM21 * (float)(r + fabs(x) + wrap) * 1.0001f + 1e-37f;
  }
  const unsigned long long kHugeKey = (unsigned long long)__double_as_longlong(CKD_HUGE);
  for (int base = 0; base < count; base += 32) {
    const int cnt = min(32, count - base);
    const int32_t p0 = start + base;
    unsigned mask = 0;
    for (int i = 0; i < cnt; ++i) {
      float v[4 * NV];
#pragma unroll
      for (int h = 0; h < NV; ++h) {
        float4 f = __ldg(&tv.pts32[(int64_t)(p0 + i) * NV + h]);
        v[4 * h] = f.x;
        v[4 * h + 1] = f.y;
        v[4 * h + 2] = f.z;
        v[4 * h + 3] = f.w;
      }
      float s = 0.0f;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        float a = fabsf(v[j] - qr[j]);
        if (PER) a = fminf(a, (float)tv.L[j] - a);
        a = fmaxf(a - e[j], 0.0f);
        s = fmaf(a, a, s);
      }
      if (s * kShrink <= H.wd32) mask |= 1u << i;
    }
    if (st) {
      st[3] += cnt;
      st[5] += __popc(mask);
    }
    while (mask) {
      int i = __ffs(mask) - 1;
      mask &= mask - 1;
      int32_t p = p0 + i;
      double d2 = point_d2<D, PER>(tv, q, p);
      unsigned long long key = (unsigned long long)__double_as_longlong(d2);
      int32_t id;
      if (H.n < H.k) {
        if (key >= kHugeKey) continue;  // the strict test against HUGE(0.0)
        id = __ldg(&tv.ids[p]);
      } else {
        if (key > H.wkey) continue;
        id = __ldg(&tv.ids[p]);
        if (key == H.wkey && id >= H.wid) continue;
      }
      if (st) st[6] += 1;
      lane_heap_insert(H, key, id);
    }
  }
}

constexpr int kUpStack = 96;

template <int D, bool PER>
__global__ void __launch_bounds__(256) k_knn_up(TreeView tv, const double* __restrict__ Q,
                                                const int32_t* __restrict__ order,
                                                const int32_t* __restrict__ qleaf, int64_t nq,
                                                int k, int sorted, double* __restrict__ dist,
                                                int64_t* __restrict__ idx,
                                                unsigned long long* __restrict__ stats) {
  constexpr int NV = (D + 3) / 4;
  constexpr int PF = 4 * NV + 1;
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long stv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long* st = stats ? stv : nullptr;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int KS = heap_stride(k);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem) + (size_t)w * 32 * KS;
  int32_t* ids = reinterpret_cast<int32_t*>(reinterpret_cast<unsigned long long*>(smem) +
                                            (size_t)nw * 32 * KS) +
                 (size_t)w * 32 * KS;
  int64_t gw = (int64_t)blockIdx.x * nw + w;
  int64_t slot = gw * 32 + lane;
  const bool valid = slot < nq;
  const int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
  QueryScreen<D, PER> qs;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    q[j] = valid ? Q[qi * D + j] : 0.0;
    qs.q32[j] = __double2float_rn(q[j]);
    qs.dlt[j] = kTwoM21 * (fabsf(qs.q32[j]) + tv.slack[j]) * 1.0001f;
  }
  LaneHeap H;
  H.hk = keys + lane * KS;
  H.hi = ids + lane * KS;
  H.k = k;
  H.n = 0;
  H.wkey = (unsigned long long)__double_as_longlong(CKD_HUGE);
  H.wid = -1;
  H.wd32 = FLT_MAX;

  // ---- per-lane state: climb position, explore stack, pending leaf
  int32_t pending = -1, C = -1, parent = -1;
  bool done = !valid;
  if (valid) {
    int32_t leaf;
    NodeMeta lm;
    if (qleaf) {
      leaf = qleaf[qi];
      lm = load_meta(tv.meta, leaf);
    } else {
      leaf = 0;
      lm = load_meta(tv.meta, 0);
      while (lm.left >= 0) {
        double qa = 0.0;
#pragma unroll
        for (int j = 0; j < D; ++j)
          if (j == lm.axis) qa = q[j];
        leaf = qa < lm.split ? lm.left : lm.left + 1;
        lm = load_meta(tv.meta, leaf);
      }
    }
    pending = leaf;
    C = leaf;
    parent = lm.parent;
  }
  int32_t sn[kUpStack];
  float sd[kUpStack];
  int top = 0;
  for (;;) {
    // advance this lane until it holds a leaf to scan or has finished
    while (!done && pending < 0) {
      if (top > 0) {
        --top;
        if (sd[top] > H.wd32) continue;
        int32_t x = sn[top];
        if (x < 0) {
          pending = x & 0x7fffffff;
          continue;
        }
        if (st) st[0] += 1;
        const float4* r2 = tv.pair + (int64_t)x * PF;
        float llo[4 * NV], lhi[4 * NV], rlo[4 * NV], rhi[4 * NV];
#pragma unroll
        for (int h = 0; h < NV; ++h) {
          float4 a = __ldg(&r2[h]), b = __ldg(&r2[NV + h]);
          float4 c = __ldg(&r2[2 * NV + h]), d = __ldg(&r2[3 * NV + h]);
          llo[4 * h] = a.x; llo[4 * h + 1] = a.y; llo[4 * h + 2] = a.z; llo[4 * h + 3] = a.w;
          lhi[4 * h] = b.x; lhi[4 * h + 1] = b.y; lhi[4 * h + 2] = b.z; lhi[4 * h + 3] = b.w;
          rlo[4 * h] = c.x; rlo[4 * h + 1] = c.y; rlo[4 * h + 2] = c.z; rlo[4 * h + 3] = c.w;
          rhi[4 * h] = d.x; rhi[4 * h + 1] = d.y; rhi[4 * h + 2] = d.z; rhi[4 * h + 3] = d.w;
        }
        int4 xi = __ldg(reinterpret_cast<const int4*>(&r2[4 * NV]));
        float ml = rec_mind_lb<D, PER>(tv, qs, llo, lhi);
        float mr = rec_mind_lb<D, PER>(tv, qs, rlo, rhi);
        int32_t L = xi.x | (xi.z ? (int32_t)0x80000000 : 0);
        int32_t R = xi.y | (xi.w ? (int32_t)0x80000000 : 0);
        bool nl = ml <= H.wd32, nr = mr <= H.wd32;
        if (nl && nr) {  // the farther first, so the nearer is taken next
          bool lf = ml <= mr;
          sn[top] = lf ? R : L;
          sd[top] = lf ? mr : ml;
          sn[top + 1] = lf ? L : R;
          sd[top + 1] = lf ? ml : mr;
          top += 2;
        } else if (nl || nr) {
          sn[top] = nl ? L : R;
          sd[top] = nl ? ml : mr;
          top += 1;
        }
      } else {
        if (parent < 0) {
          done = true;
          continue;
        }
        // stop once the k-th-distance ball lies inside C's cell
        float r = sqrtf(H.wd32) * 1.0000003f;
        const float* c32 = tv.cell32 + (int64_t)C * 2 * D;
        bool inside = true;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          float2 cl = __ldg(reinterpret_cast<const float2*>(c32) + j);
          inside = inside && (qs.q32[j] - r - qs.dlt[j] >= cl.x) &&
                   (qs.q32[j] + r + qs.dlt[j] <= cl.y);
        }
        if (inside) {
          if (st) st[7] += 1;
          done = true;
          continue;
        }
        if (st) st[1] += 1;
        // queue the sibling of C, then climb
        const float4* rec = tv.pair + (int64_t)parent * PF;
        int4 info = __ldg(reinterpret_cast<const int4*>(&rec[4 * NV]));
        const int side = (info.x == C) ? 1 : 0;
        float lo[4 * NV], hi[4 * NV];
#pragma unroll
        for (int h = 0; h < NV; ++h) {
          float4 a = __ldg(&rec[side * 2 * NV + h]), b = __ldg(&rec[side * 2 * NV + NV + h]);
          lo[4 * h] = a.x; lo[4 * h + 1] = a.y; lo[4 * h + 2] = a.z; lo[4 * h + 3] = a.w;
          hi[4 * h] = b.x; hi[4 * h + 1] = b.y; hi[4 * h + 2] = b.z; hi[4 * h + 3] = b.w;
        }
        float ms = rec_mind_lb<D, PER>(tv, qs, lo, hi);
        if (ms <= H.wd32) {
          int32_t S = side ? info.y : info.x;
          int sleaf = side ? info.w : info.z;
          sn[0] = S | (sleaf ? (int32_t)0x80000000 : 0);
          sd[0] = ms;
          top = 1;
        }
        C = parent;
        parent = load_meta(tv.meta, C).parent;
      }
    }
    if (__all_sync(0xffffffffu, pending < 0)) break;
    if (pending >= 0) {  // the lanes holding a leaf scan together
      NodeMeta xm = load_meta(tv.meta, pending);
      if (st) st[2] += 1;
      lane_scan_leaf<D, PER>(tv, q, pending, xm.start, xm.count, H, st);
      pending = -1;
    }
  }
  if (stats) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = stv[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
  if (valid) {
    lane_heap_finish(H);
    if (sorted) lane_heap_sort(H);
  }
  __syncwarp();
  for (int qq = 0; qq < 32; ++qq) {
    int64_t s2 = gw * 32 + qq;
    if (s2 >= nq) break;
    int64_t row = order ? (int64_t)order[s2] : s2;
    const unsigned long long* rk = keys + qq * KS + 1;
    const int32_t* ri = ids + qq * KS + 1;
    for (int j = lane; j < k; j += 32) {
      int32_t id = ri[j];
      dist[row * k + j] = sqrt(__longlong_as_double((long long)rk[j]));
      idx[row * k + j] = id < 0 ? -2 : (int64_t)id;
    }
  }
}

// ============================================ persistent bottom-up search (v5)
// The bottom-up search of k_knn_up run by a persistent grid: each lane keeps
// taking queries until the queue is empty.  Per-query work is very uneven
// (clustered catalogues), so a warp that owned a fixed 32 queries spent most of
// its instructions on its slowest lane; here a lane that finishes writes its row
// and takes the next query (queries are handed out in leaf order, 64 at a time
// per warp from a global counter), so lanes stay busy until the queue drains.
template <int D, bool PER>
__global__ void __launch_bounds__(128) k_knn_persist(TreeView tv, const double* __restrict__ Q,
                                                     const int32_t* __restrict__ order,
                                                     const int32_t* __restrict__ qleaf,
                                                     int64_t nq, int k, int sorted,
                                                     unsigned long long* __restrict__ counter,
                                                     double* __restrict__ dist,
                                                     int64_t* __restrict__ idx,
                                                     unsigned long long* __restrict__ stats) {
  constexpr int NV = (D + 3) / 4;
  constexpr int PF = 4 * NV + 1;
  constexpr unsigned kBatch = 64;
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long stv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long* st = stats ? stv : nullptr;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int KS = heap_stride(k);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem) + (size_t)w * 32 * KS;
  int32_t* ids = reinterpret_cast<int32_t*>(reinterpret_cast<unsigned long long*>(smem) +
                                            (size_t)nw * 32 * KS) +
                 (size_t)w * 32 * KS;
  LaneHeap H;
  H.hk = keys + lane * KS;
  H.hi = ids + lane * KS;
  H.k = k;
  const unsigned long long kHugeKey = (unsigned long long)__double_as_longlong(CKD_HUGE);

  // warp-uniform batch of query slots [bnext, bend)
  unsigned long long bnext = 0, bend = 0;
  bool exhausted = false;
  // per-lane state
  bool active = false;
  int64_t row = 0;
  double q[D];
  QueryScreen<D, PER> qs;
  int32_t pending = -1, C = -1, parent = -1;
  bool done = true;
  int32_t sn[kUpStack];
  float sd[kUpStack];
  int top = 0;
  for (;;) {
    // ---- refill idle lanes
    unsigned want = __ballot_sync(0xffffffffu, !active);
    while (want && !exhausted) {
      if (bnext >= bend) {
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(counter, (unsigned long long)kBatch);
        b = __shfl_sync(0xffffffffu, b, 0);
        if (b >= (unsigned long long)nq) {
          exhausted = true;
          break;
        }
        bnext = b;
        bend = min(b + kBatch, (unsigned long long)nq);
      }
      unsigned avail = (unsigned)(bend - bnext);
      unsigned rank = __popc(want & ((1u << lane) - 1));
      bool take = !active && rank < avail;
      unsigned taken = min((unsigned)__popc(want), avail);
      if (take) {
        int64_t slot = (int64_t)(bnext + rank);
        int64_t qi = order ? (int64_t)order[slot] : slot;
        row = qi;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          q[j] = Q[qi * D + j];
          qs.q32[j] = __double2float_rn(q[j]);
          qs.dlt[j] = kTwoM21 * (fabsf(qs.q32[j]) + tv.slack[j]) * 1.0001f;
        }
        H.n = 0;
        H.wkey = kHugeKey;
        H.wid = -1;
        H.wd32 = FLT_MAX;
        int32_t leaf;
        NodeMeta lm;
        if (qleaf) {
          leaf = qleaf[qi];
          lm = load_meta(tv.meta, leaf);
        } else {
          leaf = 0;
          lm = load_meta(tv.meta, 0);
          while (lm.left >= 0) {
            double qa = 0.0;
#pragma unroll
            for (int j = 0; j < D; ++j)
              if (j == lm.axis) qa = q[j];
            leaf = qa < lm.split ? lm.left : lm.left + 1;
            lm = load_meta(tv.meta, leaf);
          }
        }
        pending = leaf;
        C = leaf;
        parent = lm.parent;
        top = 0;
        done = false;
        active = true;
      }
      bnext += taken;
      want = __ballot_sync(0xffffffffu, !active);
    }
    if (!__any_sync(0xffffffffu, active)) break;

    // ---- advance each active lane to a leaf or to completion
    while (active && !done && pending < 0) {
      if (top > 0) {
        --top;
        if (sd[top] > H.wd32) continue;
        int32_t x = sn[top];
        if (x < 0) {
          pending = x & 0x7fffffff;
          continue;
        }
        if (st) st[0] += 1;
        const float4* r2 = tv.pair + (int64_t)x * PF;
        float llo[4 * NV], lhi[4 * NV], rlo[4 * NV], rhi[4 * NV];
#pragma unroll
        for (int h = 0; h < NV; ++h) {
          float4 a = __ldg(&r2[h]), b = __ldg(&r2[NV + h]);
          float4 c = __ldg(&r2[2 * NV + h]), d = __ldg(&r2[3 * NV + h]);
          llo[4 * h] = a.x; llo[4 * h + 1] = a.y; llo[4 * h + 2] = a.z; llo[4 * h + 3] = a.w;
          lhi[4 * h] = b.x; lhi[4 * h + 1] = b.y; lhi[4 * h + 2] = b.z; lhi[4 * h + 3] = b.w;
          rlo[4 * h] = c.x; rlo[4 * h + 1] = c.y; rlo[4 * h + 2] = c.z; rlo[4 * h + 3] = c.w;
          rhi[4 * h] = d.x; rhi[4 * h + 1] = d.y; rhi[4 * h + 2] = d.z; rhi[4 * h + 3] = d.w;
        }
        int4 xi = __ldg(reinterpret_cast<const int4*>(&r2[4 * NV]));
        float ml = rec_mind_lb<D, PER>(tv, qs, llo, lhi);
        float mr = rec_mind_lb<D, PER>(tv, qs, rlo, rhi);
        int32_t L = xi.x | (xi.z ? (int32_t)0x80000000 : 0);
        int32_t R = xi.y | (xi.w ? (int32_t)0x80000000 : 0);
        bool nl = ml <= H.wd32, nr = mr <= H.wd32;
        if (nl && nr) {
          bool lf = ml <= mr;
          sn[top] = lf ? R : L;
          sd[top] = lf ? mr : ml;
          sn[top + 1] = lf ? L : R;
          sd[top + 1] = lf ? ml : mr;
          top += 2;
        } else if (nl || nr) {
          sn[top] = nl ? L : R;
          sd[top] = nl ? ml : mr;
          top += 1;
        }
      } else {
        if (parent < 0) {
          done = true;
          continue;
        }
        float r = sqrtf(H.wd32) * 1.0000003f;
        const float* c32 = tv.cell32 + (int64_t)C * 2 * D;
        bool inside = true;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          float2 cl = __ldg(reinterpret_cast<const float2*>(c32) + j);
          inside = inside && (qs.q32[j] - r - qs.dlt[j] >= cl.x) &&
                   (qs.q32[j] + r + qs.dlt[j] <= cl.y);
        }
        if (inside) {
          if (st) st[7] += 1;
          done = true;
          continue;
        }
        if (st) st[1] += 1;
        const float4* rec = tv.pair + (int64_t)parent * PF;
        int4 info = __ldg(reinterpret_cast<const int4*>(&rec[4 * NV]));
        const int side = (info.x == C) ? 1 : 0;
        float lo[4 * NV], hi[4 * NV];
#pragma unroll
        for (int h = 0; h < NV; ++h) {
          float4 a = __ldg(&rec[side * 2 * NV + h]), b = __ldg(&rec[side * 2 * NV + NV + h]);
          lo[4 * h] = a.x; lo[4 * h + 1] = a.y; lo[4 * h + 2] = a.z; lo[4 * h + 3] = a.w;
          hi[4 * h] = b.x; hi[4 * h + 1] = b.y; hi[4 * h + 2] = b.z; hi[4 * h + 3] = b.w;
        }
        float ms = rec_mind_lb<D, PER>(tv, qs, lo, hi);
        if (ms <= H.wd32) {
          int32_t S = side ? info.y : info.x;
          int sleaf = side ? info.w : info.z;
          sn[0] = S | (sleaf ? (int32_t)0x80000000 : 0);
          sd[0] = ms;
          top = 1;
        }
        C = parent;
        parent = load_meta(tv.meta, C).parent;
      }
    }
    // ---- finished lanes order their heap; the warp writes those rows coalesced
    const bool fin = active && done && pending < 0;
    if (fin) {
      lane_heap_finish(H);
      if (sorted) lane_heap_sort(H);
      active = false;
    }
    unsigned finm = __ballot_sync(0xffffffffu, fin);
    if (finm) {
      __syncwarp();
      while (finm) {
        const int src = __ffs(finm) - 1;
        finm &= finm - 1;
        const int64_t r = __shfl_sync(0xffffffffu, row, src);
        const unsigned long long* rk = keys + src * KS + 1;
        const int32_t* ri = ids + src * KS + 1;
        for (int j = lane; j < k; j += 32) {
          int32_t id = ri[j];
          dist[r * k + j] = sqrt(__longlong_as_double((long long)rk[j]));
          idx[r * k + j] = id < 0 ? -2 : (int64_t)id;
        }
      }
      __syncwarp();
    }
    // ---- lanes holding a leaf scan together
    if (pending >= 0) {
      NodeMeta xm = load_meta(tv.meta, pending);
      if (st) st[2] += 1;
      lane_scan_leaf<D, PER>(tv, q, pending, xm.start, xm.count, H, st);
      pending = -1;
    }
  }
  if (stats) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = stv[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
}

// ========================================== warp-per-bucket search (v6)
// Queries that fall in the same leaf form a bucket; one warp serves a bucket of
// up to 32 queries with regular, fully lane-parallel loops:
//  1. a bucket radius R is guessed from the local density (the nearest ancestor
//     holding at least 2k points);
//  2. every leaf whose FP32 box lies within R of the bucket's bounding box is
//     collected by a warp-parallel frontier walk from the root, and the point
//     indices of those leaves form the candidate list (shared memory);
//  3. for each query the warp streams the candidates (one per lane, exact FP64
//     squared distance with the reference arithmetic) into a warp-wide sorted
//     top-32 list (lane j holds rank j): candidates that rank before the current
//     32nd are compacted into a pending buffer, and every 32 pending entries are
//     bitonic-sorted and bitonic-merged into the list;
//  4. every point outside the candidate list is farther than R from every query
//     of the bucket, so the list is exact iff its k-th squared distance is <= R^2
//     (or the list covers the whole tree).  Unresolved queries retry with 2R, up
//     to kBucketRounds rounds; the rest go to a fallback list that the per-lane
//     kernel finishes.
constexpr int kBucketCmax = 1536;   // candidate points per bucket
constexpr int kBucketFmax = 384;    // frontier capacity
constexpr int kBucketRounds = 4;

struct KV {
  unsigned long long k;
  int32_t i;
};

__device__ __forceinline__ bool kv_lt(unsigned long long ka, int32_t ia, unsigned long long kb,
                                      int32_t ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// one compare-exchange stage of a bitonic network across the warp
__device__ __forceinline__ void bitonic_step(unsigned long long& key, int32_t& id, int stride,
                                             bool ascending_block) {
  const int lane = threadIdx.x & 31;
  unsigned long long ok = __shfl_xor_sync(0xffffffffu, key, stride);
  int32_t oi = __shfl_xor_sync(0xffffffffu, id, stride);
  bool lower = (lane & stride) == 0;
  bool other_smaller = kv_lt(ok, oi, key, id);
  // the lower lane keeps the smaller element in an ascending block
  bool take = (lower == ascending_block) ? other_smaller : !other_smaller && !(ok == key && oi == id);
  if (take) {
    key = ok;
    id = oi;
  }
}

__device__ __forceinline__ void bitonic_sort32(unsigned long long& key, int32_t& id) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
    bool asc = (lane & size) == 0 || size == 32;
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) bitonic_step(key, id, stride, asc);
  }
}

// merge an ascending 32-list (tk, ti) with an ascending 32-list (pk, pi), keep the
// 32 smallest, ascending
__device__ __forceinline__ void merge_top32(unsigned long long& tk, int32_t& ti,
                                            unsigned long long pk, int32_t pi) {
  unsigned long long rk = __shfl_xor_sync(0xffffffffu, pk, 31);
  int32_t ri = __shfl_xor_sync(0xffffffffu, pi, 31);
  if (kv_lt(rk, ri, tk, ti)) {
    tk = rk;
    ti = ri;
  }
#pragma unroll
  for (int stride = 16; stride > 0; stride >>= 1) bitonic_step(tk, ti, stride, true);
}

template <int D, bool PER>
__device__ __forceinline__ float boxbox_gap_lb(const TreeView& tv, const float (&blo)[D],
                                               const float (&bhi)[D], const float* nb,
                                               const float (&dlt)[D]) {
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    float2 lh = __ldg(reinterpret_cast<const float2*>(nb) + j);
    float g = fmaxf(fmaxf(lh.x - bhi[j], blo[j] - lh.y), 0.0f);
    if (PER && g > 0.0f) {
      float L = (float)tv.L[j];
      float wrapg = L - (fmaxf(bhi[j], lh.y) - fminf(blo[j], lh.x));
      g = fminf(g, fmaxf(wrapg, 0.0f));
    }
    g = fmaxf(g - dlt[j], 0.0f);
    s = fmaf(g, g, s);
  }
  return s * kShrink;
}

template <int D, bool PER>
__global__ void __launch_bounds__(128) k_knn_bucket(TreeView tv, const double* __restrict__ Q,
                                                    const int32_t* __restrict__ order,
                                                    const int4* __restrict__ buckets,
                                                    int64_t nbuckets, int k, float alpha,
                                                    double* __restrict__ dist,
                                                    int64_t* __restrict__ idx,
                                                    int32_t* __restrict__ fallback,
                                                    unsigned int* __restrict__ nfallback,
                                                    int64_t fallback_cap,
                                                    unsigned long long* __restrict__ stats) {
  __shared__ int32_t s_cand[4][kBucketCmax];
  __shared__ int32_t s_front[4][2][kBucketFmax];
  __shared__ unsigned long long s_pk[4][64];
  __shared__ int32_t s_pi[4][64];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned long long kHugeKey = (unsigned long long)__double_as_longlong(CKD_HUGE);
  const unsigned lt_mask = (1u << lane) - 1;
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int32_t* cand = s_cand[w];
  for (int64_t b = (int64_t)blockIdx.x * 4 + w; b < nbuckets; b += (int64_t)gridDim.x * 4) {
    const int4 bk = buckets[b];  // {first slot in order, queries, leaf, 0}
    const int m = bk.y;
    const bool has_q = lane < m;
    const int64_t qi = has_q ? (int64_t)order[bk.x + lane] : 0;
    double q[D];
    float blo[D], bhi[D], dlt[D];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      q[j] = has_q ? Q[qi * D + j] : 0.0;
      float lo = has_q ? __double2float_rd(q[j]) : FLT_MAX;
      float hi = has_q ? __double2float_ru(q[j]) : -FLT_MAX;
      for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      }
      blo[j] = lo;
      bhi[j] = hi;
      dlt[j] = kTwoM21 * (fmaxf(fabsf(lo), fabsf(hi)) + tv.slack[j]) * 1.0001f;
    }
    // ---- density radius from the nearest ancestor with >= 2k points
    float R;
    {
      int32_t A = bk.z;
      NodeMeta am = load_meta(tv.meta, A);
      while (am.count < 2 * k && am.parent >= 0) {
        A = am.parent;
        am = load_meta(tv.meta, A);
      }
      const float* ab = tv.box32 + (int64_t)A * 2 * D;
      float side[D], smax = 0.0f;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        float2 lh = __ldg(reinterpret_cast<const float2*>(ab) + j);
        side[j] = lh.y - lh.x;
        smax = fmaxf(smax, side[j]);
      }
      float lv = 0.0f;  // log volume with degenerate sides floored
#pragma unroll
      for (int j = 0; j < D; ++j) lv += __logf(fmaxf(side[j], 1e-3f * smax + 1e-30f));
      // volume of the k-ball at the ancestor's density, unit-ball volume ~ 4 for d = 3
      float lr = (__logf((float)k / (float)am.count) + lv - __logf(4.0f)) / (float)D;
      R = alpha * __expf(lr);
      if (!(R > 0.0f) || !(R < FLT_MAX)) R = smax + 1e-30f;
    }
    unsigned unresolved = __ballot_sync(0xffffffffu, has_q);
    for (int round = 0; round < kBucketRounds && unresolved; ++round, R *= 2.0f) {
      // ---- candidate leaves within R of the bucket box (frontier walk)
      const float R2 = R * R;
      int nf = 1, cur = 0, nc = 0;
      bool overflow = false, all_leaves = true;
      if (lane == 0) s_front[w][0][0] = 0;
      __syncwarp();
      while (nf > 0 && !overflow) {
        int nn = 0;
        for (int base = 0; base < nf; base += 32) {
          const int fi = base + lane;
          int32_t node = fi < nf ? s_front[w][cur][fi] : -1;
          bool need = false, leaf = false;
          NodeMeta nm;
          if (node >= 0) {
            if (st) st[0] += 1;
            need = boxbox_gap_lb<D, PER>(tv, blo, bhi, tv.box32 + (int64_t)node * 2 * D, dlt) <= R2;
            nm = load_meta(tv.meta, node);
            leaf = nm.left < 0;
            if (!need) all_leaves = false;
          }
          // internal: both children to the next frontier
          unsigned im = __ballot_sync(0xffffffffu, need && !leaf);
          int ipos = nn + 2 * __popc(im & lt_mask);
          if (need && !leaf && ipos + 1 < kBucketFmax) {
            s_front[w][1 - cur][ipos] = nm.left;
            s_front[w][1 - cur][ipos + 1] = nm.left + 1;
          }
          nn += 2 * __popc(im);
          if (nn > kBucketFmax) overflow = true;
          // leaves: append their points
          unsigned lm = __ballot_sync(0xffffffffu, need && leaf);
          while (lm) {
            const int src = __ffs(lm) - 1;
            lm &= lm - 1;
            const int32_t s0 = __shfl_sync(0xffffffffu, nm.start, src);
            const int32_t c0 = __shfl_sync(0xffffffffu, nm.count, src);
            if (nc + c0 > kBucketCmax) {
              overflow = true;
            } else {
              for (int i = lane; i < c0; i += 32) cand[nc + i] = s0 + i;
              nc += c0;
            }
          }
        }
        __syncwarp();
        nf = nn;
        cur = 1 - cur;
      }
      // every lane must agree: a node pruned by any lane means the list is partial
      all_leaves = __all_sync(0xffffffffu, all_leaves);
      if (overflow) break;
      __syncwarp();
      if (st) st[1] += nc;
      // ---- each unresolved query: stream the candidates into a warp top-32
      unsigned todo = unresolved;
      while (todo) {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        double qq[D];
#pragma unroll
        for (int j = 0; j < D; ++j) qq[j] = __shfl_sync(0xffffffffu, q[j], src);
        unsigned long long tk = kHugeKey;  // lane j holds rank j
        int32_t ti = -1;
        unsigned long long mk = kHugeKey;  // current 32nd
        int32_t mi = -1;
        int np = 0;
        for (int base = 0; base < nc; base += 32) {
          const int c = base + lane;
          unsigned long long key = kHugeKey;
          int32_t id = -1;
          bool pass = false;
          if (c < nc) {
            const int32_t p = cand[c];
            double d2 = point_d2<D, PER>(tv, qq, p);
            key = (unsigned long long)__double_as_longlong(d2);
            if (key < mk || key == mk) {
              id = __ldg(&tv.ids[p]);
              pass = kv_lt(key, id, mk, mi);
            }
          }
          unsigned pm = __ballot_sync(0xffffffffu, pass);
          if (pass) {
            const int pos = np + __popc(pm & lt_mask);
            s_pk[w][pos] = key;
            s_pi[w][pos] = id;
          }
          np += __popc(pm);
          if (st) st[2] += __popc(pm);
          __syncwarp();
          if (np >= 32) {
            unsigned long long pk = s_pk[w][lane];
            int32_t pi = s_pi[w][lane];
            __syncwarp();
            if (lane < np - 32) {  // keep the overflow for the next merge
              s_pk[w][lane] = s_pk[w][lane + 32];
              s_pi[w][lane] = s_pi[w][lane + 32];
            }
            np -= 32;
            bitonic_sort32(pk, pi);
            merge_top32(tk, ti, pk, pi);
            mk = __shfl_sync(0xffffffffu, tk, 31);
            mi = __shfl_sync(0xffffffffu, ti, 31);
            if (st) st[3] += 1;
            __syncwarp();
          }
        }
        if (np > 0) {
          unsigned long long pk = lane < np ? s_pk[w][lane] : kHugeKey;
          int32_t pi = lane < np ? s_pi[w][lane] : -1;
          __syncwarp();
          bitonic_sort32(pk, pi);
          merge_top32(tk, ti, pk, pi);
          if (st) st[3] += 1;
        }
        // exact iff the k-th is within the radius the leaves were gathered with
        // (every point left out has a larger squared distance), or the
        // candidates cover the whole tree
        const unsigned long long kk = __shfl_sync(0xffffffffu, tk, k - 1);
        const double r2d = (double)R2;
        const bool ok = all_leaves || (kk != kHugeKey && kk <= (unsigned long long)__double_as_longlong(r2d));
        if (ok) {
          const int64_t row = __shfl_sync(0xffffffffu, qi, src);
          if (lane < k) {
            dist[row * k + lane] = sqrt(__longlong_as_double((long long)tk));
            idx[row * k + lane] = ti < 0 ? -2 : (int64_t)ti;
          }
          unresolved &= ~(1u << src);
        }
      }
    }
    // ---- leftovers go to the fallback list
    if (unresolved) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(nfallback, (unsigned)__popc(unresolved));
      base = __shfl_sync(0xffffffffu, base, 0);
      const int64_t pos = (int64_t)base + __popc(unresolved & lt_mask);
      if (((unresolved >> lane) & 1u) && pos < fallback_cap) fallback[pos] = (int32_t)qi;
      if (st) st[4] += __popc(unresolved);
    }
    __syncwarp();
  }
  if (stats) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = st[c];
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
}

// ======================================= learned-radius gather search (bounded)
// One warp serves 32 consecutive queries of the leaf order (spatially adjacent),
// each with a predicted squared radius r2[q] from k_mlp_radius:
//  1. gather: a warp-parallel frontier walk from the root collects every leaf
//     whose FP32 box lies within R = max over lanes of sqrt(r2) of the bucket's
//     bounding box;
//  2. scan: for each gathered leaf that some lane's current bound reaches, the
//     32 lanes screen the leaf's points together (the same leaf-relative FP32
//     copy read by all lanes, one query per lane); a point whose FP32 lower bound
//     is within the lane's bound joins the lane's candidate buffer;
//  3. flush: when a buffer could overflow, and at the end, every lane evaluates
//     its buffered candidates in FP64 (reference arithmetic) and inserts them into
//     its heap, which starts full of (r2, INT32_MAX) sentinels as in the bounded
//     per-lane kernel, so the bound only shrinks.
// The screen loop is one instruction stream for all lanes; only the flushes
// diverge.  A query ends exact when no sentinel remains.  Otherwise (fewer than k
// points within its radius), or when the bucket's gather overflows, or when its
// radius is not finite, the query is appended to miss[] for the plain rerun.
constexpr int kGatherC = 48;         // candidate buffer per lane (>= 32)
constexpr int kGatherLeaves = 384;   // gathered leaves per bucket
constexpr int kGatherFront = 512;    // frontier capacity per level (two buffers)
static_assert(2 * kGatherFront <= kGatherC * 32, "frontier shares the candidate buffer");

__host__ __device__ inline size_t gather_smem_per_warp(int k) {
  return (size_t)32 * heap_stride(k) * (sizeof(unsigned long long) + sizeof(int32_t)) +
         (size_t)kGatherC * 32 * sizeof(int32_t) + (size_t)kGatherLeaves * sizeof(int32_t);
}

// replace the root of a 1-based max-heap (keys = FP64 bit patterns, ties by id)
// by (key, id) and sift it down
__device__ __forceinline__ void heap_replace_top(unsigned long long* hk, int32_t* hi, int k,
                                                 unsigned long long key, int32_t id) {
  int s = 1;
  for (;;) {
    int l = 2 * s;
    if (l > k) break;
    unsigned long long kc;
    int32_t ic;
    int c;
    if (l < k) {
      ulonglong2 kk = *reinterpret_cast<const ulonglong2*>(hk + l);
      int2 ii = *reinterpret_cast<const int2*>(hi + l);
      bool right = kk.x < kk.y || (kk.x == kk.y && ii.x < ii.y);
      kc = right ? kk.y : kk.x;
      ic = right ? ii.y : ii.x;
      c = right ? l + 1 : l;
    } else {
      kc = hk[l];
      ic = hi[l];
      c = l;
    }
    if (!(key < kc || (key == kc && id < ic))) break;
    hk[s] = kc;
    hi[s] = ic;
    s = c;
  }
  hk[s] = key;
  hi[s] = id;
}

template <int D, bool PER>
__global__ void __launch_bounds__(128) k_knn_gather(TreeView tv, const double* __restrict__ Q,
                                                    const int32_t* __restrict__ order, int64_t nq,
                                                    int k, int sorted, const double* __restrict__ r2,
                                                    double* __restrict__ dist,
                                                    int64_t* __restrict__ idx,
                                                    int32_t* __restrict__ miss,
                                                    unsigned* __restrict__ nmiss,
                                                    unsigned long long* __restrict__ stats) {
  constexpr int NV = (D + 3) / 4;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int KS = heap_stride(k);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem) + (size_t)w * 32 * KS;
  int32_t* i32 = reinterpret_cast<int32_t*>(reinterpret_cast<unsigned long long*>(smem) +
                                            (size_t)nw * 32 * KS);
  int32_t* ids = i32 + (size_t)w * 32 * KS;
  int32_t* cand = i32 + (size_t)nw * 32 * KS + (size_t)w * kGatherC * 32;  // [slot][lane]
  int32_t* front = cand;  // gather phase only
  int32_t* leaves = i32 + (size_t)nw * 32 * KS + (size_t)nw * kGatherC * 32 +
                    (size_t)w * kGatherLeaves;

  const int64_t gw = (int64_t)blockIdx.x * nw + w;
  const int64_t slot = gw * 32 + lane;
  const bool valid = slot < nq;
  const int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
  QueryScreen<D, PER> qs;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    q[j] = valid ? Q[qi * D + j] : 0.0;
    qs.q32[j] = __double2float_rn(q[j]);
    qs.dlt[j] = kTwoM21 * (fabsf(qs.q32[j]) + tv.slack[j]) * 1.0001f;
  }
  // heap full of sentinels at the predicted radius
  const double rr = valid ? r2[qi] : 0.0;
  const bool part = valid && rr < CKD_HUGE;  // takes part in the bounded search
  unsigned long long* hk = keys + lane * KS;
  int32_t* hi = ids + lane * KS;
  const unsigned long long skey =
      part ? (unsigned long long)__double_as_longlong(rr) : 0ull;
  for (int s = 1; s <= k; ++s) {
    hk[s] = skey;
    hi[s] = 0x7fffffff;
  }
  unsigned long long wkey = skey;
  int32_t wid = 0x7fffffff;
  float wd32 = part ? __double2float_ru(rr) : -1.0f;  // -1: never passes a screen

  // ---- bucket box and gather radius over the participating lanes
  float blo[D], bhi[D], dlt[D];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    float lo = part ? __double2float_rd(q[j]) : FLT_MAX;
    float hh = part ? __double2float_ru(q[j]) : -FLT_MAX;
    for (int o = 16; o > 0; o >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(FULL, lo, o));
      hh = fmaxf(hh, __shfl_xor_sync(FULL, hh, o));
    }
    blo[j] = lo;
    bhi[j] = hh;
    dlt[j] = kTwoM21 * (fmaxf(fabsf(lo), fabsf(hh)) + tv.slack[j]) * 1.0001f;
  }
  float R = part ? __fsqrt_ru(wd32) : 0.0f;
  for (int o = 16; o > 0; o >>= 1) R = fmaxf(R, __shfl_xor_sync(FULL, R, o));
  const float R2 = __fmul_ru(R, R);
  const bool any_part = __any_sync(FULL, part);

  // ---- 1. gather the leaves within R of the bucket box
  int nlv = 0;
  bool overflow = false;
  if (any_part) {
    int nf = 1, cur = 0;
    if (lane == 0) front[0] = 0;
    __syncwarp();
    while (nf > 0 && !overflow) {
      int nn = 0;
      for (int base = 0; base < nf; base += 32) {
        const int fi = base + lane;
        const int32_t node = fi < nf ? front[cur * kGatherFront + fi] : -1;
        bool need = false, leaf = false;
        NodeMeta nm;
        if (node >= 0) {
          if (stats) st[0] += 1;
          need = boxbox_gap_lb<D, PER>(tv, blo, bhi, tv.box32 + (int64_t)node * 2 * D, dlt) <= R2;
          nm = load_meta(tv.meta, node);
          leaf = nm.left < 0;
        }
        const unsigned im = __ballot_sync(FULL, need && !leaf);
        const int ipos = nn + 2 * __popc(im & lt_mask);
        if (need && !leaf && ipos + 1 < kGatherFront) {
          front[(1 - cur) * kGatherFront + ipos] = nm.left;
          front[(1 - cur) * kGatherFront + ipos + 1] = nm.left + 1;
        }
        nn += 2 * __popc(im);
        const unsigned lm = __ballot_sync(FULL, need && leaf);
        const int lpos = nlv + __popc(lm & lt_mask);
        if (need && leaf && lpos < kGatherLeaves) leaves[lpos] = node;
        nlv += __popc(lm);
      }
      if (nn > kGatherFront || nlv > kGatherLeaves) overflow = true;
      __syncwarp();
      nf = nn;
      cur = 1 - cur;
    }
  }
  if (stats && lane == 0) st[1] += nlv;

  // ---- 2./3. screen the gathered leaves, flushing candidates into the heaps
  int cnt = 0;
  auto flush = [&]() {
    const int mx = __reduce_max_sync(FULL, (unsigned)cnt);
    if (stats && lane == 0) st[4] += 1;
    for (int j = 0; j < mx; ++j) {
      if (j < cnt) {
        if (stats) st[5] += 1;
        const int32_t p = cand[j * 32 + lane];
        const double d2 = point_d2<D, PER>(tv, q, p);
        const unsigned long long key = (unsigned long long)__double_as_longlong(d2);
        if (key <= wkey) {
          const int32_t id = __ldg(&tv.ids[p]);
          if (key < wkey || id < wid) {
            if (stats) st[6] += 1;
            heap_replace_top(hk, hi, k, key, id);
            wkey = hk[1];
            wid = hi[1];
            wd32 = __double2float_ru(__longlong_as_double((long long)wkey));
          }
        }
      }
    }
    cnt = 0;
    __syncwarp();
  };
  if (!overflow) {
    __syncwarp();  // the frontier shared the candidate buffer
    for (int li = 0; li < nlv; ++li) {
      const int32_t leaf = leaves[li];
      const bool reach = part && node_mind_lb<D, PER>(tv, qs, leaf) <= wd32;
      if (!__any_sync(FULL, reach)) continue;
      if (stats) st[2] += reach;
      const NodeMeta m = load_meta(tv.meta, leaf);
      float qr[D], e[D];
      {
        const double* b = tv.box + (int64_t)leaf * 2 * D;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          double lo = __ldg(&b[2 * j]), hh = __ldg(&b[2 * j + 1]);
          double c = leaf_centre(lo, hh);
          double r = fmax(c - lo, hh - c);
          double x = q[j] - c;
          if (PER) {
            double h = 0.5 * tv.L[j];
            if (x > h) x -= tv.L[j];
            else if (x < -h) x += tv.L[j];
          }
          qr[j] = __double2float_rn(x);
          e[j] = kTwoM21 * (float)(r + fabs(x) + (PER ? tv.L[j] : 0.0)) * 1.0001f + 1e-37f;
        }
      }
      for (int base = 0; base < m.count; base += 32) {
        const int c = min(32, m.count - base);
        if (__any_sync(FULL, cnt + c > kGatherC)) flush();
        const int32_t p0 = m.start + base;
        if (stats) st[3] += c;
        for (int i = 0; i < c; ++i) {
          float v[4 * NV];
#pragma unroll
          for (int h = 0; h < NV; ++h) {
            float4 f = __ldg(&tv.pts32[(int64_t)(p0 + i) * NV + h]);
            v[4 * h] = f.x;
            v[4 * h + 1] = f.y;
            v[4 * h + 2] = f.z;
            v[4 * h + 3] = f.w;
          }
          float s = 0.0f;
#pragma unroll
          for (int j = 0; j < D; ++j) {
            float a = fabsf(v[j] - qr[j]);
            if (PER) a = fminf(a, (float)tv.L[j] - a);
            a = fmaxf(a - e[j], 0.0f);
            s = fmaf(a, a, s);
          }
          if (s * kShrink <= wd32) {
            cand[cnt * 32 + lane] = p0 + i;
            ++cnt;
          }
        }
      }
    }
    flush();
  }

  // ---- queries left with a sentinel go to the plain rerun
  const bool missed = valid && (!part || overflow || wid == 0x7fffffff);
  const unsigned missmask = __ballot_sync(FULL, missed);
  if (missmask) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(nmiss, (unsigned)__popc(missmask));
    base = __shfl_sync(FULL, base, 0);
    if (missed) miss[base + __popc(missmask & lt_mask)] = (int32_t)qi;
    if (stats && lane == 0) st[7] += __popc(missmask);
  }
  if (stats) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = st[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
  if (sorted && valid && !missed) {
    for (int end = k; end > 1; --end) {
      unsigned long long key = hk[end];
      int32_t id = hi[end];
      hk[end] = hk[1];
      hi[end] = hi[1];
      int s = 1;
      for (;;) {
        int l = 2 * s;
        if (l >= end) break;
        int c = l;
        unsigned long long kc = hk[l];
        int32_t ic = hi[l];
        if (l + 1 < end) {
          unsigned long long kr = hk[l + 1];
          int32_t ir = hi[l + 1];
          if (kc < kr || (kc == kr && ic < ir)) {
            c = l + 1;
            kc = kr;
            ic = ir;
          }
        }
        if (!(key < kc || (key == kc && id < ic))) break;
        hk[s] = kc;
        hi[s] = ic;
        s = c;
      }
      hk[s] = key;
      hi[s] = id;
    }
  }
  __syncwarp();
  for (int qq = 0; qq < 32; ++qq) {
    const int64_t s2 = gw * 32 + qq;
    if (s2 >= nq) break;
    if ((missmask >> qq) & 1u) continue;
    const int64_t row = order ? (int64_t)order[s2] : s2;
    const unsigned long long* rk = keys + qq * KS + 1;
    const int32_t* ri = ids + qq * KS + 1;
    for (int j = lane; j < k; j += 32) {
      dist[row * k + j] = sqrt(__longlong_as_double((long long)rk[j]));
      idx[row * k + j] = (int64_t)ri[j];
    }
  }
}

// bucket list: for every leaf holding queries, ceil(count / 32) buckets
__global__ void k_bucket_count(const NodeMeta* __restrict__ meta, int32_t n_nodes,
                               const int32_t* __restrict__ off, int32_t* __restrict__ nb) {
  int32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_nodes) return;
  NodeMeta m = meta[a];
  int c = 0;
  if (m.left < 0) {
    int32_t cnt = off[m.start + 1] - off[m.start];
    c = (cnt + 31) / 32;
  }
  nb[a] = c;
}

__global__ void k_bucket_emit(const NodeMeta* __restrict__ meta, int32_t n_nodes,
                              const int32_t* __restrict__ off, const int32_t* __restrict__ nbo,
                              int4* __restrict__ buckets) {
  int32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_nodes) return;
  NodeMeta m = meta[a];
  if (m.left >= 0) return;
  int32_t b0 = off[m.start], cnt = off[m.start + 1] - b0;
  int32_t o = nbo[a];
  for (int c = 0; c * 32 < cnt; ++c)
    buckets[o + c] = make_int4(b0 + 32 * c, min(32, cnt - 32 * c), a, 0);
}

// ------------------------------------------------------------ query order
template <int D>
__global__ void k_locate(const NodeMeta* __restrict__ meta, const double* __restrict__ Q,
                         int64_t nq, int32_t* __restrict__ key, int32_t* __restrict__ hist,
                         int32_t* __restrict__ qleaf, const int32_t* __restrict__ qroot) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  double q[D];
#pragma unroll
  for (int j = 0; j < D; ++j) q[j] = Q[i * D + j];
  int32_t node = qroot ? qroot[i] : 0;
  NodeMeta m = load_meta(meta, node);
  while (m.left >= 0) {
    double qa = 0.0;
#pragma unroll
    for (int j = 0; j < D; ++j)
      if (j == m.axis) qa = q[j];
    node = qa < m.split ? m.left : m.left + 1;
    m = load_meta(meta, node);
  }
  key[i] = m.start;
  if (qleaf) qleaf[i] = node;
  atomicAdd(&hist[m.start], 1);
}

__global__ void k_bucket_scatter(const int32_t* __restrict__ key, int64_t nq,
                                 const int32_t* __restrict__ off, int32_t* __restrict__ cursor,
                                 int32_t* __restrict__ order) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  int32_t b = key[i];
  int32_t pos = off[b] + atomicAdd(&cursor[b], 1);
  order[pos] = (int32_t)i;
}

template <int D, bool PER>
ckd_status knn_launch(const ckd_tree* t, const double* q, const int32_t* order,
                      const int32_t* qleaf, int64_t nq, int k, int sorted, double* dist,
                      int64_t* idx, cudaStream_t s, int force_variant = -1) {
  TreeView tv = t->view();
  const int var = force_variant >= 0 ? force_variant : knn_variant();
  if (force_variant < 0) timing_begin(s);
  struct TimingEnd {
    cudaStream_t s;
    bool on;
    ~TimingEnd() {
      if (on) timing_end(s);
    }
  } timing_guard{s, force_variant < 0};
  if (k <= kSmemK && t->screen_ok && var == 5 && t->depth < kUpStack - 2) {
    const int nwp = 4;
    size_t sm = (size_t)nwp * heap_stride(k) * 32 * (sizeof(unsigned long long) + sizeof(int32_t));
    CKD_CUDA(cudaFuncSetAttribute(k_knn_persist<D, PER>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int dev = 0, sms = 0, per_sm = 0;
    CKD_CUDA(cudaGetDevice(&dev));
    CKD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CKD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_knn_persist<D, PER>,
                                                           nwp * 32, sm));
    if (knn_blocks_per_sm() > 0) per_sm = std::min(per_sm, knn_blocks_per_sm());
    int64_t grid = std::min<int64_t>((int64_t)std::max(1, per_sm) * sms, cdiv(cdiv(nq, 32), nwp));
    unsigned long long* counter = nullptr;
    CKD_CUDA(dev_alloc((void**)&counter, sizeof(unsigned long long), s));
    CKD_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    k_knn_persist<D, PER><<<(unsigned)grid, nwp * 32, sm, s>>>(
        tv, q, order, qleaf, nq, k, sorted, counter, dist, idx, knn_stats_buffer());
    CKD_LAUNCH_CHECK();
    CKD_CUDA(dev_free(counter, s));
    return CKD_OK;
  }
  if (k <= kSmemK && t->screen_ok && var == 4 && t->depth < kUpStack - 2) {
    const int nwu = knn_warps_per_block();
    const int64_t blocks_u = cdiv(cdiv(nq, 32), nwu);
    size_t sm = (size_t)nwu * heap_stride(k) * 32 * (sizeof(unsigned long long) + sizeof(int32_t));
    const int bps = knn_blocks_per_sm();
    if (bps > 0) sm = std::max(sm, (size_t)(200 * 1024) / bps);  // cap residency via shared memory
    CKD_CUDA(cudaFuncSetAttribute(k_knn_up<D, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm));
    k_knn_up<D, PER><<<(unsigned)blocks_u, nwu * 32, sm, s>>>(tv, q, order, qleaf, nq, k, sorted,
                                                              dist, idx, knn_stats_buffer());
    CKD_LAUNCH_CHECK();
    return CKD_OK;
  }
  const int threads = 128, nw = threads / 32;
  int64_t warps = cdiv(nq, 32);
  unsigned blocks = (unsigned)cdiv(warps, nw);
  int stack_len = std::max(kStack, t->depth + 4);
  int32_t* gstack = nullptr;
  bool use_gstack = stack_len > kStack || k > kSmemK;
  if (use_gstack)
    CKD_CUDA(dev_alloc((void**)&gstack, sizeof(int32_t) * stack_len * (int64_t)blocks * nw, s));
  if (k <= kSmemK && t->screen_ok && (var == 0 || var == 7 || var == 8) &&
      t->depth < kLaneStack - 1) {
    const int nw7 = std::min(4, knn_warps_per_block());
    const unsigned blocks7 = (unsigned)cdiv(cdiv(nq, 32), nw7);
    size_t sm = (size_t)nw7 * compact_heap_bytes(k);
    const int bps = knn_blocks_per_sm();
    if (bps > 0) sm = std::max(sm, (size_t)(200 * 1024) / bps);
    if (var == 8) {
      CKD_CUDA(cudaFuncSetAttribute(k_knn_lane2<D, PER, false, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      k_knn_lane2<D, PER, false, true><<<blocks7, nw7 * 32, sm, s>>>(
          tv, q, order, nq, k, sorted, dist, idx, knn_stats_buffer());
    } else {
      CKD_CUDA(cudaFuncSetAttribute(k_knn_lane2<D, PER>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      k_knn_lane2<D, PER><<<blocks7, nw7 * 32, sm, s>>>(tv, q, order, nq, k, sorted, dist, idx,
                                                        knn_stats_buffer());
    }
    CKD_LAUNCH_CHECK();
    if (gstack) CKD_CUDA(dev_free(gstack, s));
    return CKD_OK;
  }
  if (k <= kSmemK && t->screen_ok && var == 3 && t->depth < kLaneStack - 1) {
    size_t sm = (size_t)nw * heap_stride(k) * 32 * (sizeof(unsigned long long) + sizeof(int32_t));
    CKD_CUDA(cudaFuncSetAttribute(k_knn_lane<D, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm));
    k_knn_lane<D, PER><<<blocks, threads, sm, s>>>(tv, q, order, nq, k, sorted, dist, idx,
                                                   knn_stats_buffer());
  } else if (k <= kSmemK && t->screen_ok && var != 1) {
    size_t sm = (size_t)nw * heap_stride(k) * 32 * (sizeof(unsigned long long) + sizeof(int32_t)) +
                (use_gstack ? 0 : (size_t)nw * kStack * sizeof(int32_t));
    CKD_CUDA(cudaFuncSetAttribute(k_knn_screen<D, PER>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_knn_screen<D, PER><<<blocks, threads, sm, s>>>(tv, q, order, nq, k, sorted,
                                                     use_gstack ? gstack : nullptr, stack_len,
                                                     dist, idx, knn_stats_buffer());
  } else if (k <= kSmemK) {
    size_t sm = (size_t)nw * k * 32 * (sizeof(double) + sizeof(int32_t)) +
                (use_gstack ? 0 : (size_t)nw * kStack * sizeof(int32_t));
    CKD_CUDA(cudaFuncSetAttribute(k_knn_smem<D, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm));
    k_knn_smem<D, PER><<<blocks, threads, sm, s>>>(tv, q, order, nq, k, sorted,
                                                   use_gstack ? gstack : nullptr, stack_len, dist,
                                                   idx);
  } else {
    k_knn_rows<D, PER><<<blocks, threads, 0, s>>>(tv, q, order, nq, k, sorted, gstack, stack_len,
                                                  dist, idx);
  }
  CKD_LAUNCH_CHECK();
  if (gstack) CKD_CUDA(dev_free(gstack, s));
  return CKD_OK;
}

template <int D>
ckd_status knn_dispatch_d(const ckd_tree* t, const double* q, const int32_t* order,
                          const int32_t* qleaf, int64_t nq, int k, int sorted, double* dist,
                          int64_t* idx, cudaStream_t s) {
  if (t->periodic) return knn_launch<D, true>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
  return knn_launch<D, false>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
}

template <int D>
ckd_status order_impl(const ckd_tree* t, const double* q, int64_t nq, int32_t* order,
                      int32_t* qleaf, cudaStream_t s, int32_t** off_out = nullptr,
                      const int32_t* qroot = nullptr) {
  int64_t n = t->n;
  int32_t *key = nullptr, *hist = nullptr, *off = nullptr;
  CKD_CUDA(dev_alloc((void**)&key, sizeof(int32_t) * nq, s));
  CKD_CUDA(dev_alloc((void**)&hist, sizeof(int32_t) * n, s));
  CKD_CUDA(dev_alloc((void**)&off, sizeof(int32_t) * (n + 1), s));
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * n, s));
  unsigned g = (unsigned)cdiv(nq, 256);
  k_locate<D><<<g, 256, 0, s>>>(t->meta, q, nq, key, hist, qleaf, qroot);
  CKD_LAUNCH_CHECK();
  CKD_TRY(scan_i32(hist, off, n, s));
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * n, s));
  k_bucket_scatter<<<g, 256, 0, s>>>(key, nq, off, hist, order);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(dev_free(key, s));
  CKD_CUDA(dev_free(hist, s));
  if (off_out)
    *off_out = off;
  else
    CKD_CUDA(dev_free(off, s));
  return CKD_OK;
}

// Warp-per-bucket search: locate + counting sort, bucket list, bucket kernel,
// then the per-lane kernel for any query the bucket rounds left unresolved.
template <int D, bool PER>
ckd_status bucket_run(const ckd_tree* t, const double* q, int64_t nq, int k, double* dist,
                      int64_t* idx, cudaStream_t s) {
  int32_t *order = nullptr, *off = nullptr, *nb = nullptr, *nbo = nullptr, *fb = nullptr;
  unsigned int* nfb = nullptr;
  int4* buckets = nullptr;
  const int32_t nn = t->n_nodes;
  CKD_CUDA(dev_alloc((void**)&order, sizeof(int32_t) * nq, s));
  CKD_TRY(order_impl<D>(t, q, nq, order, nullptr, s, &off));
  CKD_CUDA(dev_alloc((void**)&nb, sizeof(int32_t) * nn, s));
  CKD_CUDA(dev_alloc((void**)&nbo, sizeof(int32_t) * (nn + 1), s));
  k_bucket_count<<<(unsigned)cdiv(nn, 256), 256, 0, s>>>(t->meta, nn, off, nb);
  CKD_LAUNCH_CHECK();
  CKD_TRY(scan_i32(nb, nbo, nn, s));
  int32_t nbuckets = 0;
  CKD_CUDA(cudaMemcpyAsync(&nbuckets, nbo + nn, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaStreamSynchronize(s));
  CKD_CUDA(dev_alloc((void**)&buckets, sizeof(int4) * std::max(1, nbuckets), s));
  k_bucket_emit<<<(unsigned)cdiv(nn, 256), 256, 0, s>>>(t->meta, nn, off, nbo, buckets);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(dev_alloc((void**)&fb, sizeof(int32_t) * nq, s));
  CKD_CUDA(dev_alloc((void**)&nfb, sizeof(unsigned int), s));
  CKD_CUDA(cudaMemsetAsync(nfb, 0, sizeof(unsigned int), s));
  TreeView tv = t->view();
  int dev = 0, sms = 0, per_sm = 0;
  CKD_CUDA(cudaGetDevice(&dev));
  CKD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CKD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_knn_bucket<D, PER>, 128, 0));
  int64_t grid = std::min<int64_t>((int64_t)std::max(1, per_sm) * sms * 4, cdiv(nbuckets, 4));
  if (nbuckets > 0) {
    timing_begin(s);
    k_knn_bucket<D, PER><<<(unsigned)std::max<int64_t>(1, grid), 128, 0, s>>>(
        tv, q, order, buckets, nbuckets, k, knn_bucket_alpha(), dist, idx, fb, nfb, nq,
        knn_stats_buffer());
    CKD_LAUNCH_CHECK();
    timing_end(s);
  }
  unsigned int nfallback = 0;
  CKD_CUDA(cudaMemcpyAsync(&nfallback, nfb, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaStreamSynchronize(s));
  if ((int64_t)nfallback > nq) return fail(CKD_ERR_CUDA, "internal error: fallback list overflow");
  ckd_status st = CKD_OK;
  if (nfallback > 0) st = knn_launch<D, PER>(t, q, fb, nullptr, nfallback, k, 1, dist, idx, s, 7);
  for (void* p : {(void*)order, (void*)off, (void*)nb, (void*)nbo, (void*)fb, (void*)nfb,
                  (void*)buckets})
    dev_free(p, s);
  return st;
}

}  // namespace

ckd_status knn_stats(int enable, int64_t* out) {
  void* p = nullptr;
  CKD_CUDA(cudaGetSymbolAddress(&p, g_knn_stats));
  if (out) {
    CKD_CUDA(cudaDeviceSynchronize());
    CKD_CUDA(cudaMemcpy(out, p, sizeof(int64_t) * 8, cudaMemcpyDeviceToHost));
  }
  CKD_CUDA(cudaMemset(p, 0, sizeof(unsigned long long) * 8));
  CKD_CUDA(cudaDeviceSynchronize());
  g_stats_on = enable != 0;
  return CKD_OK;
}

ckd_status query_order(const ckd_tree* t, const double* q, int64_t nq, int32_t* order,
                       int32_t* qleaf, cudaStream_t s) {
  switch (t->d) {
    case 1: return order_impl<1>(t, q, nq, order, qleaf, s);
    case 2: return order_impl<2>(t, q, nq, order, qleaf, s);
    case 3: return order_impl<3>(t, q, nq, order, qleaf, s);
    case 4: return order_impl<4>(t, q, nq, order, qleaf, s);
    case 5: return order_impl<5>(t, q, nq, order, qleaf, s);
    case 6: return order_impl<6>(t, q, nq, order, qleaf, s);
    case 7: return order_impl<7>(t, q, nq, order, qleaf, s);
    case 8: return order_impl<8>(t, q, nq, order, qleaf, s);
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

ckd_status query_order(const ckd_tree* t, const double* q, int64_t nq, int32_t* order,
                       cudaStream_t s) {
  return query_order(t, q, nq, order, nullptr, s);
}

// leaf order of queries that each start at their own tree's root (forests)
ckd_status query_order_roots(const ckd_tree* t, const double* q, int64_t nq, int32_t* order,
                             const int32_t* qroot, cudaStream_t s) {
  switch (t->d) {
#define CKD_QO(DD) \
  case DD: return order_impl<DD>(t, q, nq, order, nullptr, s, nullptr, qroot);
    CKD_QO(1) CKD_QO(2) CKD_QO(3) CKD_QO(4) CKD_QO(5) CKD_QO(6) CKD_QO(7) CKD_QO(8)
#undef CKD_QO
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

// Queries are ordered by leaf when there are enough of them to fill many warps.
// (tuning key 6: 0 automatic, 1 always, 2 never)
bool want_order(const ckd_tree* t, int64_t nq) {
  const int mode = query_order_mode();
  if (mode == 1) return nq > 1;
  if (mode == 2) return false;
  return nq >= 4096 && nq * 8 >= t->n / 64;
}

ckd_status knn_ordered(const ckd_tree* t, const double* q, const int32_t* order,
                       const int32_t* qleaf, int64_t nq, int k, int sorted, double* dist,
                       int64_t* idx, cudaStream_t s) {
  switch (t->d) {
    case 1: return knn_dispatch_d<1>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
    case 2: return knn_dispatch_d<2>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
    case 3: return knn_dispatch_d<3>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
    case 4: return knn_dispatch_d<4>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
    case 5: return knn_dispatch_d<5>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
    case 6: return knn_dispatch_d<6>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
    case 7: return knn_dispatch_d<7>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
    case 8: return knn_dispatch_d<8>(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

ckd_status knn_ordered(const ckd_tree* t, const double* q, const int32_t* order, int64_t nq, int k,
                       int sorted, double* dist, int64_t* idx, cudaStream_t s) {
  return knn_ordered(t, q, order, nullptr, nq, k, sorted, dist, idx, s);
}

bool use_bucket(const ckd_tree* t, int64_t nq, int k) {
  const int var = knn_variant();
  return var == 6 && k <= 32 && t->screen_ok && want_order(t, nq);
}

ckd_status knn_run(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted, double* dist,
                   int64_t* idx, cudaStream_t s) {
  if (use_bucket(t, nq, k)) {
    switch (t->d * 2 + (t->periodic ? 1 : 0)) {
#define CKD_BK(DD)                                                           \
  case 2 * DD: return bucket_run<DD, false>(t, q, nq, k, dist, idx, s);      \
  case 2 * DD + 1: return bucket_run<DD, true>(t, q, nq, k, dist, idx, s);
      CKD_BK(1) CKD_BK(2) CKD_BK(3) CKD_BK(4) CKD_BK(5) CKD_BK(6) CKD_BK(7) CKD_BK(8)
#undef CKD_BK
    }
  }
  int32_t* order = nullptr;
  int32_t* qleaf = nullptr;
  if (want_order(t, nq)) {
    CKD_CUDA(dev_alloc((void**)&order, sizeof(int32_t) * nq, s));
    CKD_CUDA(dev_alloc((void**)&qleaf, sizeof(int32_t) * nq, s));
    CKD_TRY(query_order(t, q, nq, order, qleaf, s));
  }
  ckd_status st = knn_ordered(t, q, order, qleaf, nq, k, sorted, dist, idx, s);
  if (order) dev_free(order, s);
  if (qleaf) dev_free(qleaf, s);
  return st;
}

// ===================================================================
// kNN over a forest (ckd_forest_knn): every query carries its tree (qroot =
// the tree's root node); the queries of all trees are ordered by leaf and
// searched by one per-lane launch that starts each lane at its own root.
namespace {

template <int D, bool PER>
ckd_status forest_knn_impl(const ckd_tree* t, const double* q, const int32_t* qroot, int64_t nq,
                           int k, int sorted, double* dist, int64_t* idx, cudaStream_t s) {
  int32_t* order = nullptr;
  CKD_CUDA(dev_alloc((void**)&order, sizeof(int32_t) * nq, s));
  ckd_status st = order_impl<D>(t, q, nq, order, nullptr, s, nullptr, qroot);
  if (st == CKD_OK) {
    const int nw = std::min(4, knn_warps_per_block());
    const unsigned blocks = (unsigned)cdiv(cdiv(nq, 32), nw);
    size_t sm = (size_t)nw * compact_heap_bytes(k);
    const int bps = knn_blocks_per_sm();
    if (bps > 0) sm = std::max(sm, (size_t)(200 * 1024) / bps);
    cudaError_t e = cudaFuncSetAttribute(k_knn_lane2<D, PER>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) {
      dev_free(order, s);
      return cuda_fail(e, "cudaFuncSetAttribute(k_knn_lane2)");
    }
    timing_begin(s);
    k_knn_lane2<D, PER><<<blocks, nw * 32, sm, s>>>(t->view(), q, order, nq, k, sorted, dist, idx,
                                                    knn_stats_buffer(), nullptr, nullptr, nullptr,
                                                    nullptr, qroot);
    note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) st = cuda_fail(e, "k_knn_lane (forest)");
    else timing_end(s);
  }
  dev_free(order, s);
  return st;
}

}  // namespace

ckd_status forest_knn(const ckd_tree* t, const double* q, const int32_t* qroot, int64_t nq, int k,
                      int sorted, double* dist, int64_t* idx, cudaStream_t s) {
  if (!(t->screen_ok && t->depth < kLaneStack - 1 && k <= kSmemK))
    return fail(CKD_ERR_BAD_ARG,
                "forest kNN needs k <= 64, trees shallower than 127 levels and coordinates "
                "below 1e18");
  switch (t->d * 2 + (t->periodic ? 1 : 0)) {
#define CKD_FK(DD)                                                                        \
  case 2 * DD: return forest_knn_impl<DD, false>(t, q, qroot, nq, k, sorted, dist, idx, s); \
  case 2 * DD + 1: return forest_knn_impl<DD, true>(t, q, qroot, nq, k, sorted, dist, idx, s);
    CKD_FK(1) CKD_FK(2) CKD_FK(3) CKD_FK(4) CKD_FK(5) CKD_FK(6) CKD_FK(7) CKD_FK(8)
#undef CKD_FK
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

// ===================================================================
// kNN with the learned bound (ckd_knn_learned)
//
// locate + order the queries, predict each query's squared k-th distance
// (k_mlp_radius), run the bounded per-lane search, then rerun the queries it
// could not settle with the plain search.  The bounded kernel needs the FP32
// screen, k <= kSmemK and a stack deep enough for the tree; otherwise every query
// takes the plain path.
namespace {

template <int D, bool PER>
ckd_status knn_learned_impl(const ckd_tree* t, const ckd_mlp* net, const double* q, int64_t nq,
                            int k, int sorted, double* dist, int64_t* idx, int64_t* nfb_out,
                            cudaStream_t s) {
  int32_t *order = nullptr, *qleaf = nullptr, *miss = nullptr;
  double* r2 = nullptr;
  unsigned* nmiss = nullptr;
  CKD_CUDA(dev_alloc((void**)&order, sizeof(int32_t) * nq, s));
  CKD_CUDA(dev_alloc((void**)&qleaf, sizeof(int32_t) * nq, s));
  CKD_CUDA(dev_alloc((void**)&r2, sizeof(double) * nq, s));
  CKD_CUDA(dev_alloc((void**)&miss, sizeof(int32_t) * nq, s));
  CKD_CUDA(dev_alloc((void**)&nmiss, sizeof(unsigned), s));
  CKD_CUDA(cudaMemsetAsync(nmiss, 0, sizeof(unsigned), s));
  ckd_status st = order_impl<D>(t, q, nq, order, qleaf, s);
  if (st == CKD_OK) {
    timing_begin(s);
    st = mlp_radius(t, net, q, order, qleaf, nq, k, r2, s);
  }
  if (st == CKD_OK && (learned_kernel() == 0 || learned_kernel() == 3)) {
    const int nw = std::min(4, knn_warps_per_block());
    const unsigned blocks = (unsigned)cdiv(cdiv(nq, 32), nw);
    size_t sm = (size_t)nw * compact_heap_bytes(k);
    const int bps = knn_blocks_per_sm();
    if (bps > 0) sm = std::max(sm, (size_t)(200 * 1024) / bps);
    const bool pair = learned_kernel() == 3;
    cudaError_t e = pair ? cudaFuncSetAttribute(k_knn_lane2<D, PER, true, true>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)
                         : cudaFuncSetAttribute(k_knn_lane2<D, PER, true>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_knn_lane2)");
    if (pair)
      k_knn_lane2<D, PER, true, true><<<blocks, nw * 32, sm, s>>>(
          t->view(), q, order, nq, k, sorted, dist, idx, knn_stats_buffer(), r2, miss, nmiss, qleaf);
    else
      k_knn_lane2<D, PER, true><<<blocks, nw * 32, sm, s>>>(t->view(), q, order, nq, k, sorted,
                                                            dist, idx, knn_stats_buffer(), r2,
                                                            miss, nmiss, qleaf);
    note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) st = cuda_fail(e, "k_knn_lane2 (bounded)");
  } else if (st == CKD_OK && learned_kernel() == 2) {
    const int nw = knn_warps_per_block();
    const unsigned blocks = (unsigned)cdiv(cdiv(nq, 32), nw);
    size_t sm = (size_t)nw * heap_stride(k) * 32 * (sizeof(unsigned long long) + sizeof(int32_t));
    const int bps = knn_blocks_per_sm();
    if (bps > 0) sm = std::max(sm, (size_t)(200 * 1024) / bps);
    cudaError_t e = cudaFuncSetAttribute(k_knn_lane<D, PER, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_knn_lane)");
    k_knn_lane<D, PER, true><<<blocks, nw * 32, sm, s>>>(t->view(), q, order, nq, k, sorted, dist,
                                                         idx, knn_stats_buffer(), r2, miss, nmiss,
                                                         qleaf);
    note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) st = cuda_fail(e, "k_knn_lane (bounded)");
  } else if (st == CKD_OK) {
    const int nw = gather_warps_per_block();
    const unsigned blocks = (unsigned)cdiv(cdiv(nq, 32), nw);
    const size_t sm = (size_t)nw * gather_smem_per_warp(k);
    cudaError_t e = cudaFuncSetAttribute(k_knn_gather<D, PER>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_knn_gather)");
    k_knn_gather<D, PER><<<blocks, nw * 32, sm, s>>>(t->view(), q, order, nq, k, sorted, r2, dist,
                                                     idx, miss, nmiss, knn_stats_buffer());
    note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) st = cuda_fail(e, "k_knn_gather");
  }
  unsigned nm = 0;
  if (st == CKD_OK) {
    cudaError_t e = cudaMemcpyAsync(&nm, nmiss, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_fail(e, "reading the fallback count");
    else if ((int64_t)nm > nq) st = fail(CKD_ERR_CUDA, "internal error: fallback list overflow");
  }
  if (st == CKD_OK && nm > 0)
    st = knn_launch<D, PER>(t, q, miss, nullptr, (int64_t)nm, k, sorted, dist, idx, s, 7);
  if (st == CKD_OK) timing_end(s);
  if (nfb_out) *nfb_out = nm;
  for (void* p : {(void*)order, (void*)qleaf, (void*)r2, (void*)miss, (void*)nmiss}) dev_free(p, s);
  return st;
}

}  // namespace

ckd_status knn_learned(const ckd_tree* t, const ckd_mlp* net, const double* q, int64_t nq, int k,
                       int sorted, double* dist, int64_t* idx, int64_t* nfb, cudaStream_t s) {
  if (!(t->screen_ok && t->depth < kLaneStack - 1 && k <= kSmemK)) {
    if (nfb) *nfb = nq;
    return knn_run(t, q, nq, k, sorted, dist, idx, s);
  }
  switch (t->d * 2 + (t->periodic ? 1 : 0)) {
#define CKD_LB(DD)                                                                          \
  case 2 * DD: return knn_learned_impl<DD, false>(t, net, q, nq, k, sorted, dist, idx, nfb, s); \
  case 2 * DD + 1: return knn_learned_impl<DD, true>(t, net, q, nq, k, sorted, dist, idx, nfb, s);
    CKD_LB(1) CKD_LB(2) CKD_LB(3) CKD_LB(4) CKD_LB(5) CKD_LB(6) CKD_LB(7) CKD_LB(8)
#undef CKD_LB
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

// ===================================================================
// kNN without any device allocation (ckd_knn_noalloc)
//
// For callers that cannot allocate device memory during a search: host
// applications that reserve all device memory up front and hand nothing to the
// CUDA allocator afterwards, or latency-critical loops that cannot afford the
// implicit synchronisation of an allocation.  The query-ordering scratch of the
// search (per-query keys and the processing order, a histogram of coarse leaf
// bins and its prefix sums) lives in one file-scope device array instead of
// pool allocations; the search kernel itself needs only shared memory.
//
// Limits: at most kNoAllocMaxQ queries per call, k <= 64, tree depth < 92.
// Every call shares the array, so calls whose work overlaps on the GPU (two
// streams, or two host threads) race on it and must be serialised by the
// caller.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current); make that first call
// before any stream capture.  The array holds ~18 MB on every device that
// loads the library, until the process exits.
namespace {

constexpr int64_t kNoAllocMaxQ = int64_t(1) << 21;  // queries per call
constexpr int kNoAllocBins = 1 << 18;              // coarse leaf bins
constexpr size_t kNoAllocBytes =
    sizeof(int32_t) * (2 * (size_t)kNoAllocMaxQ + 2 * (size_t)kNoAllocBins + 64);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};

// host address of the scratch array on the current device (set up once per device)
ckd_status noalloc_scratch(void** out) {
  int dev = 0;
  CKD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(CKD_ERR_NO_DEVICE, "device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return CKD_OK;
}

// leaf of each query, binned coarsely by the leaf's first point
template <int D>
__global__ void k_locate_bins(const NodeMeta* __restrict__ meta, const double* __restrict__ Q,
                              int64_t nq, int shift, int32_t* __restrict__ key,
                              int32_t* __restrict__ hist) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  double q[D];
#pragma unroll
  for (int j = 0; j < D; ++j) q[j] = Q[i * D + j];
  NodeMeta m = load_meta(meta, 0);
  while (m.left >= 0) {
    double qa = 0.0;
#pragma unroll
    for (int j = 0; j < D; ++j)
      if (j == m.axis) qa = q[j];
    m = load_meta(meta, qa < m.split ? m.left : m.left + 1);
  }
  int32_t b = m.start >> shift;
  key[i] = b;
  atomicAdd(&hist[b], 1);
}

// exclusive scan of n <= kNoAllocBins counts by one block (out[n] = total)
__global__ void __launch_bounds__(1024) k_scan_one_block(const int32_t* __restrict__ in, int n,
                                                         int32_t* __restrict__ out) {
  __shared__ int32_t tmp[32];
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per, b1 = min(n, b0 + per);
  int32_t s = 0;
  for (int i = b0; i < b1; ++i) s += in[i];
  int32_t tot;
  int32_t pre = block_exclusive_scan<int32_t, 1024>(s, tmp, tot);
  for (int i = b0; i < b1; ++i) {
    int32_t v = in[i];
    out[i] = pre;
    pre += v;
  }
  if (threadIdx.x == 0) out[n] = tot;
}

template <int D, bool PER>
ckd_status knn_noalloc_impl(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted,
                            double* dist, int64_t* idx, cudaStream_t s) {
  void* base = nullptr;
  CKD_TRY(noalloc_scratch(&base));
  int32_t* order = reinterpret_cast<int32_t*>(base);
  int32_t* key = order + kNoAllocMaxQ;
  int32_t* hist = key + kNoAllocMaxQ;
  int32_t* off = hist + kNoAllocBins;
  int shift = 0;
  while ((t->n >> shift) >= kNoAllocBins) ++shift;
  const int nbins = (int)((t->n >> shift) + 1);
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * nbins, s));
  const unsigned g = (unsigned)cdiv(nq, 256);
  k_locate_bins<D><<<g, 256, 0, s>>>(t->meta, q, nq, shift, key, hist);
  CKD_LAUNCH_CHECK();
  k_scan_one_block<<<1, 1024, 0, s>>>(hist, nbins, off);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * nbins, s));
  k_bucket_scatter<<<g, 256, 0, s>>>(key, nq, off, hist, order);
  CKD_LAUNCH_CHECK();
  TreeView tv = t->view();
  const int nw = 4;
  const unsigned blocks = (unsigned)cdiv(cdiv(nq, 32), nw);
  if (t->screen_ok && t->depth < kLaneStack - 1) {
    size_t sm = (size_t)nw * compact_heap_bytes(k);
    CKD_CUDA(cudaFuncSetAttribute(k_knn_lane2<D, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm));
    k_knn_lane2<D, PER><<<blocks, nw * 32, sm, s>>>(tv, q, order, nq, k, sorted, dist, idx,
                                                    nullptr);
  } else {
    size_t sm = (size_t)nw * k * 32 * (sizeof(double) + sizeof(int32_t)) +
                (size_t)nw * kStack * sizeof(int32_t);
    CKD_CUDA(cudaFuncSetAttribute(k_knn_smem<D, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm));
    k_knn_smem<D, PER><<<blocks, nw * 32, sm, s>>>(tv, q, order, nq, k, sorted, nullptr, kStack,
                                                   dist, idx);
  }
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

}  // namespace

ckd_status knn_noalloc(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted,
                       double* dist, int64_t* idx, cudaStream_t s) {
  if (nq > kNoAllocMaxQ)
    return fail(CKD_ERR_BAD_ARG, "ckd_knn_noalloc: at most 2097152 queries per call");
  if (k > kSmemK) return fail(CKD_ERR_BAD_ARG, "ckd_knn_noalloc: k must be <= 64");
  if (t->depth >= kStack - 4)
    return fail(CKD_ERR_BAD_ARG, "ckd_knn_noalloc: tree deeper than 91 levels");
  switch (t->d * 2 + (t->periodic ? 1 : 0)) {
#define CKD_NA(DD)                                                                     \
  case 2 * DD: return knn_noalloc_impl<DD, false>(t, q, nq, k, sorted, dist, idx, s); \
  case 2 * DD + 1: return knn_noalloc_impl<DD, true>(t, q, nq, k, sorted, dist, idx, s);
    CKD_NA(1) CKD_NA(2) CKD_NA(3) CKD_NA(4) CKD_NA(5) CKD_NA(6) CKD_NA(7) CKD_NA(8)
#undef CKD_NA
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

}  // namespace ckd
