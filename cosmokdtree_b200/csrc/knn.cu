// knn.cu -- exact k-nearest-neighbour search (cosmokdtree.f90:504-905): query
// ordering, the per-lane and packet kernels, the kernel choice, forests, the
// learned-bound path and the allocation-free entry point.
//
// One query per lane.  Each lane keeps its k best (squared distance, id) in a
// max-heap (root = current k-th); a candidate enters iff it ranks strictly before
// the root under (d2, id) order, the canonical form of the strict test at
// cosmokdtree.f90:658.  The heap starts full of (HUGE(0.0), -1) sentinels
// (cosmokdtree.f90:517-518).  Distances are FP64, separately rounded, so results
// are bit-identical to the CPU restatement.
#include <algorithm>
#include <mutex>

#include "ckd_common.cuh"
#include "ckd_knn.cuh"
#include "ckd_knn_lane.cuh"
#include "ckd_mlp.cuh"
#include "ckd_scan.cuh"
#include "ckd_traverse.cuh"

namespace ckd {

namespace {

constexpr int kStack = 96;   // per-warp traversal stack of the packet kernel

// process-wide traversal statistics of the screened kernel (diagnostics)
__device__ unsigned long long g_knn_stats[8];
bool g_stats_on = false;
unsigned long long* knn_stats_buffer() {
  if (!g_stats_on) return nullptr;
  void* p = nullptr;
  cudaGetSymbolAddress(&p, g_knn_stats);
  return reinterpret_cast<unsigned long long*>(p);
}

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

// The per-lane kernel: one warp per 32 query slots (knn_lane_run).
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
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint2* Hw = reinterpret_cast<uint2*>(smem) + (size_t)w * 32 * (k + 1);
  const int64_t gw = (int64_t)blockIdx.x * nw + w;
  knn_lane_run<D, PER, BOUNDED, PAIR>(tv, Q, order, nq, k, sorted, dist, idx, stats, r2, miss,
                                      nmiss, qleaf, qroot, 0, Hw, lane, gw);
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

// Kernel choice (ckd_set_knn_variant): 0 automatic, 1 FP64 packet traversal,
// 7 per-lane compact heap, 8 the same expanding nodes from child-pair records.
// Automatic takes 8;
// trees too deep for its stack, coordinates beyond the FP32 screen's range and
// k > 64 take the packet kernel.
template <int D, bool PER>
ckd_status knn_launch(const ckd_tree* t, const double* q, const int32_t* order, int64_t nq, int k,
                      int sorted, double* dist, int64_t* idx, cudaStream_t s,
                      int force_variant = -1) {
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
  if (k <= kSmemK && t->screen_ok && var != 1 && t->depth < kLaneStack - 1) {
    const int nw7 = std::min(4, knn_warps_per_block());
    const unsigned blocks7 = (unsigned)cdiv(cdiv(nq, 32), nw7);
    size_t sm = (size_t)nw7 * compact_heap_bytes(k);
    const int bps = knn_blocks_per_sm();
    if (bps > 0) sm = std::max(sm, (size_t)(200 * 1024) / bps);
    if (var != 7) {
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
  struct Free {
    int32_t* p;
    cudaStream_t s;
    ~Free() {
      if (p) dev_free(p, s);
    }
  } free_guard{gstack, s};
  if (k <= kSmemK) {
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
  return CKD_OK;
}

template <int D>
ckd_status knn_dispatch_d(const ckd_tree* t, const double* q, const int32_t* order, int64_t nq,
                          int k, int sorted, double* dist, int64_t* idx, cudaStream_t s) {
  if (t->periodic) return knn_launch<D, true>(t, q, order, nq, k, sorted, dist, idx, s);
  return knn_launch<D, false>(t, q, order, nq, k, sorted, dist, idx, s);
}

template <int D>
ckd_status order_impl(const ckd_tree* t, const double* q, int64_t nq, int32_t* order,
                      int32_t* qleaf, cudaStream_t s, int32_t** off_out = nullptr,
                      const int32_t* qroot = nullptr) {
  int64_t n = t->n;
  Scratch sc(s);
  int32_t *key = nullptr, *hist = nullptr, *off = nullptr;
  CKD_CUDA(sc.alloc(&key, sizeof(int32_t) * nq));
  CKD_CUDA(sc.alloc(&hist, sizeof(int32_t) * n));
  CKD_CUDA(sc.alloc(&off, sizeof(int32_t) * (n + 1)));
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * n, s));
  unsigned g = (unsigned)cdiv(nq, 256);
  k_locate<D><<<g, 256, 0, s>>>(t->meta, q, nq, key, hist, qleaf, qroot);
  CKD_LAUNCH_CHECK();
  CKD_TRY(scan_i32(hist, off, n, s));
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * n, s));
  k_bucket_scatter<<<g, 256, 0, s>>>(key, nq, off, hist, order);
  CKD_LAUNCH_CHECK();
  if (off_out) {
    *off_out = off;
    sc.release(off);
  }
  return CKD_OK;
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
                       cudaStream_t s) {
  switch (t->d) {
#define CKD_QO(DD) \
  case DD: return order_impl<DD>(t, q, nq, order, nullptr, s);
    CKD_QO(1) CKD_QO(2) CKD_QO(3) CKD_QO(4) CKD_QO(5) CKD_QO(6) CKD_QO(7) CKD_QO(8)
#undef CKD_QO
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
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

ckd_status knn_ordered(const ckd_tree* t, const double* q, const int32_t* order, int64_t nq, int k,
                       int sorted, double* dist, int64_t* idx, cudaStream_t s) {
  switch (t->d) {
    case 1: return knn_dispatch_d<1>(t, q, order, nq, k, sorted, dist, idx, s);
    case 2: return knn_dispatch_d<2>(t, q, order, nq, k, sorted, dist, idx, s);
    case 3: return knn_dispatch_d<3>(t, q, order, nq, k, sorted, dist, idx, s);
    case 4: return knn_dispatch_d<4>(t, q, order, nq, k, sorted, dist, idx, s);
    case 5: return knn_dispatch_d<5>(t, q, order, nq, k, sorted, dist, idx, s);
    case 6: return knn_dispatch_d<6>(t, q, order, nq, k, sorted, dist, idx, s);
    case 7: return knn_dispatch_d<7>(t, q, order, nq, k, sorted, dist, idx, s);
    case 8: return knn_dispatch_d<8>(t, q, order, nq, k, sorted, dist, idx, s);
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

ckd_status knn_run(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted, double* dist,
                   int64_t* idx, cudaStream_t s) {
  Scratch sc(s);
  int32_t* order = nullptr;
  if (want_order(t, nq)) {
    CKD_CUDA(sc.alloc(&order, sizeof(int32_t) * nq));
    CKD_TRY(query_order(t, q, nq, order, s));
  }
  return knn_ordered(t, q, order, nq, k, sorted, dist, idx, s);
}

// ===================================================================
// kNN over a forest (ckd_forest_knn): every query carries its tree (qroot =
// the tree's root node); the queries of all trees are ordered by leaf and
// searched by one per-lane launch that starts each lane at its own root.
namespace {

template <int D, bool PER>
ckd_status forest_knn_impl(const ckd_tree* t, const double* q, const int32_t* qroot, int64_t nq,
                           int k, int sorted, double* dist, int64_t* idx, cudaStream_t s) {
  Scratch sc(s);
  int32_t* order = nullptr;
  CKD_CUDA(sc.alloc(&order, sizeof(int32_t) * nq));
  CKD_TRY(order_impl<D>(t, q, nq, order, nullptr, s, nullptr, qroot));
  timing_begin(s);
  const int nw = std::min(4, knn_warps_per_block());
  const unsigned blocks = (unsigned)cdiv(cdiv(nq, 32), nw);
  size_t sm = (size_t)nw * compact_heap_bytes(k);
  const int bps = knn_blocks_per_sm();
  if (bps > 0) sm = std::max(sm, (size_t)(200 * 1024) / bps);
  CKD_CUDA(cudaFuncSetAttribute(k_knn_lane2<D, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sm));
  k_knn_lane2<D, PER><<<blocks, nw * 32, sm, s>>>(t->view(), q, order, nq, k, sorted, dist, idx,
                                                  knn_stats_buffer(), nullptr, nullptr, nullptr,
                                                  nullptr, qroot);
  CKD_LAUNCH_CHECK();
  timing_end(s);
  return CKD_OK;
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
  Scratch sc(s);
  CKD_CUDA(sc.alloc(&order, sizeof(int32_t) * nq));
  CKD_CUDA(sc.alloc(&qleaf, sizeof(int32_t) * nq));
  CKD_CUDA(sc.alloc(&r2, sizeof(double) * nq));
  CKD_CUDA(sc.alloc(&miss, sizeof(int32_t) * nq));
  CKD_CUDA(sc.alloc(&nmiss, sizeof(unsigned)));
  CKD_CUDA(cudaMemsetAsync(nmiss, 0, sizeof(unsigned), s));
  ckd_status st = order_impl<D>(t, q, nq, order, qleaf, s);
  if (st == CKD_OK) {
    timing_begin(s);
    st = mlp_radius(t, net, q, order, qleaf, nq, k, r2, s);
  }
  if (st == CKD_OK) {
    const int nw = std::min(4, knn_warps_per_block());
    const unsigned blocks = (unsigned)cdiv(cdiv(nq, 32), nw);
    size_t sm = (size_t)nw * compact_heap_bytes(k);
    const int bps = knn_blocks_per_sm();
    if (bps > 0) sm = std::max(sm, (size_t)(200 * 1024) / bps);
    const bool pair = learned_kernel() != 0;
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
  }
  unsigned nm = 0;
  if (st == CKD_OK) {
    cudaError_t e = cudaMemcpyAsync(&nm, nmiss, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_fail(e, "reading the fallback count");
    else if ((int64_t)nm > nq) st = fail(CKD_ERR_CUDA, "internal error: fallback list overflow");
  }
  if (st == CKD_OK && nm > 0)
    st = knn_launch<D, PER>(t, q, miss, (int64_t)nm, k, sorted, dist, idx, s, 7);
  if (st == CKD_OK) timing_end(s);
  if (nfb_out) *nfb_out = nm;
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
// before any stream capture.  The lookup is repeated when the device's current
// context changed since (cudaDeviceReset, a caller-made context), so such a call
// should also come outside a capture.  The array holds ~18 MB on every device
// that loads the library, until the process exits.
namespace {

constexpr int64_t kNoAllocMaxQ = int64_t(1) << 21;  // queries per call
constexpr int kNoAllocBins = 1 << 18;              // coarse leaf bins
constexpr size_t kNoAllocBytes =
    sizeof(int32_t) * (2 * (size_t)kNoAllocMaxQ + 2 * (size_t)kNoAllocBins + 64);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};
void* g_noalloc_ctx[64] = {nullptr};

// the driver's current context (cuCtxGetCurrent, fetched through the runtime so
// the library needs no link against the driver library); null if unavailable
void* current_context() {
  using CtxFn = int (*)(void**);
  static CtxFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxFn>(f);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of the scratch array in the current device's context, looked up
// once per device and again whenever that device's current context is another
// one than at the last lookup (after cudaDeviceReset, or when the caller made a
// context of its own current): a context's module copy of the array has its own
// address.
ckd_status noalloc_scratch(void** out) {
  int dev = 0;
  CKD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(CKD_ERR_NO_DEVICE, "device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  void* ctx = current_context();
  if (!g_noalloc_ptr[dev] || !ctx || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
    g_noalloc_ptr[dev] = p;
    // cudaGetSymbolAddress made the primary context current if none was
    g_noalloc_ctx[dev] = ctx ? ctx : current_context();
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