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

#include "ckd_common.cuh"
#include "ckd_scan.cuh"
#include "ckd_traverse.cuh"

namespace ckd {

namespace {

constexpr int kStack = 96;   // per-warp traversal stack in shared memory
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

// ------------------------------------------------------------ query order
template <int D>
__global__ void k_locate(const NodeMeta* __restrict__ meta, const double* __restrict__ Q,
                         int64_t nq, int32_t* __restrict__ key, int32_t* __restrict__ hist) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  double q[D];
#pragma unroll
  for (int j = 0; j < D; ++j) q[j] = Q[i * D + j];
  int32_t node = 0;
  NodeMeta m = load_meta(meta, 0);
  while (m.left >= 0) {
    double qa = 0.0;
#pragma unroll
    for (int j = 0; j < D; ++j)
      if (j == m.axis) qa = q[j];
    node = qa < m.split ? m.left : m.left + 1;
    m = load_meta(meta, node);
  }
  key[i] = m.start;
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
ckd_status knn_launch(const ckd_tree* t, const double* q, const int32_t* order, int64_t nq, int k,
                      int sorted, double* dist, int64_t* idx, cudaStream_t s) {
  TreeView tv = t->view();
  const int threads = 128, nw = threads / 32;
  int64_t warps = cdiv(nq, 32);
  unsigned blocks = (unsigned)cdiv(warps, nw);
  int stack_len = std::max(kStack, t->depth + 4);
  int32_t* gstack = nullptr;
  bool use_gstack = stack_len > kStack || k > kSmemK;
  if (use_gstack)
    CKD_CUDA(dev_alloc((void**)&gstack, sizeof(int32_t) * stack_len * (int64_t)blocks * nw, s));
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
  if (gstack) CKD_CUDA(dev_free(gstack, s));
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
                      cudaStream_t s) {
  int64_t n = t->n;
  int32_t *key = nullptr, *hist = nullptr, *off = nullptr;
  CKD_CUDA(dev_alloc((void**)&key, sizeof(int32_t) * nq, s));
  CKD_CUDA(dev_alloc((void**)&hist, sizeof(int32_t) * n, s));
  CKD_CUDA(dev_alloc((void**)&off, sizeof(int32_t) * (n + 1), s));
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * n, s));
  unsigned g = (unsigned)cdiv(nq, 256);
  k_locate<D><<<g, 256, 0, s>>>(t->meta, q, nq, key, hist);
  CKD_LAUNCH_CHECK();
  CKD_TRY(scan_i32(hist, off, n, s));
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * n, s));
  k_bucket_scatter<<<g, 256, 0, s>>>(key, nq, off, hist, order);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(dev_free(key, s));
  CKD_CUDA(dev_free(hist, s));
  CKD_CUDA(dev_free(off, s));
  return CKD_OK;
}

}  // namespace

ckd_status query_order(const ckd_tree* t, const double* q, int64_t nq, int32_t* order,
                       cudaStream_t s) {
  switch (t->d) {
    case 1: return order_impl<1>(t, q, nq, order, s);
    case 2: return order_impl<2>(t, q, nq, order, s);
    case 3: return order_impl<3>(t, q, nq, order, s);
    case 4: return order_impl<4>(t, q, nq, order, s);
    case 5: return order_impl<5>(t, q, nq, order, s);
    case 6: return order_impl<6>(t, q, nq, order, s);
    case 7: return order_impl<7>(t, q, nq, order, s);
    case 8: return order_impl<8>(t, q, nq, order, s);
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

// Queries are ordered by leaf when there are enough of them to fill many warps.
bool want_order(const ckd_tree* t, int64_t nq) { return nq >= 4096 && nq * 8 >= t->n / 64; }

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
  int32_t* order = nullptr;
  if (want_order(t, nq)) {
    CKD_CUDA(dev_alloc((void**)&order, sizeof(int32_t) * nq, s));
    CKD_TRY(query_order(t, q, nq, order, s));
  }
  ckd_status st = knn_ordered(t, q, order, nq, k, sorted, dist, idx, s);
  if (order) dev_free(order, s);
  return st;
}

}  // namespace ckd
