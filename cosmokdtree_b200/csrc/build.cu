// build.cu -- level-synchronous sliding-midpoint k-d tree construction on one GPU.
//
// Restates the recursion of src/cosmokdtree.f90:286-451 breadth-first: every
// level processes all open nodes of all sizes at once.
//
//   k_seg_box     per-node bounding box of the open nodes (segmented min/max)
//   k_decide      axis (longest cell side, spread tie-break), midpoint, slide mode
//   k_argext      slide point = first position holding the extreme (atomicMin)
//   k_flags       left/right flag per position, per-tile sums, segment-end prefixes
//   scan          tile offsets
//   k_children    n_left per node, child pairs, child cells, next open list
//   k_scatter     stable out-of-place partition into the other buffer; points of
//                 new leaves also land in the final leaf-ordered arrays
//
// Points live in SoA ping-pong buffers X[2][d][n]; each position carries the id
// of the node whose segment holds it (NID).  A position is open at level L iff
// its node has depth L and more than `leaf` points, so stale NIDs of finished
// segments never need clearing.  The partition is stable, so every segment stays
// sorted by original index and "first occurrence" (Fortran minloc/maxloc,
// cosmokdtree.f90:372-373) is the lowest index holding the extreme.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ckd_common.cuh"
#include "ckd_scan.cuh"

namespace ckd {

namespace {

constexpr int kBT = 256;          // threads per tile kernel
constexpr int kItems = 8;         // passes per tile
constexpr int kTile = kBT * kItems;
constexpr int kMaxLevels = 8192;  // depth guard (degenerate duplicate clusters peel one point per level)

struct BuildBufs {
  int d = 0;
  int64_t n = 0;
  double* X[2] = {nullptr, nullptr};
  int32_t* I[2] = {nullptr, nullptr};
  int32_t* NID[2] = {nullptr, nullptr};
  // per node (capacity cap)
  int64_t cap = 0;
  NodeMeta* meta = nullptr;
  double* cell = nullptr;
  double* box = nullptr;
  unsigned long long* keys = nullptr;  // [cap][2d] ordered min/max keys
  int32_t* ext = nullptr;              // slide point position
  int32_t* mode = nullptr;             // 0 midpoint, 1 slide left, 2 slide right
  int32_t* pstart = nullptr;           // local exclusive prefix at segment start
  int32_t* pend = nullptr;             // local inclusive prefix at segment end
  int32_t* nleft = nullptr;
  int32_t* pbase = nullptr;
  // per level
  int32_t* act[2] = {nullptr, nullptr};
  int32_t* nxt_cnt = nullptr;
  int32_t* nxt_off = nullptr;
  int32_t* tile_sum = nullptr;
  int32_t* tile_off = nullptr;
  int32_t* scal = nullptr;  // device scalars: [0] next open count, [1] error flag
  // per tile of kTile positions: 1 if the tile holds a position of an open node
  // this level (the tile kernels return at once for the other tiles)
  unsigned char* tile_act = nullptr;
};

// ------------------------------------------------------------------ kernels

// row-major (n x d) FP64/FP32 -> SoA FP64.  Tree t of a forest owns positions
// [off[t], off[t+1]) and is rooted at node t; ids are local to their tree
// (0..n_t-1), NID[0] = the tree's root, NID[1] = -1.  off == nullptr: one tree.
template <typename T>
__global__ void k_init_points(const T* __restrict__ in, int64_t n, int d, double* __restrict__ X,
                              int32_t* __restrict__ I, int32_t* __restrict__ N0,
                              int32_t* __restrict__ N1, const int64_t* __restrict__ off,
                              int32_t n_trees) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  for (int j = 0; j < d; ++j) X[(int64_t)j * n + p] = (double)in[p * d + j];
  int32_t t = 0;
  if (off) {  // last tree with off[t] <= p
    int32_t lo = 0, hi = n_trees - 1;
    while (lo < hi) {
      int32_t mid = (lo + hi + 1) >> 1;
      if (off[mid] <= p) lo = mid;
      else hi = mid - 1;
    }
    t = lo;
  }
  I[p] = (int32_t)(p - (off ? off[t] : 0));
  N0[p] = t;
  N1[p] = -1;
}

__device__ __forceinline__ bool open_node(const NodeMeta* __restrict__ meta, int32_t a, int level,
                                          int leaf) {
  if (a < 0) return false;
  NodeMeta m = meta[a];
  return m.depth == level && m.count > leaf;
}

// tile_act[t] = 1 for every tile that a segment of an open node overlaps
__global__ void k_mark_tiles(const int32_t* __restrict__ act, int m,
                             const NodeMeta* __restrict__ meta,
                             unsigned char* __restrict__ tile_act) {
  const int i = blockIdx.x;
  if (i >= m) return;
  const NodeMeta nm = meta[act[i]];
  const int64_t t0 = nm.start / kTile, t1 = ((int64_t)nm.start + nm.count - 1) / kTile;
  for (int64_t t = t0 + threadIdx.x; t <= t1; t += blockDim.x) tile_act[t] = 1;
}

// Segmented min/max over open positions; one atomicMin/atomicMax per segment
// piece that crosses a warp-chunk boundary, direct atomics for pieces inside.
template <int D>
__global__ void __launch_bounds__(kBT) k_seg_box(const double* __restrict__ X,
                                                 const int32_t* __restrict__ NID,
                                                 const NodeMeta* __restrict__ meta, int level,
                                                 int leaf, int64_t n,
                                                 unsigned long long* __restrict__ keys,
                                                 const unsigned char* __restrict__ tile_act) {
  if (tile_act && !tile_act[blockIdx.x]) return;
  constexpr int W = kBT / 32;
  __shared__ int32_t rec_id[kItems * W][2];
  __shared__ unsigned long long rec_v[kItems * W][2][2 * D];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kTile;
  for (int it = 0; it < kItems; ++it) {
    int64_t p = base + (int64_t)it * kBT + threadIdx.x;
    int32_t a = -1;
    if (p < n) {
      a = NID[p];
      if (!open_node(meta, a, level, leaf)) a = -1;
    }
    unsigned long long mn[D], mx[D];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      unsigned long long k = a >= 0 ? dkey(X[(int64_t)j * n + p]) : 0ull;
      mn[j] = k;
      mx[j] = k;
    }
    // segmented inclusive scan (runs of equal `a` are contiguous)
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int32_t au = __shfl_up_sync(0xffffffffu, a, o);
      bool take = lane >= o && au == a;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        unsigned long long u = __shfl_up_sync(0xffffffffu, mn[j], o);
        unsigned long long v = __shfl_up_sync(0xffffffffu, mx[j], o);
        if (take) {
          mn[j] = u < mn[j] ? u : mn[j];
          mx[j] = v > mx[j] ? v : mx[j];
        }
      }
    }
    int32_t a_next = __shfl_down_sync(0xffffffffu, a, 1);
    int32_t a0 = __shfl_sync(0xffffffffu, a, 0);
    bool tail = (lane == 31) || (a_next != a);
    bool first_run = (a == a0);
    bool last_run = (a == __shfl_sync(0xffffffffu, a, 31));
    int chunk = it * W + w;
    if (tail && a >= 0 && !first_run && !last_run) {
#pragma unroll
      for (int j = 0; j < D; ++j) {
        atomicMin(&keys[(int64_t)a * 2 * D + 2 * j], mn[j]);
        atomicMax(&keys[(int64_t)a * 2 * D + 2 * j + 1], mx[j]);
      }
    }
    if (tail && first_run) {
      rec_id[chunk][0] = a;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        rec_v[chunk][0][2 * j] = mn[j];
        rec_v[chunk][0][2 * j + 1] = mx[j];
      }
    }
    if (lane == 31) {
      // the last run; equal to the first run when the whole warp is one run
      rec_id[chunk][1] = first_run ? -2 : a;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        rec_v[chunk][1][2 * j] = mn[j];
        rec_v[chunk][1][2 * j + 1] = mx[j];
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t cur = -1;
    unsigned long long v[2 * D];
    auto flush = [&]() {
      if (cur >= 0) {
#pragma unroll
        for (int j = 0; j < D; ++j) {
          atomicMin(&keys[(int64_t)cur * 2 * D + 2 * j], v[2 * j]);
          atomicMax(&keys[(int64_t)cur * 2 * D + 2 * j + 1], v[2 * j + 1]);
        }
      }
    };
    for (int c = 0; c < kItems * W; ++c) {
      for (int r = 0; r < 2; ++r) {
        int32_t id = rec_id[c][r];
        if (id == -2) continue;  // no separate last run
        if (id == cur) {
#pragma unroll
          for (int j = 0; j < D; ++j) {
            v[2 * j] = rec_v[c][r][2 * j] < v[2 * j] ? rec_v[c][r][2 * j] : v[2 * j];
            v[2 * j + 1] = rec_v[c][r][2 * j + 1] > v[2 * j + 1] ? rec_v[c][r][2 * j + 1] : v[2 * j + 1];
          }
        } else {
          flush();
          cur = id;
#pragma unroll
          for (int j = 0; j < 2 * D; ++j) v[j] = rec_v[c][r][j];
        }
      }
    }
    flush();
  }
}

// Split decision per open node (cosmokdtree.f90:347-410).
template <int D>
__global__ void k_decide(const int32_t* __restrict__ act, int m, NodeMeta* __restrict__ meta,
                         double* __restrict__ cell, double* __restrict__ box,
                         const unsigned long long* __restrict__ keys, int32_t* __restrict__ mode,
                         int32_t* __restrict__ ext) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int32_t a = act[i];
  double lo[D], hi[D], clo[D], chi[D];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    lo[j] = dkey_inv(keys[(int64_t)a * 2 * D + 2 * j]);
    hi[j] = dkey_inv(keys[(int64_t)a * 2 * D + 2 * j + 1]);
    box[(int64_t)a * 2 * D + 2 * j] = lo[j];
    box[(int64_t)a * 2 * D + 2 * j + 1] = hi[j];
  }
#pragma unroll
  for (int j = 0; j < D; ++j) {
    clo[j] = cell[(int64_t)a * 2 * D + 2 * j];
    chi[j] = cell[(int64_t)a * 2 * D + 2 * j + 1];
  }
  // longest cell side; exact ties go to the larger data spread (:355-365)
  double maxside = dsub(chi[0], clo[0]);
  int axis = 0;
#pragma unroll
  for (int j = 1; j < D; ++j) {
    double side = dsub(chi[j], clo[j]);
    if (side > maxside) {
      maxside = side;
      axis = j;
    }
    if (side == maxside && dsub(hi[j], lo[j]) > dsub(hi[axis], lo[axis])) axis = j;
  }
  double cl = 0.0, ch = 0.0, minx = 0.0, maxx = 0.0;
#pragma unroll
  for (int j = 0; j < D; ++j)
    if (j == axis) {
      cl = clo[j];
      ch = chi[j];
      minx = lo[j];
      maxx = hi[j];
    }
  double mid = dmul(0.5, dadd(cl, ch));  // :367
  int md = 0;
  if (minx >= mid) {  // :376
    mid = minx;
    md = 1;
  } else if (maxx < mid) {  // :391
    mid = maxx;
    md = 2;
  }
  meta[a].split = mid;
  meta[a].axis = axis;
  mode[a] = md;
  ext[a] = 0x7fffffff;
}

// first position of a sliding segment that holds the extreme value
__global__ void k_argext(const double* __restrict__ X, const int32_t* __restrict__ NID,
                         const NodeMeta* __restrict__ meta, const int32_t* __restrict__ mode,
                         int level, int leaf, int64_t n, int32_t* __restrict__ ext,
                         const unsigned char* __restrict__ tile_act) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (!tile_act[p / kTile]) return;
  int32_t a = NID[p];
  if (!open_node(meta, a, level, leaf)) return;
  if (mode[a] == 0) return;
  NodeMeta m = meta[a];
  if (X[(int64_t)m.axis * n + p] == m.split) atomicMin(&ext[a], (int32_t)p);
}

__device__ __forceinline__ int flag_of(const double* __restrict__ X, int64_t n, int64_t p,
                                       const NodeMeta& m, int md, int32_t ext) {
  if (md == 0) return X[(int64_t)m.axis * n + p] < m.split ? 1 : 0;  // :470
  if (md == 1) return p == ext ? 1 : 0;                               // :376-388
  return p != ext ? 1 : 0;                                            // :391-403
}

// per-tile left counts and the segment-start / segment-end local prefixes
__global__ void __launch_bounds__(kBT) k_flags(const double* __restrict__ X,
                                               const int32_t* __restrict__ NID,
                                               const NodeMeta* __restrict__ meta,
                                               const int32_t* __restrict__ mode,
                                               const int32_t* __restrict__ ext, int level, int leaf,
                                               int64_t n, int32_t* __restrict__ tile_sum,
                                               int32_t* __restrict__ pstart,
                                               int32_t* __restrict__ pend,
                                               const unsigned char* __restrict__ tile_act) {
  __shared__ int32_t tmp[kBT / 32];
  if (!tile_act[blockIdx.x]) {
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = 0;
    return;
  }
  const int64_t base = (int64_t)blockIdx.x * kTile;
  int32_t run = 0;
  for (int it = 0; it < kItems; ++it) {
    int64_t p = base + (int64_t)it * kBT + threadIdx.x;
    int32_t a = p < n ? NID[p] : -1;
    int f = 0;
    NodeMeta m;
    if (open_node(meta, a, level, leaf)) {
      m = meta[a];
      f = flag_of(X, n, p, m, mode[a], ext[a]);
    } else {
      a = -1;
    }
    int32_t tot;
    int32_t ex = block_exclusive_scan<int32_t, kBT>(f, tmp, tot) + run;
    if (a >= 0) {
      if (p == m.start) pstart[a] = ex;
      if (p == (int64_t)m.start + m.count - 1) pend[a] = ex + f;
    }
    run += tot;
  }
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = run;
}

// n_left, child pairs and cells; counts the next open list (cosmokdtree.f90:412-448)
template <int D>
__global__ void k_children(const int32_t* __restrict__ act, int m, NodeMeta* __restrict__ meta,
                           double* __restrict__ cell, const int32_t* __restrict__ pstart,
                           const int32_t* __restrict__ pend, const int32_t* __restrict__ tile_off,
                           int32_t* __restrict__ nleft, int32_t* __restrict__ pbase,
                           unsigned long long* __restrict__ keys, int32_t first_child, int leaf,
                           int32_t* __restrict__ nxt_cnt, int32_t* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int32_t a = act[i];
  NodeMeta pm = meta[a];
  int64_t s = pm.start, e = (int64_t)pm.start + pm.count - 1;
  int32_t P0 = tile_off[s / kTile] + pstart[a];
  int32_t P1 = tile_off[e / kTile] + pend[a];
  int32_t nl = P1 - P0;
  if (nl <= 0 || nl >= pm.count) {  // cannot happen for a valid sliding-midpoint split
    atomicExch(err, 1);
    nl = nl <= 0 ? 1 : pm.count - 1;
  }
  nleft[a] = nl;
  pbase[a] = P0;
  int32_t c0 = first_child + 2 * i;
  meta[a].left = c0;
  int cnt = 0;
  for (int side = 0; side < 2; ++side) {
    int32_t c = c0 + side;
    NodeMeta cm;
    cm.split = 0.0;
    cm.left = -1;
    cm.axis = -1;
    cm.start = side == 0 ? pm.start : pm.start + nl;
    cm.count = side == 0 ? nl : pm.count - nl;
    cm.depth = pm.depth + 1;
    cm.parent = a;
    meta[c] = cm;
#pragma unroll
    for (int j = 0; j < D; ++j) {  // :419-422
      double lo = cell[(int64_t)a * 2 * D + 2 * j], hi = cell[(int64_t)a * 2 * D + 2 * j + 1];
      if (j == pm.axis) {
        if (side == 0) hi = pm.split;
        else lo = pm.split;
      }
      cell[(int64_t)c * 2 * D + 2 * j] = lo;
      cell[(int64_t)c * 2 * D + 2 * j + 1] = hi;
      keys[(int64_t)c * 2 * D + 2 * j] = ~0ull;
      keys[(int64_t)c * 2 * D + 2 * j + 1] = 0ull;
    }
    if (cm.count > leaf) ++cnt;
  }
  nxt_cnt[i] = cnt;
}

__global__ void k_next_list(const int32_t* __restrict__ act, int m,
                            const NodeMeta* __restrict__ meta, const int32_t* __restrict__ nxt_off,
                            int leaf, int32_t* __restrict__ nxt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int32_t c0 = meta[act[i]].left;
  int32_t o = nxt_off[i];
  if (meta[c0].count > leaf) nxt[o++] = c0;
  if (meta[c0 + 1].count > leaf) nxt[o] = c0 + 1;
}

// stable partition of every open segment into the other buffer
template <int D>
__global__ void __launch_bounds__(kBT) k_scatter(
    const double* __restrict__ X, const int32_t* __restrict__ I, const int32_t* __restrict__ NID,
    const NodeMeta* __restrict__ meta, const int32_t* __restrict__ mode,
    const int32_t* __restrict__ ext, const int32_t* __restrict__ tile_off,
    const int32_t* __restrict__ nleft, const int32_t* __restrict__ pbase, int level, int leaf,
    int64_t n, double* __restrict__ Xo, int32_t* __restrict__ Io, int32_t* __restrict__ NIDo,
    double* __restrict__ Pf, int32_t* __restrict__ If, int32_t* __restrict__ err,
    const unsigned char* __restrict__ tile_act) {
  __shared__ int32_t tmp[kBT / 32];
  if (!tile_act[blockIdx.x]) return;
  const int64_t base = (int64_t)blockIdx.x * kTile;
  int32_t run = tile_off[blockIdx.x];
  for (int it = 0; it < kItems; ++it) {
    int64_t p = base + (int64_t)it * kBT + threadIdx.x;
    int32_t a = p < n ? NID[p] : -1;
    int f = 0;
    NodeMeta m;
    if (open_node(meta, a, level, leaf)) {
      m = meta[a];
      f = flag_of(X, n, p, m, mode[a], ext[a]);
    } else {
      a = -1;
    }
    int32_t tot;
    int32_t ex = block_exclusive_scan<int32_t, kBT>(f, tmp, tot) + run;
    run += tot;
    if (a < 0) continue;
    int32_t rl = ex - pbase[a];
    int32_t nl = nleft[a];
    int64_t dst = f ? (int64_t)m.start + rl : (int64_t)m.start + nl + ((p - m.start) - rl);
    if (dst < m.start || dst >= (int64_t)m.start + m.count) {  // never for a consistent scan
      atomicExch(err, 2);
      continue;
    }
    int32_t child = m.left + (f ? 0 : 1);
    int32_t ccount = f ? nl : m.count - nl;
    int32_t id = I[p];
    Io[dst] = id;
    NIDo[dst] = child;
    bool is_leaf = ccount <= leaf;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double v = X[(int64_t)j * n + p];
      Xo[(int64_t)j * n + dst] = v;
      if (is_leaf) Pf[(int64_t)j * n + dst] = v;
    }
    if (is_leaf) If[dst] = id;
  }
}

// bounding boxes of the leaves from the final leaf-ordered points
template <int D>
__global__ void k_leaf_box(const NodeMeta* __restrict__ meta, int32_t n_nodes, int leaf,
                           const double* __restrict__ Pf, int64_t n, double* __restrict__ box) {
  int32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_nodes) return;
  NodeMeta m = meta[a];
  if (m.count > leaf) return;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double lo = Pf[(int64_t)j * n + m.start], hi = lo;
    for (int i = 1; i < m.count; ++i) {
      double v = Pf[(int64_t)j * n + m.start + i];
      lo = v < lo ? v : lo;
      hi = v > hi ? v : hi;
    }
    box[(int64_t)a * 2 * D + 2 * j] = lo;
    box[(int64_t)a * 2 * D + 2 * j + 1] = hi;
  }
}

// FP32 node boxes rounded outwards (lo down, hi up): every FP32 gap computed from
// them is a lower bound of the FP64 gap up to the screen's rounding slack.
template <int D>
__global__ void k_box32(const double* __restrict__ box, int32_t n_nodes, float* __restrict__ box32) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)n_nodes * 2 * D) return;
  double v = box[i];
  box32[i] = (i & 1) ? __double2float_ru(v) : __double2float_rd(v);
}

// FP64 points as packed records of (d + 3) / 4 double4s (zero padded)
template <int D>
__global__ void k_pts64(const double* __restrict__ Pf, int64_t n, double4* __restrict__ P64) {
  constexpr int NV = (D + 3) / 4;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  double v[4 * NV];
#pragma unroll
  for (int j = 0; j < 4 * NV; ++j) v[j] = j < D ? Pf[(int64_t)(j < D ? j : 0) * n + p] : 0.0;
#pragma unroll
  for (int h = 0; h < NV; ++h)
    P64[p * NV + h] = make_double4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
}

// Each point relative to its leaf's box centre, rounded to FP32, packed in float4s.
template <int D>
__global__ void k_pts32(const NodeMeta* __restrict__ meta, int32_t n_nodes, int leaf,
                        const double* __restrict__ box, const double* __restrict__ Pf, int64_t n,
                        float4* __restrict__ P32) {
  constexpr int NV = (D + 3) / 4;
  int32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_nodes) return;
  NodeMeta m = meta[a];
  if (m.left >= 0) return;
  double c[D];
#pragma unroll
  for (int j = 0; j < D; ++j)
    c[j] = leaf_centre(box[(int64_t)a * 2 * D + 2 * j], box[(int64_t)a * 2 * D + 2 * j + 1]);
  for (int i = 0; i < m.count; ++i) {
    int64_t p = (int64_t)m.start + i;
    float v[4 * NV];
#pragma unroll
    for (int j = 0; j < 4 * NV; ++j)
      v[j] = j < D ? __double2float_rn(__dsub_rn(Pf[(int64_t)j * n + p], c[j < D ? j : 0])) : 0.0f;
#pragma unroll
    for (int h = 0; h < NV; ++h)
      P32[p * NV + h] = make_float4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
  }
}

// Bottom-up search records: inward-rounded FP32 cells, FP64 leaf centres, and for
// each internal node the child-pair record (both children's outward FP32 boxes,
// ids and leaf flags) so one load serves a whole expansion.
template <int D>
__global__ void k_search_records(const NodeMeta* __restrict__ meta, int32_t n_nodes,
                                 const double* __restrict__ box, const double* __restrict__ cell,
                                 float4* __restrict__ pair, float* __restrict__ cell32,
                                 double* __restrict__ centre) {
  constexpr int NV = (D + 3) / 4;
  constexpr int PF = 4 * NV + 1;
  int32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_nodes) return;
  NodeMeta m = meta[a];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    cell32[(int64_t)a * 2 * D + 2 * j] = __double2float_ru(cell[(int64_t)a * 2 * D + 2 * j]);
    cell32[(int64_t)a * 2 * D + 2 * j + 1] = __double2float_rd(cell[(int64_t)a * 2 * D + 2 * j + 1]);
  }
  if (m.left < 0) {
#pragma unroll
    for (int j = 0; j < D; ++j)
      centre[(int64_t)a * D + j] =
          leaf_centre(box[(int64_t)a * 2 * D + 2 * j], box[(int64_t)a * 2 * D + 2 * j + 1]);
    return;
  }
  float4* rec = pair + (int64_t)a * PF;
  for (int side = 0; side < 2; ++side) {
    int32_t c = m.left + side;
    float lo[4 * NV], hi[4 * NV];
#pragma unroll
    for (int j = 0; j < 4 * NV; ++j) {
      lo[j] = j < D ? __double2float_rd(box[(int64_t)c * 2 * D + 2 * (j < D ? j : 0)]) : 0.0f;
      hi[j] = j < D ? __double2float_ru(box[(int64_t)c * 2 * D + 2 * (j < D ? j : 0) + 1]) : 0.0f;
    }
#pragma unroll
    for (int h = 0; h < NV; ++h) {
      rec[side * 2 * NV + h] = make_float4(lo[4 * h], lo[4 * h + 1], lo[4 * h + 2], lo[4 * h + 3]);
      rec[side * 2 * NV + NV + h] =
          make_float4(hi[4 * h], hi[4 * h + 1], hi[4 * h + 2], hi[4 * h + 3]);
    }
  }
  int4 info = make_int4(m.left, m.left + 1, meta[m.left].left < 0 ? 1 : 0,
                        meta[m.left + 1].left < 0 ? 1 : 0);
  rec[4 * NV] = *reinterpret_cast<float4*>(&info);
}

// roots: node t = root of tree t (positions off[t] .. off[t+1]-1)
template <int D>
__global__ void k_root_init(NodeMeta* meta, double* cell, unsigned long long* keys,
                            const int64_t* __restrict__ off, int32_t n_trees, const double* L,
                            int periodic) {
  int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_trees) return;
  NodeMeta m;
  m.split = 0.0;
  m.left = -1;
  m.axis = -1;
  m.start = (int32_t)off[t];
  m.count = (int32_t)(off[t + 1] - off[t]);
  m.depth = 0;
  m.parent = -1;
  meta[t] = m;
  for (int j = 0; j < D; ++j) {
    cell[(int64_t)t * 2 * D + 2 * j] = periodic ? -L[j] / 2. : 0.0;  // :218-224 (every axis)
    cell[(int64_t)t * 2 * D + 2 * j + 1] = periodic ? L[j] / 2. : 0.0;
    keys[(int64_t)t * 2 * D + 2 * j] = ~0ull;
    keys[(int64_t)t * 2 * D + 2 * j + 1] = 0ull;
  }
}

// non-periodic root cells = the data bounding box of each tree (:226-229)
template <int D>
__global__ void k_root_cells(double* cell, const unsigned long long* __restrict__ keys,
                             int32_t n_trees) {
  int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_trees) return;
  for (int j = 0; j < 2 * D; ++j) cell[(int64_t)t * 2 * D + j] = dkey_inv(keys[(int64_t)t * 2 * D + j]);
}

// ------------------------------------------------------------------ host side

template <typename T>
cudaError_t grow(T** p, int64_t old_n, int64_t new_n, cudaStream_t s) {
  T* q = nullptr;
  cudaError_t e = dev_alloc((void**)&q, sizeof(T) * new_n, s);
  if (e != cudaSuccess) return e;
  if (*p && old_n > 0) {
    e = cudaMemcpyAsync(q, *p, sizeof(T) * old_n, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    dev_free(*p, s);
  }
  *p = q;
  return cudaSuccess;
}

ckd_status ensure_node_cap(BuildBufs& B, int64_t need, cudaStream_t s) {
  if (need <= B.cap) return CKD_OK;
  int64_t nc = std::max<int64_t>(need, B.cap * 2);
  int d2 = 2 * B.d;
  CKD_CUDA(grow(&B.meta, B.cap, nc, s));
  CKD_CUDA(grow(&B.cell, B.cap * d2, nc * d2, s));
  CKD_CUDA(grow(&B.box, B.cap * d2, nc * d2, s));
  CKD_CUDA(grow(&B.keys, B.cap * d2, nc * d2, s));
  CKD_CUDA(grow(&B.ext, B.cap, nc, s));
  CKD_CUDA(grow(&B.mode, B.cap, nc, s));
  CKD_CUDA(grow(&B.pstart, B.cap, nc, s));
  CKD_CUDA(grow(&B.pend, B.cap, nc, s));
  CKD_CUDA(grow(&B.nleft, B.cap, nc, s));
  CKD_CUDA(grow(&B.pbase, B.cap, nc, s));
  B.cap = nc;
  return CKD_OK;
}

void free_bufs(BuildBufs& B, cudaStream_t s) {
  void* ps[] = {B.X[0],   B.X[1],    B.I[0],      B.I[1],     B.NID[0],  B.NID[1], B.meta,
                B.cell,   B.box,     B.keys,      B.ext,      B.mode,    B.pstart, B.pend,
                B.nleft,  B.pbase,   B.act[0],    B.act[1],   B.nxt_cnt, B.nxt_off, B.tile_sum,
                B.tile_off, B.scal, B.tile_act};
  for (void* p : ps)
    if (p) dev_free(p, s);
  B = BuildBufs();
}

template <int D>
ckd_status build_impl(ckd_tree* t, const void* pts_dev, int dtype, cudaStream_t s) {
  const int64_t n = t->n;
  const int leaf = t->leaf;
  BuildBufs B;
  B.d = D;
  B.n = n;
  struct Guard {
    BuildBufs* b;
    cudaStream_t s;
    ~Guard() { free_bufs(*b, s); }
  } guard{&B, s};

  const int64_t ntiles = cdiv(n, kTile);
  for (int b = 0; b < 2; ++b) {
    CKD_CUDA(dev_alloc((void**)&B.X[b], sizeof(double) * D * n, s));
    CKD_CUDA(dev_alloc((void**)&B.I[b], sizeof(int32_t) * n, s));
    CKD_CUDA(dev_alloc((void**)&B.NID[b], sizeof(int32_t) * n, s));
  }
  int64_t max_open = n / (leaf + 1) + 2 + t->n_trees;
  for (int b = 0; b < 2; ++b) CKD_CUDA(dev_alloc((void**)&B.act[b], sizeof(int32_t) * max_open, s));
  CKD_CUDA(dev_alloc((void**)&B.nxt_cnt, sizeof(int32_t) * max_open, s));
  CKD_CUDA(dev_alloc((void**)&B.nxt_off, sizeof(int32_t) * (max_open + 1), s));
  CKD_CUDA(dev_alloc((void**)&B.tile_sum, sizeof(int32_t) * ntiles, s));
  CKD_CUDA(dev_alloc((void**)&B.tile_off, sizeof(int32_t) * (ntiles + 1), s));
  CKD_CUDA(dev_alloc((void**)&B.scal, sizeof(int32_t) * 4, s));
  CKD_CUDA(dev_alloc((void**)&B.tile_act, (size_t)ntiles, s));
  CKD_CUDA(cudaMemsetAsync(B.scal, 0, sizeof(int32_t) * 4, s));

  // final outputs
  CKD_CUDA(cudaMalloc((void**)&t->pts, sizeof(double) * D * n));
  CKD_CUDA(cudaMalloc((void**)&t->ids, sizeof(int32_t) * n));

  // trees of a forest: positions off[t] .. off[t+1]-1, root node t
  const int32_t T = (int32_t)t->n_trees;
  const std::vector<int64_t>& off = t->tree_off;
  int64_t* off_dev = nullptr;
  CKD_CUDA(dev_alloc((void**)&off_dev, sizeof(int64_t) * (T + 1), s));
  CKD_CUDA(cudaMemcpyAsync(off_dev, off.data(), sizeof(int64_t) * (T + 1), cudaMemcpyHostToDevice, s));
  {
    unsigned g = (unsigned)cdiv(n, 256);
    const int64_t* offp = T > 1 ? off_dev : nullptr;
    if (dtype == CKD_F32)
      k_init_points<float><<<g, 256, 0, s>>>((const float*)pts_dev, n, D, B.X[0], B.I[0],
                                             B.NID[0], B.NID[1], offp, T);
    else
      k_init_points<double><<<g, 256, 0, s>>>((const double*)pts_dev, n, D, B.X[0], B.I[0],
                                              B.NID[0], B.NID[1], offp, T);
    CKD_LAUNCH_CHECK();
  }
  double* Ldev = nullptr;
  CKD_CUDA(dev_alloc((void**)&Ldev, sizeof(double) * CKD_MAX_D, s));
  CKD_CUDA(cudaMemcpyAsync(Ldev, t->L, sizeof(double) * CKD_MAX_D, cudaMemcpyHostToDevice, s));
  CKD_TRY(ensure_node_cap(B, (int64_t)T + std::max<int64_t>(64, 4 * (n / std::max(1, leaf)) + 64), s));
  k_root_init<D><<<(unsigned)cdiv(T, 128), 128, 0, s>>>(B.meta, B.cell, B.keys, off_dev, T, Ldev,
                                                        t->periodic);
  CKD_LAUNCH_CHECK();

  // Root bounding boxes: validation (finite, inside the periodic box) and the
  // non-periodic root cells.  Computed with the open-node reduction using a leaf
  // threshold of 0 so that every root is "open" here.
  k_seg_box<D><<<(unsigned)ntiles, kBT, 0, s>>>(B.X[0], B.NID[0], B.meta, 0, 0, n, B.keys,
                                                 nullptr);
  CKD_LAUNCH_CHECK();
  std::vector<unsigned long long> rk((size_t)T * 2 * D);
  CKD_CUDA(cudaMemcpyAsync(rk.data(), B.keys, sizeof(unsigned long long) * 2 * D * T,
                           cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaStreamSynchronize(s));
  double rlo[CKD_MAX_D], rhi[CKD_MAX_D];
  for (int j = 0; j < D; ++j) {
    rlo[j] = INFINITY;
    rhi[j] = -INFINITY;
  }
  for (int32_t tr = 0; tr < T; ++tr) {
    for (int j = 0; j < D; ++j) {
      auto inv = [](unsigned long long k) {
        unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
        double x;
        std::memcpy(&x, &b, 8);
        return x;
      };
      double lo = inv(rk[(size_t)tr * 2 * D + 2 * j]), hi = inv(rk[(size_t)tr * 2 * D + 2 * j + 1]);
      if (!std::isfinite(lo) || !std::isfinite(hi)) {
        dev_free(Ldev, s);
        dev_free(off_dev, s);
        return fail(CKD_ERR_BAD_ARG, "points contain NaN or infinite coordinates");
      }
      if (t->periodic && (lo < -t->L[j] / 2 || hi > t->L[j] / 2)) {
        dev_free(Ldev, s);
        dev_free(off_dev, s);
        return fail(CKD_ERR_OUT_OF_BOX, "Points outside (-L/2, L/2) range");
      }
      rlo[j] = std::min(rlo[j], lo);
      rhi[j] = std::max(rhi[j], hi);
    }
  }
  if (!t->periodic) {
    k_root_cells<D><<<(unsigned)cdiv(T, 128), 128, 0, s>>>(B.cell, B.keys, T);
    CKD_LAUNCH_CHECK();
  }
  // points of trees that are a single leaf never move: start from the input order
  CKD_CUDA(cudaMemcpyAsync(t->pts, B.X[0], sizeof(double) * D * n, cudaMemcpyDeviceToDevice, s));
  CKD_CUDA(cudaMemcpyAsync(t->ids, B.I[0], sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
  // open roots
  std::vector<int32_t> roots;
  for (int32_t tr = 0; tr < T; ++tr)
    if (off[tr + 1] - off[tr] > leaf) roots.push_back(tr);
  if (!roots.empty())
    CKD_CUDA(cudaMemcpyAsync(B.act[0], roots.data(), sizeof(int32_t) * roots.size(),
                             cudaMemcpyHostToDevice, s));
  CKD_CUDA(cudaStreamSynchronize(s));  // `roots` and `rk` are host buffers of the copies
  dev_free(off_dev, s);

  int32_t n_nodes = T;
  int m = (int)roots.size();
  int cur = 0;
  int level = 0;
  while (m > 0) {
    if (level >= kMaxLevels) {
      dev_free(Ldev, s);
      return fail(CKD_ERR_DEPTH, "tree depth exceeds the build's level cap (8192 levels)");
    }
    CKD_TRY(ensure_node_cap(B, (int64_t)n_nodes + 2 * (int64_t)m, s));
    const int32_t* act = B.act[cur];
    unsigned gm = (unsigned)cdiv(m, 128);
    CKD_CUDA(cudaMemsetAsync(B.tile_act, 0, (size_t)ntiles, s));
    k_mark_tiles<<<(unsigned)m, 128, 0, s>>>(act, m, B.meta, B.tile_act);
    CKD_LAUNCH_CHECK();
    if (level > 0) {
      k_seg_box<D><<<(unsigned)ntiles, kBT, 0, s>>>(B.X[cur], B.NID[cur], B.meta, level, leaf, n,
                                                    B.keys, B.tile_act);
      CKD_LAUNCH_CHECK();
    }
    k_decide<D><<<gm, 128, 0, s>>>(act, m, B.meta, B.cell, B.box, B.keys, B.mode, B.ext);
    CKD_LAUNCH_CHECK();
    k_argext<<<(unsigned)cdiv(n, 256), 256, 0, s>>>(B.X[cur], B.NID[cur], B.meta, B.mode, level,
                                                    leaf, n, B.ext, B.tile_act);
    CKD_LAUNCH_CHECK();
    k_flags<<<(unsigned)ntiles, kBT, 0, s>>>(B.X[cur], B.NID[cur], B.meta, B.mode, B.ext, level,
                                             leaf, n, B.tile_sum, B.pstart, B.pend, B.tile_act);
    CKD_LAUNCH_CHECK();
    CKD_TRY(scan_i32(B.tile_sum, B.tile_off, ntiles, s));
    k_children<D><<<gm, 128, 0, s>>>(act, m, B.meta, B.cell, B.pstart, B.pend, B.tile_off,
                                     B.nleft, B.pbase, B.keys, n_nodes, leaf, B.nxt_cnt,
                                     B.scal + 1);
    CKD_LAUNCH_CHECK();
    CKD_TRY(scan_i32(B.nxt_cnt, B.nxt_off, m, s));
    k_next_list<<<gm, 128, 0, s>>>(act, m, B.meta, B.nxt_off, leaf, B.act[1 - cur]);
    CKD_LAUNCH_CHECK();
    k_scatter<D><<<(unsigned)ntiles, kBT, 0, s>>>(
        B.X[cur], B.I[cur], B.NID[cur], B.meta, B.mode, B.ext, B.tile_off, B.nleft, B.pbase,
        level, leaf, n, B.X[1 - cur], B.I[1 - cur], B.NID[1 - cur], t->pts, t->ids, B.scal + 1,
        B.tile_act);
    CKD_LAUNCH_CHECK();
    int32_t nm = 0;
    CKD_CUDA(cudaMemcpyAsync(&nm, B.nxt_off + m, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CKD_CUDA(cudaStreamSynchronize(s));
    n_nodes += 2 * m;
    m = nm;
    cur = 1 - cur;
    ++level;
  }
  int32_t err = 0;
  CKD_CUDA(cudaMemcpyAsync(&err, B.scal + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  dev_free(Ldev, s);

  k_leaf_box<D><<<(unsigned)cdiv(n_nodes, 128), 128, 0, s>>>(B.meta, n_nodes, leaf, t->pts, n,
                                                             B.box);
  CKD_LAUNCH_CHECK();
  t->n_nodes = n_nodes;
  t->depth = level;
  CKD_CUDA(cudaMalloc((void**)&t->meta, sizeof(NodeMeta) * n_nodes));
  CKD_CUDA(cudaMalloc((void**)&t->box, sizeof(double) * 2 * D * n_nodes));
  CKD_CUDA(cudaMalloc((void**)&t->cell, sizeof(double) * 2 * D * n_nodes));
  CKD_CUDA(cudaMemcpyAsync(t->meta, B.meta, sizeof(NodeMeta) * n_nodes, cudaMemcpyDeviceToDevice, s));
  CKD_CUDA(cudaMemcpyAsync(t->box, B.box, sizeof(double) * 2 * D * n_nodes, cudaMemcpyDeviceToDevice, s));
  CKD_CUDA(cudaMemcpyAsync(t->cell, B.cell, sizeof(double) * 2 * D * n_nodes, cudaMemcpyDeviceToDevice, s));
  // FP32 screening copies.  The node-gap slack per axis is 2^-21 * (|q| + B) with
  // B bounding every stored coordinate (and the box side when periodic); the
  // screen is disabled for coordinates near the FP32 range.
  t->screen_ok = true;
  for (int j = 0; j < D; ++j) {
    double b = std::max(std::fabs(rlo[j]), std::fabs(rhi[j])) + (t->periodic ? t->L[j] : 0.0);
    if (!(b < 1e18)) t->screen_ok = false;
    t->slack[j] = (float)(b * (1.0 + 1e-6));
  }
  constexpr int NV = (D + 3) / 4;
  CKD_CUDA(cudaMalloc((void**)&t->box32, sizeof(float) * 2 * D * n_nodes));
  CKD_CUDA(cudaMalloc((void**)&t->pts32, sizeof(float4) * NV * n));
  CKD_CUDA(cudaMalloc((void**)&t->pts64, sizeof(double4) * NV * n));
  k_pts64<D><<<(unsigned)cdiv(n, 256), 256, 0, s>>>(t->pts, n, t->pts64);
  CKD_LAUNCH_CHECK();
  k_box32<D><<<(unsigned)cdiv((int64_t)n_nodes * 2 * D, 256), 256, 0, s>>>(t->box, n_nodes, t->box32);
  CKD_LAUNCH_CHECK();
  k_pts32<D><<<(unsigned)cdiv(n_nodes, 128), 128, 0, s>>>(t->meta, n_nodes, leaf, t->box, t->pts, n,
                                                          t->pts32);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(cudaMalloc((void**)&t->pair, sizeof(float4) * pair_f4(D) * n_nodes));
  CKD_CUDA(cudaMalloc((void**)&t->cell32, sizeof(float) * 2 * D * n_nodes));
  CKD_CUDA(cudaMalloc((void**)&t->centre, sizeof(double) * D * n_nodes));
  k_search_records<D><<<(unsigned)cdiv(n_nodes, 128), 128, 0, s>>>(
      t->meta, n_nodes, t->box, t->cell, t->pair, t->cell32, t->centre);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(cudaStreamSynchronize(s));
  if (err) return fail(CKD_ERR_CUDA, "internal error: inconsistent partition in build");
  // leaves = (nodes + 1) / 2 for each full binary tree
  t->n_leaves = (n_nodes + T) / 2;
  return CKD_OK;
}

}  // namespace

ckd_status build_dispatch(ckd_tree* t, const void* pts_dev, int dtype, cudaStream_t s) {
  switch (t->d) {
    case 1: return build_impl<1>(t, pts_dev, dtype, s);
    case 2: return build_impl<2>(t, pts_dev, dtype, s);
    case 3: return build_impl<3>(t, pts_dev, dtype, s);
    case 4: return build_impl<4>(t, pts_dev, dtype, s);
    case 5: return build_impl<5>(t, pts_dev, dtype, s);
    case 6: return build_impl<6>(t, pts_dev, dtype, s);
    case 7: return build_impl<7>(t, pts_dev, dtype, s);
    case 8: return build_impl<8>(t, pts_dev, dtype, s);
    default: return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
  }
}

}  // namespace ckd
