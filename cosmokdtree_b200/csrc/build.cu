// build.cu -- level-synchronous sliding-midpoint k-d tree construction on one GPU.
//
// Restates the recursion of src/cosmokdtree.f90:286-451 breadth-first: every
// level processes all open nodes of all sizes at once.
//
//   k_seg_box     per-node bounding box of the open nodes (segmented min/max)
//   k_decide      axis (longest cell side, spread tie-break), midpoint, slide mode
//   k_flags       left flag per position of a midpoint split, per-tile sums and
//                 segment-end prefixes; slide point of a sliding split = first
//                 position holding the extreme (atomicMin)
//   scan          tile offsets
//   k_children    n_left per node, child pairs, child cells, next open list
//   k_scatter     stable out-of-place partition into the other buffer; points of
//                 new leaves also land in the final leaf-ordered arrays
//
// The working set of a level holds only the points of open nodes (more than
// `leaf` points), compacted into SoA ping-pong buffers X[2][d][n] (stride n):
// open node a owns working positions [wst[a], wst[a] + count), in the order of
// its final leaf-ordered range [start, start + count), and every position
// carries its node's id (NID).  A point whose child is a leaf goes straight to
// its final place in the leaf-ordered arrays and leaves the working set, so the
// per-level passes touch only the points still being split.  The partition is
// stable, so every segment stays sorted by original index and "first
// occurrence" (Fortran minloc/maxloc, cosmokdtree.f90:372-373) is the lowest
// index holding the extreme.
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

// What the flag pass needs of an open node, in one 32-byte record.
struct __align__(16) FlagRec {
  double split;
  int32_t axis, md, wst, count;
  int32_t pad[2];
};

// What the scatter needs of an open node, in two int4: {start, wst, nleft, count}
// and {pbase (midpoint split) or slide point, left child, working start of the
// left / right child or -1 for a leaf child, -2 for the slide point's leaf}.
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
  int32_t* wst = nullptr;              // first working position of an open node
  FlagRec* frec = nullptr;
  int4* srec = nullptr;                // [cap][2]
  // per level
  int32_t* act[2] = {nullptr, nullptr};
  // per open node: (open children << 32) | points of the open children, and
  // the exclusive prefix of that (next list slot, next working start)
  int64_t* nxt_cnt = nullptr;
  int64_t* nxt_off = nullptr;
  int32_t* tile_sum = nullptr;
  int32_t* tile_off = nullptr;
  unsigned* flags = nullptr;  // left flags of the working positions, one bit each
  int32_t* scal = nullptr;  // device scalars: [0] next open count, [1] error flag
  // level state {open nodes, working points, nodes so far, levels with open nodes},
  // double-buffered: a level reads lst[p] and its last node kernel writes lst[1-p]
  int4* lst = nullptr;
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

// Working set of the first level when some roots are already leaves: the points
// of the open roots, compacted in tree order (wst[t] = -1 for a leaf root).
template <int D>
__global__ void k_compact_roots(const double* __restrict__ X, const int32_t* __restrict__ I,
                                const int32_t* __restrict__ NID, const int32_t* __restrict__ wst,
                                const int64_t* __restrict__ off, int64_t n,
                                double* __restrict__ Xo, int32_t* __restrict__ Io,
                                int32_t* __restrict__ NIDo) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int32_t t = NID[p];
  const int32_t w0 = wst[t];
  if (w0 < 0) return;
  const int64_t w = w0 + (p - off[t]);
#pragma unroll
  for (int j = 0; j < D; ++j) Xo[(int64_t)j * n + w] = X[(int64_t)j * n + p];
  Io[w] = I[p];
  NIDo[w] = t;
}

// Segmented min/max over the working positions.  Each thread reduces kItems
// consecutive positions in registers; one segmented warp scan per dimension
// joins the pieces of runs that cross thread boundaries.  Runs that end
// inside a warp chunk go straight to atomicMin/atomicMax; the first and last
// run of every warp chunk are merged per block by thread 0.
template <int D>
__global__ void __launch_bounds__(kBT, 5) k_seg_box(const double* __restrict__ X,
                                                 const int32_t* __restrict__ NID,
                                                 int64_t n, int64_t nw,
                                                 unsigned long long* __restrict__ keys,
                                                 const int4* __restrict__ st = nullptr) {
  constexpr int W = kBT / 32;
  __shared__ int32_t rec_id[W][2];
  __shared__ unsigned long long rec_v[W][2][2 * D];
  if (st) nw = st->y;  // working points of this level (device state)
  if ((int64_t)blockIdx.x * kTile >= nw) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t p0 = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
  // node of every position (-1 past the working set), run breaks inside the thread
  static_assert(kItems == 8, "two int4 / four double2 loads per thread");
  int32_t a[kItems];
  // vector loads when the thread's 8 positions are all working positions and
  // aligned (NID from the pool; X rows start at j * n, even for even n)
  const bool full = p0 + kItems <= nw;
  const bool vec = full && (n & 1) == 0 && (reinterpret_cast<uintptr_t>(NID) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  if (vec) {
    const int4 u = __ldg(reinterpret_cast<const int4*>(NID + p0));
    const int4 v = __ldg(reinterpret_cast<const int4*>(NID + p0) + 1);
    a[0] = u.x, a[1] = u.y, a[2] = u.z, a[3] = u.w, a[4] = v.x, a[5] = v.y, a[6] = v.z, a[7] = v.w;
  } else {
#pragma unroll
    for (int i = 0; i < kItems; ++i) a[i] = p0 + i < nw ? NID[p0 + i] : -1;
  }
  unsigned brk = 0;
#pragma unroll
  for (int i = 1; i < kItems; ++i) brk |= (a[i] != a[i - 1]) ? (1u << i) : 0u;
  const int32_t hd = a[0], tl = a[kItems - 1];
  const bool single = brk == 0;
  // scan steps that stay inside the tail run (equal ids of open nodes are contiguous)
  unsigned take = 0;
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int32_t au = __shfl_up_sync(0xffffffffu, tl, 1 << s);
    take |= (lane >= (1 << s) && au == tl) ? (1u << s) : 0u;
  }
  const int32_t prev_tl = __shfl_up_sync(0xffffffffu, tl, 1);
  const int32_t next_hd = __shfl_down_sync(0xffffffffu, hd, 1);
  const int32_t first_id = __shfl_sync(0xffffffffu, hd, 0);
  const bool join_prev = lane > 0 && prev_tl == hd;  // head run continues the previous lane's tail
  const bool tail_end = lane == 31 || next_hd != tl;
#pragma unroll 1
  for (int j = 0; j < D; ++j) {
    // coordinates read as raw 64-bit patterns (NaNs keep their bits)
    const unsigned long long* __restrict__ Xj =
        reinterpret_cast<const unsigned long long*>(X) + (int64_t)j * n;
    unsigned long long kk[kItems];
    if (vec) {
#pragma unroll
      for (int h = 0; h < kItems / 2; ++h) {
        const ulonglong2 x = __ldg(reinterpret_cast<const ulonglong2*>(Xj + p0) + h);
        kk[2 * h] = dkey_bits(x.x);
        kk[2 * h + 1] = dkey_bits(x.y);
      }
    } else {
#pragma unroll
      for (int i = 0; i < kItems; ++i) kk[i] = a[i] >= 0 ? dkey_bits(Xj[p0 + i]) : 0ull;
    }
    unsigned long long hmn = kk[0], hmx = kk[0], cmn = kk[0], cmx = kk[0];
    int32_t ca = a[0];
    bool head_open = true;
#pragma unroll
    for (int i = 1; i < kItems; ++i) {
      if (brk & (1u << i)) {
        if (head_open) {
          hmn = cmn;
          hmx = cmx;
          head_open = false;
        } else if (ca >= 0) {  // a run that starts and ends inside this thread
          atomicMin(&keys[(int64_t)ca * 2 * D + 2 * j], cmn);
          atomicMax(&keys[(int64_t)ca * 2 * D + 2 * j + 1], cmx);
        }
        ca = a[i];
        cmn = kk[i];
        cmx = kk[i];
      } else {
        cmn = kk[i] < cmn ? kk[i] : cmn;
        cmx = kk[i] > cmx ? kk[i] : cmx;
      }
    }
    // segmented inclusive scan of the tail runs
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      const unsigned long long u = __shfl_up_sync(0xffffffffu, cmn, 1 << s);
      const unsigned long long v = __shfl_up_sync(0xffffffffu, cmx, 1 << s);
      if (take & (1u << s)) {
        cmn = u < cmn ? u : cmn;
        cmx = v > cmx ? v : cmx;
      }
    }
    const unsigned long long pmn = __shfl_up_sync(0xffffffffu, cmn, 1);
    const unsigned long long pmx = __shfl_up_sync(0xffffffffu, cmx, 1);
    // run ends: the head run when it ends inside this thread, the tail run when
    // the next lane starts another node (or at the end of the chunk)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      int32_t id;
      unsigned long long mn, mx;
      bool is_end;
      if (e == 0) {
        is_end = !single;
        id = hd;
        mn = hmn;
        mx = hmx;
        if (join_prev) {
          mn = pmn < mn ? pmn : mn;
          mx = pmx > mx ? pmx : mx;
        }
      } else {
        is_end = tail_end;
        id = tl;
        mn = cmn;
        mx = cmx;
      }
      if (!is_end) continue;
      if (id == first_id) {
        if (j == 0) rec_id[w][0] = id;
        rec_v[w][0][2 * j] = mn;
        rec_v[w][0][2 * j + 1] = mx;
        if (lane == 31 && e == 1 && j == 0) rec_id[w][1] = -2;  // one run spans the chunk
      } else if (e == 1 && lane == 31) {
        if (j == 0) rec_id[w][1] = id;
        rec_v[w][1][2 * j] = mn;
        rec_v[w][1][2 * j + 1] = mx;
      } else if (id >= 0) {
        atomicMin(&keys[(int64_t)id * 2 * D + 2 * j], mn);
        atomicMax(&keys[(int64_t)id * 2 * D + 2 * j + 1], mx);
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
    for (int c = 0; c < W; ++c) {
      for (int r = 0; r < 2; ++r) {
        const int32_t id = rec_id[c][r];
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
__global__ void k_decide(const int32_t* __restrict__ act, const int4* __restrict__ st,
                         NodeMeta* __restrict__ meta,
                         double* __restrict__ cell, double* __restrict__ box,
                         const unsigned long long* __restrict__ keys, int32_t* __restrict__ mode,
                         int32_t* __restrict__ ext, const int32_t* __restrict__ wst,
                         FlagRec* __restrict__ frec) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= st->x) return;
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
  FlagRec r;
  r.split = mid;
  r.axis = axis;
  r.md = md;
  r.wst = wst[a];
  r.count = meta[a].count;
  r.pad[0] = r.pad[1] = 0;
  frec[a] = r;
}

// Exclusive prefix, in position order, of one tile's 0/1 flags, visited as
// p = base + it * kBT + threadIdx.x: msk[it] is the warp's ballot of pass it.
// Leaves in cpre[it * W + w] the offset of warp w's 32 positions of pass it and
// returns the tile total.  Two barriers per tile.
__device__ __forceinline__ int32_t tile_chunk_prefix(const unsigned (&msk)[kItems],
                                                     int32_t* cpre) {
  constexpr int W = kBT / 32, NC = kItems * W;
  static_assert(NC == 64, "two warp chunks per lane in the chunk scan");
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int it = 0; it < kItems; ++it) cpre[it * W + w] = __popc(msk[it]);
  }
  __syncthreads();
  if (w == 0) {
    const int32_t x0 = cpre[2 * lane], x1 = cpre[2 * lane + 1], s = x0 + x1;
    const int32_t inc = warp_inclusive_scan(s);
    cpre[2 * lane] = inc - s;
    cpre[2 * lane + 1] = inc - s + x0;
    if (lane == 31) cpre[NC] = inc;
  }
  __syncthreads();
  return cpre[NC];
}

// Per-tile left counts and the segment-start / segment-end local prefixes of the
// midpoint splits (x < split goes left, cosmokdtree.f90:470).  A sliding split
// sends exactly one point, the first holding the extreme (:376-403), to the
// side that would be empty; its positions count 0 here and record that point.
// Each thread takes 8 consecutive positions (vector loads of the node ids and,
// when they all belong to one node, of that node's split coordinate), so the
// chain node id -> split record -> coordinate costs three loads per thread
// instead of three per position.  The left flags go to a bitmap (bit p & 31 of
// word p >> 5) that the scatter reads back.
__global__ void __launch_bounds__(kBT) k_flags(const double* __restrict__ X,
                                               const int32_t* __restrict__ NID,
                                               const FlagRec* __restrict__ frec,
                                               int32_t* __restrict__ ext, int64_t n,
                                               const int4* __restrict__ st,
                                               int32_t* __restrict__ tile_sum,
                                               int32_t* __restrict__ pstart,
                                               int32_t* __restrict__ pend,
                                               unsigned* __restrict__ flags) {
  static_assert(kItems == 8, "8 consecutive positions per thread");
  __shared__ int32_t tmp[kBT / 32];
  const int64_t nw = st->y;
  if ((int64_t)blockIdx.x * kTile >= nw) {  // past this level's working set
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = 0;
    return;
  }
  const int lane = threadIdx.x & 31;
  const int64_t p0 = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
  int32_t a[kItems];
  const bool full = p0 + kItems <= nw;
  const bool vec = full && (n & 1) == 0 && (reinterpret_cast<uintptr_t>(NID) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  if (vec) {
    const int4 u = __ldg(reinterpret_cast<const int4*>(NID + p0));
    const int4 v = __ldg(reinterpret_cast<const int4*>(NID + p0) + 1);
    a[0] = u.x, a[1] = u.y, a[2] = u.z, a[3] = u.w, a[4] = v.x, a[5] = v.y, a[6] = v.z, a[7] = v.w;
  } else {
#pragma unroll
    for (int i = 0; i < kItems; ++i) a[i] = p0 + i < nw ? NID[p0 + i] : -1;
  }
  bool single = a[0] >= 0;
#pragma unroll
  for (int i = 1; i < kItems; ++i) single = single && a[i] == a[0];
  unsigned f8 = 0, se = 0;  // left flags; segment start (bit 2i) and end (bit 2i+1)
  auto one = [&](int i, const FlagRec& r, double x) {
    const int64_t p = p0 + i;
    if (r.md == 0) f8 |= (x < r.split ? 1u : 0u) << i;
    else if (x == r.split) atomicMin(&ext[a[i]], (int32_t)p);
    if (p == r.wst) se |= 1u << (2 * i);
    if (p == (int64_t)r.wst + r.count - 1) se |= 2u << (2 * i);
  };
  if (single && vec) {
    const FlagRec r = frec[a[0]];
    const double2* xr = reinterpret_cast<const double2*>(X + (int64_t)r.axis * n + p0);
#pragma unroll
    for (int h = 0; h < kItems / 2; ++h) {
      const double2 x = __ldg(xr + h);
      one(2 * h, r, x.x);
      one(2 * h + 1, r, x.y);
    }
  } else {
    FlagRec r;
    int32_t ra = -1;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      if (a[i] < 0) continue;
      if (a[i] != ra) {
        r = frec[a[i]];
        ra = a[i];
      }
      one(i, r, X[(int64_t)r.axis * n + p0 + i]);
    }
  }
  int32_t tot;
  const int32_t ex = block_exclusive_scan<int32_t, kBT>(__popc(f8), tmp, tot);
  if (se) {
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      const unsigned b = (se >> (2 * i)) & 3u;
      if (b == 0) continue;
      const int32_t e = ex + __popc(f8 & ((1u << i) - 1u));
      if (b & 1u) pstart[a[i]] = e;
      if (b & 2u) pend[a[i]] = e + (int32_t)((f8 >> i) & 1u);
    }
  }
  // 4 lanes (32 positions) per bitmap word
  unsigned word = f8 << (8 * (lane & 3));
  word |= __shfl_xor_sync(0xffffffffu, word, 1);
  word |= __shfl_xor_sync(0xffffffffu, word, 2);
  if ((lane & 3) == 0) flags[p0 >> 5] = word;
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

// n_left, child pairs and cells; counts the next open list and its working
// points (cosmokdtree.f90:412-448)
template <int D>
__global__ void k_children(const int32_t* __restrict__ act, const int4* __restrict__ st, int mb,
                           NodeMeta* __restrict__ meta,
                           double* __restrict__ cell, const int32_t* __restrict__ pstart,
                           const int32_t* __restrict__ pend, const int32_t* __restrict__ tile_off,
                           const int32_t* __restrict__ wst, const int32_t* __restrict__ mode,
                           const int32_t* __restrict__ ext, int32_t* __restrict__ nleft,
                           int32_t* __restrict__ pbase, unsigned long long* __restrict__ keys,
                           int leaf, int64_t* __restrict__ nxt_cnt, int32_t* __restrict__ err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = st->x;
  const int32_t first_child = st->z;
  if (i >= m) {  // zeros up to the launch bound, so the scan over mb entries is exact
    if (i < mb) nxt_cnt[i] = 0;
    return;
  }
  int32_t a = act[i];
  NodeMeta pm = meta[a];
  const int md = mode[a];
  int32_t nl, P0 = 0;
  if (md == 0) {
    int64_t s = wst[a], e = (int64_t)wst[a] + pm.count - 1;
    P0 = tile_off[s / kTile] + pstart[a];
    int32_t P1 = tile_off[e / kTile] + pend[a];
    nl = P1 - P0;
  } else {
    nl = md == 1 ? 1 : pm.count - 1;
    if (ext[a] == 0x7fffffff) nl = 0;  // no slide point found: flagged below
  }
  if (nl <= 0 || nl >= pm.count) {  // cannot happen for a valid sliding-midpoint split
    atomicExch(err, 1);
    nl = nl <= 0 ? 1 : pm.count - 1;
  }
  nleft[a] = nl;
  pbase[a] = P0;
  int32_t c0 = first_child + 2 * i;
  meta[a].left = c0;
  int cnt = 0, pts = 0;
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
    if (cm.count > leaf) {
      ++cnt;
      pts += cm.count;
    }
  }
  nxt_cnt[i] = ((int64_t)cnt << 32) | (int64_t)pts;
}

// next open list (children in list order, so in leaf order) and their working starts
__global__ void k_next_list(const int32_t* __restrict__ act, const int4* __restrict__ st,
                            int4* __restrict__ st_next, int mb,
                            const NodeMeta* __restrict__ meta,
                            const int64_t* __restrict__ nxt_off, int leaf,
                            const int32_t* __restrict__ mode, const int32_t* __restrict__ ext,
                            const int32_t* __restrict__ nleft, const int32_t* __restrict__ pbase,
                            int32_t* __restrict__ nxt, int32_t* __restrict__ wst,
                            int4* __restrict__ srec) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int4 cs = *st;
  const int m = cs.x;
  if (i == 0) {  // the next level's state
    const int64_t tot = nxt_off[mb];
    *st_next = make_int4((int32_t)(tot >> 32), (int32_t)(tot & 0xffffffffll), cs.z + 2 * m,
                         cs.w + (m > 0 ? 1 : 0));
  }
  if (i >= m) return;
  const int32_t a = act[i];
  const NodeMeta pm = meta[a];
  const int32_t c0 = pm.left;
  int32_t o = (int32_t)(nxt_off[i] >> 32), w = (int32_t)(nxt_off[i] & 0xffffffffll);
  const int32_t n0 = meta[c0].count, n1 = meta[c0 + 1].count;
  const int md = mode[a];
  int32_t wl = md == 1 ? -2 : -1, wr = md == 2 ? -2 : -1;
  if (n0 > leaf) {
    nxt[o++] = c0;
    wst[c0] = w;
    wl = w;
    w += n0;
  }
  if (n1 > leaf) {
    nxt[o] = c0 + 1;
    wst[c0 + 1] = w;
    wr = w;
  }
  srec[2 * (int64_t)a] = make_int4(pm.start, wst[a], nleft[a], pm.count);
  srec[2 * (int64_t)a + 1] = make_int4(md == 0 ? pbase[a] : ext[a], c0, wl, wr);
}

// bulk asynchronous copies (global -> this CTA's shared memory) completing on an
// mbarrier; every wait is bounded
constexpr unsigned kBarWaitLimit = 1u << 24;
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ bool bar_wait0(uint32_t bar) {
  for (unsigned it = 0; it < kBarWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}" : "=r"(done) : "r"(bar), "r"(0u) : "memory");
    if (done) return true;
  }
  return false;
}

// scatter tile staging: dynamic shared memory of the staged scatter
__host__ __device__ constexpr size_t scatter_smem(int d) {
  return (size_t)d * kTile * sizeof(double) + (size_t)kTile * sizeof(int32_t);
}

// Stable partition of every open segment: points of open children go to the
// next working set, points of new leaves to the final leaf-ordered arrays.
// STAGED: the tile's coordinate rows and ids are brought into shared memory by
// bulk asynchronous copies issued at the start (one per row, 16-byte aligned
// because the working rows have an even stride), overlapping the first pass and
// the tile scan; the second pass then reads them from shared memory.
template <int D, bool STAGED>
__global__ void __launch_bounds__(kBT) k_scatter(
    const double* __restrict__ X, const int32_t* __restrict__ I, const int32_t* __restrict__ NID,
    const int4* __restrict__ srec, const int32_t* __restrict__ tile_off,
    const unsigned* __restrict__ flags, int64_t n, const int4* __restrict__ st,
    double* __restrict__ Xo,
    int32_t* __restrict__ Io, int32_t* __restrict__ NIDo, double* __restrict__ Pf,
    int32_t* __restrict__ If, int32_t* __restrict__ err) {
  constexpr int W = kBT / 32;
  __shared__ int32_t cpre[kItems * W + 1];
  __shared__ __align__(8) unsigned long long bar;
  extern __shared__ __align__(16) unsigned char stage[];
  double* sx = reinterpret_cast<double*>(stage);
  int32_t* si = reinterpret_cast<int32_t*>(stage + (size_t)D * kTile * sizeof(double));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kTile;
  const int64_t nw = st->y;
  if (base >= nw) return;  // past this level's working set (the whole block)
  if (STAGED) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int64_t cnt = min((int64_t)kTile, nw - base);
      const uint32_t bx = (uint32_t)(((cnt + 1) & ~1ll) * 8), bi = (uint32_t)(((cnt + 3) & ~3ll) * 4);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&bar)),
                   "r"(D * bx + bi)
                   : "memory");
#pragma unroll
      for (int j = 0; j < D; ++j)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(smem_u32(sx + j * kTile)),
            "l"(X + (int64_t)j * n + base), "r"(bx), "r"(smem_u32(&bar))
            : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
          "[%3];" ::"r"(smem_u32(si)),
          "l"(I + base), "r"(bi), "r"(smem_u32(&bar))
          : "memory");
    }
  }
  unsigned msk[kItems];
  int32_t av[kItems];
#pragma unroll
  for (int it = 0; it < kItems; ++it) {
    const int64_t p = base + (int64_t)it * kBT + threadIdx.x;
    av[it] = p < nw ? NID[p] : -1;
    msk[it] = flags[(base >> 5) + it * W + w];  // the flag pass's ballot of these 32 positions
  }
  tile_chunk_prefix(msk, cpre);
  if (STAGED && !bar_wait0(smem_u32(&bar))) {
    atomicExch(err, 3);             // copies did not land: report, let them finish, leave
    bar_wait0(smem_u32(&bar));
    return;
  }
  const int32_t run = tile_off[blockIdx.x];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int it = 0; it < kItems; ++it) {
    const int32_t a = av[it];
    if (a < 0) continue;
    const int64_t p = base + (int64_t)it * kBT + threadIdx.x;
    const int4 r0 = srec[2 * (int64_t)a], r1 = srec[2 * (int64_t)a + 1];
    const int32_t start = r0.x, nl = r0.z, count = r0.w;
    const int32_t q = (int32_t)(p - r0.y);  // position in the segment
    int f;
    int32_t rank;  // rank in the child
    if (r1.z == -2 || r1.w == -2) {  // the slide point alone on one side, the others keep their order
      const bool sp = p == r1.x;
      f = (r1.z == -2) == sp ? 1 : 0;
      rank = sp ? 0 : q - (p > r1.x ? 1 : 0);
    } else {
      f = (int)((msk[it] >> lane) & 1u);
      const int32_t ex = run + cpre[it * W + w] + __popc(msk[it] & lt);
      const int32_t rl = ex - r1.x;  // left points before p in the segment
      rank = f ? rl : q - rl;
    }
    const int32_t ccount = f ? nl : count - nl;
    if (rank < 0 || rank >= ccount) {  // never for a consistent scan
      atomicExch(err, 2);
      continue;
    }
    const int t = (int)(p - base);
    const int32_t id = STAGED ? si[t] : I[p];
    double xv[D];
#pragma unroll
    for (int j = 0; j < D; ++j) xv[j] = STAGED ? sx[j * kTile + t] : X[(int64_t)j * n + p];
    const int32_t wc = f ? r1.z : r1.w;  // child's working start, negative for a leaf
    if (wc < 0) {
      const int64_t dst = (int64_t)start + (f ? 0 : nl) + rank;
#pragma unroll
      for (int j = 0; j < D; ++j) Pf[(int64_t)j * n + dst] = xv[j];
      If[dst] = id;
    } else {
      const int64_t wd = (int64_t)wc + rank;
#pragma unroll
      for (int j = 0; j < D; ++j) Xo[(int64_t)j * n + wd] = xv[j];
      Io[wd] = id;
      NIDo[wd] = r1.y + (f ? 0 : 1);
    }
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

// Absolute coordinates rounded to FP32, packed in float4s (zero padded).
template <int D>
__global__ void k_pts32(const double* __restrict__ Pf, int64_t n, float4* __restrict__ P32) {
  constexpr int NV = (D + 3) / 4;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  float v[4 * NV];
#pragma unroll
  for (int j = 0; j < 4 * NV; ++j) v[j] = j < D ? __double2float_rn(Pf[(int64_t)(j < D ? j : 0) * n + p]) : 0.0f;
#pragma unroll
  for (int h = 0; h < NV; ++h)
    P32[p * NV + h] = make_float4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
}

// Search records: inward-rounded FP32 cells, FP64 leaf centres, and for each
// internal node the child-pair record (both children's outward FP32 boxes, ids,
// leaf flags and position ranges) so one load serves a whole expansion.
template <int D>
__global__ void k_search_records(const NodeMeta* __restrict__ meta, int32_t n_nodes,
                                 const double* __restrict__ box, const double* __restrict__ cell,
                                 float4* __restrict__ pair, float* __restrict__ cell32,
                                 double* __restrict__ centre) {
  constexpr int NV = (D + 3) / 4;
  constexpr int PF = pair_f4(D);
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
  const NodeMeta ml = meta[m.left], mr = meta[m.left + 1];
  int4 info = make_int4(m.left, m.left + 1, ml.left < 0 ? 1 : 0, mr.left < 0 ? 1 : 0);
  rec[4 * NV] = *reinterpret_cast<float4*>(&info);
  int4 range = make_int4(ml.start, ml.count, mr.start, mr.count);
  rec[4 * NV + 1] = *reinterpret_cast<float4*>(&range);
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
  CKD_CUDA(grow(&B.wst, B.cap, nc, s));
  CKD_CUDA(grow(&B.frec, B.cap, nc, s));
  CKD_CUDA(grow(&B.srec, B.cap * 2, nc * 2, s));
  B.cap = nc;
  return CKD_OK;
}

void free_bufs(BuildBufs& B, cudaStream_t s) {
  void* ps[] = {B.X[0],   B.X[1],    B.I[0],      B.I[1],     B.NID[0],  B.NID[1], B.meta,
                B.cell,   B.box,     B.keys,      B.ext,      B.mode,    B.pstart, B.pend,
                B.nleft,  B.pbase,   B.wst,       B.act[0],   B.act[1],  B.nxt_cnt, B.nxt_off,
                B.tile_sum, B.tile_off, B.scal, B.flags, B.frec, B.srec, B.lst};
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
    CKD_CUDA(dev_alloc((void**)&B.I[b], sizeof(int32_t) * (n + 4), s));  // + the copy's rounding
    CKD_CUDA(dev_alloc((void**)&B.NID[b], sizeof(int32_t) * n, s));
  }
  int64_t max_open = n / (leaf + 1) + 2 + t->n_trees;
  for (int b = 0; b < 2; ++b) CKD_CUDA(dev_alloc((void**)&B.act[b], sizeof(int32_t) * max_open, s));
  CKD_CUDA(dev_alloc((void**)&B.nxt_cnt, sizeof(int64_t) * max_open, s));
  CKD_CUDA(dev_alloc((void**)&B.nxt_off, sizeof(int64_t) * (max_open + 1), s));
  CKD_CUDA(dev_alloc((void**)&B.tile_sum, sizeof(int32_t) * ntiles, s));
  CKD_CUDA(dev_alloc((void**)&B.tile_off, sizeof(int32_t) * (ntiles + 1), s));
  CKD_CUDA(dev_alloc((void**)&B.flags, sizeof(unsigned) * ntiles * (kTile / 32), s));
  CKD_CUDA(dev_alloc((void**)&B.scal, sizeof(int32_t) * 4, s));
  CKD_CUDA(dev_alloc((void**)&B.lst, sizeof(int4) * 2, s));
  CKD_CUDA(cudaMemsetAsync(B.scal, 0, sizeof(int32_t) * 4, s));

  // final outputs
  CKD_CUDA(dev_alloc((void**)&t->pts, sizeof(double) * D * n, s));
  CKD_CUDA(dev_alloc((void**)&t->ids, sizeof(int32_t) * n, s));

  // trees of a forest: positions off[t] .. off[t+1]-1, root node t
  const int32_t T = (int32_t)t->n_trees;
  const std::vector<int64_t>& off = t->tree_off;
  Scratch sc(s);  // small per-build buffers (tree offsets, box sides)
  int64_t* off_dev = nullptr;
  CKD_CUDA(sc.alloc(&off_dev, sizeof(int64_t) * (T + 1)));
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
  CKD_CUDA(sc.alloc(&Ldev, sizeof(double) * CKD_MAX_D));
  CKD_CUDA(cudaMemcpyAsync(Ldev, t->L, sizeof(double) * CKD_MAX_D, cudaMemcpyHostToDevice, s));
  CKD_TRY(ensure_node_cap(B, (int64_t)T + std::max<int64_t>(64, 4 * (n / std::max(1, leaf)) + 64), s));
  k_root_init<D><<<(unsigned)cdiv(T, 128), 128, 0, s>>>(B.meta, B.cell, B.keys, off_dev, T, Ldev,
                                                        t->periodic);
  CKD_LAUNCH_CHECK();

  // Root bounding boxes: validation (finite, inside the periodic box) and the
  // non-periodic root cells, from the segmented reduction over every point
  // (position p belongs to root NID[p]).
  k_seg_box<D><<<(unsigned)ntiles, kBT, 0, s>>>(B.X[0], B.NID[0], n, n, B.keys);
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
      if (!std::isfinite(lo) || !std::isfinite(hi))
        return fail(CKD_ERR_BAD_ARG, "points contain NaN or infinite coordinates");
      if (t->periodic && (lo < -t->L[j] / 2 || hi > t->L[j] / 2))
        return fail(CKD_ERR_OUT_OF_BOX, "Points outside (-L/2, L/2) range");
      rlo[j] = std::min(rlo[j], lo);
      rhi[j] = std::max(rhi[j], hi);
    }
  }
  if (!t->periodic) {
    k_root_cells<D><<<(unsigned)cdiv(T, 128), 128, 0, s>>>(B.cell, B.keys, T);
    CKD_LAUNCH_CHECK();
  }
  // open roots and the first working set
  std::vector<int32_t> roots;
  std::vector<int32_t> wst0((size_t)T, -1);
  int64_t nw = 0;
  for (int32_t tr = 0; tr < T; ++tr)
    if (off[tr + 1] - off[tr] > leaf) {
      roots.push_back(tr);
      wst0[tr] = (int32_t)nw;
      nw += off[tr + 1] - off[tr];
    }
  int cur = 0;
  if (nw < n) {
    // points of trees that are a single leaf never move: start from the input order
    CKD_CUDA(cudaMemcpyAsync(t->pts, B.X[0], sizeof(double) * D * n, cudaMemcpyDeviceToDevice, s));
    CKD_CUDA(cudaMemcpyAsync(t->ids, B.I[0], sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
  }
  CKD_CUDA(cudaMemcpyAsync(B.wst, wst0.data(), sizeof(int32_t) * T, cudaMemcpyHostToDevice, s));
  if (nw < n && nw > 0) {
    k_compact_roots<D><<<(unsigned)cdiv(n, 256), 256, 0, s>>>(B.X[0], B.I[0], B.NID[0], B.wst,
                                                             off_dev, n, B.X[1], B.I[1], B.NID[1]);
    CKD_LAUNCH_CHECK();
    cur = 1;
  }
  if (!roots.empty())
    CKD_CUDA(cudaMemcpyAsync(B.act[0], roots.data(), sizeof(int32_t) * roots.size(),
                             cudaMemcpyHostToDevice, s));
  CKD_CUDA(cudaStreamSynchronize(s));  // `roots`, `wst0` and `rk` are host buffers of the copies

  // the staged scatter needs 16-byte aligned rows (even stride) and fits D <= 4
  // (<= 72 KB of shared memory per block)
  const bool staged = D <= 4 && (n & 1) == 0;
  if (staged)
    CKD_CUDA(cudaFuncSetAttribute(k_scatter<D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)scatter_smem(D)));
  // pinned word for the readback of the level state
  static thread_local int4* level_st = nullptr;
  if (!level_st) CKD_CUDA(cudaMallocHost((void**)&level_st, sizeof(int4)));
  // Levels run ahead of the host: a chunk of up to kRunAhead levels is launched
  // with grids sized by bounds known at the last readback (the working set never
  // grows; a level has at most twice the previous level's open nodes and at most
  // nw / (leaf + 1) of them), every kernel reads the exact counts from the
  // device state and idles past them, and the host reads the state once per
  // chunk.  Levels after the last open node are no-ops.
  constexpr int kRunAhead = 6;
  int32_t n_nodes = T;
  int64_t m = (int64_t)roots.size();
  *level_st = make_int4((int32_t)m, (int32_t)nw, n_nodes, 0);
  CKD_CUDA(cudaMemcpyAsync(B.lst, level_st, sizeof(int4), cudaMemcpyHostToDevice, s));
  int depth_levels = 0;
  int par = 0;    // state slot of the next level
  int alist = 0;  // open list buffer of the next level
  int level = 0;  // levels launched
  while (m > 0) {
    if (level >= kMaxLevels)
      return fail(CKD_ERR_DEPTH, "tree depth exceeds the build's level cap (8192 levels)");
    int64_t mb[kRunAhead];
    mb[0] = m;
    int64_t grow = 2 * m;
    int S = 1;
    for (int c = 1; c < kRunAhead && level + c < kMaxLevels; ++c) {
      mb[c] = std::min<int64_t>(2 * mb[c - 1], nw / (leaf + 1));
      if (n_nodes + grow + 2 * mb[c] > B.cap) break;
      grow += 2 * mb[c];
      S = c + 1;
    }
    CKD_TRY(ensure_node_cap(B, (int64_t)n_nodes + grow, s));
    const unsigned ntw = (unsigned)cdiv(nw, kTile);
    for (int c = 0; c < S; ++c, ++level) {
      const int4* st = B.lst + par;
      int4* st_next = B.lst + (1 - par);
      const int32_t* act = B.act[alist];
      const int mbi = (int)std::max<int64_t>(1, mb[c]);
      const unsigned gm = (unsigned)cdiv(mbi, 128);
      if (level > 0) {  // the roots' boxes come from the validation pass
        k_seg_box<D><<<ntw, kBT, 0, s>>>(B.X[cur], B.NID[cur], n, nw, B.keys, st);
        CKD_LAUNCH_CHECK();
      }
      k_decide<D><<<gm, 128, 0, s>>>(act, st, B.meta, B.cell, B.box, B.keys, B.mode, B.ext, B.wst,
                                     B.frec);
      CKD_LAUNCH_CHECK();
      k_flags<<<ntw, kBT, 0, s>>>(B.X[cur], B.NID[cur], B.frec, B.ext, n, st, B.tile_sum,
                                  B.pstart, B.pend, B.flags);
      CKD_LAUNCH_CHECK();
      CKD_TRY(scan_i32(B.tile_sum, B.tile_off, ntw, s));
      k_children<D><<<gm, 128, 0, s>>>(act, st, mbi, B.meta, B.cell, B.pstart, B.pend, B.tile_off,
                                       B.wst, B.mode, B.ext, B.nleft, B.pbase, B.keys, leaf,
                                       B.nxt_cnt, B.scal + 1);
      CKD_LAUNCH_CHECK();
      CKD_TRY(scan_i64(B.nxt_cnt, B.nxt_off, mbi, s));
      k_next_list<<<gm, 128, 0, s>>>(act, st, st_next, mbi, B.meta, B.nxt_off, leaf, B.mode, B.ext,
                                     B.nleft, B.pbase, B.act[1 - alist], B.wst, B.srec);
      CKD_LAUNCH_CHECK();
      if (staged)
        k_scatter<D, true><<<ntw, kBT, scatter_smem(D), s>>>(
            B.X[cur], B.I[cur], B.NID[cur], B.srec, B.tile_off, B.flags, n, st, B.X[1 - cur],
            B.I[1 - cur], B.NID[1 - cur], t->pts, t->ids, B.scal + 1);
      else
        k_scatter<D, false><<<ntw, kBT, 0, s>>>(B.X[cur], B.I[cur], B.NID[cur], B.srec,
                                                B.tile_off, B.flags, n, st, B.X[1 - cur],
                                                B.I[1 - cur], B.NID[1 - cur], t->pts, t->ids,
                                                B.scal + 1);
      CKD_LAUNCH_CHECK();
      cur = 1 - cur;
      alist = 1 - alist;
      par = 1 - par;
    }
    CKD_CUDA(cudaMemcpyAsync(level_st, B.lst + par, sizeof(int4), cudaMemcpyDeviceToHost, s));
    CKD_CUDA(cudaStreamSynchronize(s));
    m = level_st->x;
    nw = level_st->y;
    n_nodes = level_st->z;
    depth_levels = level_st->w;
  }
  int32_t err = 0;
  CKD_CUDA(cudaMemcpyAsync(&err, B.scal + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));

  k_leaf_box<D><<<(unsigned)cdiv(n_nodes, 128), 128, 0, s>>>(B.meta, n_nodes, leaf, t->pts, n,
                                                             B.box);
  CKD_LAUNCH_CHECK();
  t->n_nodes = n_nodes;
  t->depth = depth_levels;
  CKD_CUDA(dev_alloc((void**)&t->meta, sizeof(NodeMeta) * n_nodes, s));
  CKD_CUDA(dev_alloc((void**)&t->box, sizeof(double) * 2 * D * n_nodes, s));
  CKD_CUDA(dev_alloc((void**)&t->cell, sizeof(double) * 2 * D * n_nodes, s));
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
  CKD_CUDA(dev_alloc((void**)&t->box32, sizeof(float) * 2 * D * n_nodes, s));
  CKD_CUDA(dev_alloc((void**)&t->pts32, sizeof(float4) * NV * n, s));
  CKD_CUDA(dev_alloc((void**)&t->pts64, sizeof(double4) * NV * n, s));
  k_pts64<D><<<(unsigned)cdiv(n, 256), 256, 0, s>>>(t->pts, n, t->pts64);
  CKD_LAUNCH_CHECK();
  k_pts32<D><<<(unsigned)cdiv(n, 256), 256, 0, s>>>(t->pts, n, t->pts32);
  CKD_LAUNCH_CHECK();
  k_box32<D><<<(unsigned)cdiv((int64_t)n_nodes * 2 * D, 256), 256, 0, s>>>(t->box, n_nodes, t->box32);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(dev_alloc((void**)&t->pair, sizeof(float4) * pair_f4(D) * n_nodes, s));
  CKD_CUDA(dev_alloc((void**)&t->cell32, sizeof(float) * 2 * D * n_nodes, s));
  CKD_CUDA(dev_alloc((void**)&t->centre, sizeof(double) * D * n_nodes, s));
  k_search_records<D><<<(unsigned)cdiv(n_nodes, 128), 128, 0, s>>>(
      t->meta, n_nodes, t->box, t->cell, t->pair, t->cell32, t->centre);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(cudaStreamSynchronize(s));
  if (err == 3) return fail(CKD_ERR_TIMEOUT, "build: a tile copy into shared memory timed out");
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
